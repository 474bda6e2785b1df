"""CPU tests of the block-set builders: topology, node continuity, BC arrays."""
import numpy as np

from cffc_b200 import cases


def test_periodic_neighbours_are_mutual():
    bs = cases.periodic_box_bumps(nb=3, nc=4)
    opposite = [1, 0, 3, 2, 7, 6, 5, 4]
    for b in range(bs.nblk):
        for k in range(8):
            n = bs.neighbour[b, k]
            assert n >= 0
            assert bs.neighbour[n, opposite[k]] == b


def test_interior_nodes_match_across_block_edges():
    bs = cases.curvilinear_mach2(nbi=3, nbj=2, nc=6, seed=2)
    g = bs.ng
    for b in range(bs.nblk):
        e = bs.neighbour[b, 1]
        if e < 0 or e < b:
            continue
        # east edge nodes of b == west edge nodes of e (up to the periodic shift)
        xb = bs.node_x[b, g:g + bs.ncj + 1, g + bs.nci]
        xe = bs.node_x[e, g:g + bs.ncj + 1, g]
        assert np.allclose(xb, xe)


def test_channel_bc_arrays_and_no_wraparound():
    bs = cases.channel(nbi=3, nbj=2)
    assert (bs.neighbour[0, [0, 2, 4, 5, 6]] == -1).all()
    assert (bs.bc_w[0] == cases.BC_FIXED).all()
    assert (bs.bc_w[1] == cases.BC_NONE).all()
    assert (bs.bc_s[0] == cases.BC_REFLECTION).all()
    assert (bs.bc_n[bs.nblk - 1] == cases.BC_REFLECTION).all()


def test_case_file_roundtrip_size(tmp_path):
    bs = cases.channel()
    p = tmp_path / "c.bin"
    cases.write_case(str(p), bs)
    per_block = (8 + 2 * bs.NCj + 2 * bs.NCi) * 4 + 8 * (2 * (bs.NCi + 1) * (bs.NCj + 1)
                                                           + 8 * bs.NCj + 8 * bs.NCi + 4 * bs.NCi * bs.NCj)
    assert p.stat().st_size == 8 + 16 + 32 + 32 + 16 + bs.nblk * per_block

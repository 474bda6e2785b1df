"""Test infrastructure only (the library never imports it): a restatement
of BPKIT's symbolic ILU(k) factorization, symbolic_ilu
(bpkit/src/SparseUtil.cc:198-330), on the block matrix the reference's
Block_Preconditioner builds (Setup_Jacobian_approximation and
Get_Block_Index, NewtonKrylovSchwarz2D/Block_Preconditioner2D.h:180-345):
one block row per cell of the NCi x NCj block (ghost cells included),
five-point stencil.  Pure Python; meant for small blocks.

symbolic_ilu keeps each row as a sorted linked list of columns with a level
per entry (0 for A's entries).  It walks the row's columns below the
diagonal in ascending order, including fill added on the way; for each such
column k it merges U(k) past its diagonal into the row: a column j already
present takes min(level, lev(i,k) + lev(k,j) + 1), an absent one is added
when that sum is at most the level of fill."""


def full_pattern(NCi, NCj, level):
    """Rows of the full block matrix: list of (column, level) sorted."""
    n = NCi * NCj
    rows = []
    upper = []  # per row: [(col, lev)] for col >= row, diagonal first
    for i in range(n):
        # Get_Block_Index order N, E, C, W, S; entries outside the matrix dropped
        cols = [i - NCi, i - 1 if i % NCi != 0 else -1, i, i + 1 if (i + 1) % NCi != 0 else -1, i + NCi]
        lev = {j: 0 for j in cols if 0 <= j < n}
        k = min(lev)
        while k < i:
            lk = lev[k]
            for j, lkj in upper[k][1:]:
                nl = lk + lkj + 1
                if j in lev:
                    lev[j] = min(lev[j], nl)
                elif nl <= level:
                    lev[j] = nl
            k = min((c for c in lev if c > k), default=i)
        row = sorted(lev.items())
        rows.append(row)
        upper.append([(j, l) for j, l in row if j >= i])
    return rows


def interior_pattern(nci, ncj, level):
    """(row_ptr, col) of the pattern restricted to interior cells (two ghost
    layers), interior index y * nci + x."""
    NCi, NCj = nci + 4, ncj + 4
    rows = full_pattern(NCi, NCj, level)

    def interior(f):
        x, y = f % NCi, f // NCi
        return (y - 2) * nci + (x - 2) if 2 <= x < NCi - 2 and 2 <= y < NCj - 2 else -1

    row_ptr, col = [0], []
    for f in range(NCi * NCj):
        if interior(f) < 0:
            continue
        col += [interior(c) for c, _ in rows[f] if interior(c) >= 0]
        row_ptr.append(len(col))
    return row_ptr, col

// Test driver of the C++ host layer (include/cffc_euler2d.hpp), built by the
// tests against libcffc_e2d.so.
//
//   host_driver parse DECK CASE_OUT             deck -> blocks -> case file (no GPU)
//   host_driver run DECK CASE_OUT STATE_OUT     + explicit steps / Newton-Krylov on the GPU;
//                                               final W as [nblk][4][NCj][NCi] doubles
//   host_driver residual1 DECK OUT              single-block dUdt_Residual_Evaluation and
//                                               CFL of every block of the deck's set after a
//                                               multi-block ghost fill; writes per block
//                                               dUdt (single), dUdt (multi), dt (single)
//
// Prints one line "ok <n ignored keywords> <Wo.d> <Wo.u> <Wo.p>" on success.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cffc_euler2d.hpp"

using namespace cffc_b200;

static void write_W(FILE* f, const std::vector<Euler2D_Quad_Block>& blocks) {
  for (const auto& B : blocks)
    for (int v = 1; v <= 4; ++v)
      for (int j = 0; j < B.NCj; ++j)
        for (int i = 0; i < B.NCi; ++i) fwrite(&B.W[i][j][v], sizeof(double), 1, f);
}

static void write_R(FILE* f, const Euler2D_Quad_Block& B) {
  for (int v = 1; v <= 4; ++v)
    for (int j = 0; j < B.NCj; ++j)
      for (int i = 0; i < B.NCi; ++i) fwrite(&B.dUdt[i][j][v], sizeof(double), 1, f);
}

// The block set of a case file (the layout cffc_b200.cases.write_case writes),
// with U = U(W) as the reference's harness sets it.
static bool read_case(const char* path, std::vector<Euler2D_Quad_Block>& blocks, std::vector<int>& neighbour,
                      Euler2D_Input_Parameters& IP) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  int hdr[2], dims[4], opts[8];
  double dopts[4];
  bool ok = fread(hdr, 4, 2, f) == 2 && fread(dims, 4, 4, f) == 4 && fread(opts, 4, 8, f) == 8 &&
            fread(dopts, 8, 4, f) == 4;
  int opts2[4] = {0, 2, 0, 0};
  if (ok && hdr[1] == 2) ok = fread(opts2, 4, 4, f) == 4;  // version 2: scheme extras
  const int nblk = dims[0], nci = dims[1], ncj = dims[2], ng = dims[3];
  const int NCi = nci + 2 * ng, NCj = ncj + 2 * ng, NNi = NCi + 1, NNj = NCj + 1;
  IP.Number_of_Blocks_Idir = opts[5];
  IP.Number_of_Blocks_Jdir = opts[6];
  IP.Grid_Type = opts[7] ? "Periodic_Box" : "Rectangular_Box";
  blocks.assign(nblk, Euler2D_Quad_Block());
  neighbour.assign(size_t(8) * nblk, -1);
  auto rd = [&](void* p, size_t sz, size_t n) { ok = ok && fread(p, sz, n, f) == n; };
  for (int b = 0; ok && b < nblk; ++b) {
    Euler2D_Quad_Block& B = blocks[b];
    B.allocate(nci, ncj, ng);
    rd(&neighbour[8 * b], 4, 8);
    std::vector<int> bc(2 * NCj + 2 * NCi);
    rd(bc.data(), 4, bc.size());
    for (int j = 0; j < NCj; ++j) { B.Grid.BCtypeW[j] = bc[j]; B.Grid.BCtypeE[j] = bc[NCj + j]; }
    for (int i = 0; i < NCi; ++i) { B.Grid.BCtypeS[i] = bc[2 * NCj + i]; B.Grid.BCtypeN[i] = bc[2 * NCj + NCi + i]; }
    std::vector<double> xy(2 * NNi * NNj);
    rd(xy.data(), 8, xy.size());
    for (int j = 0; j < NNj; ++j)
      for (int i = 0; i < NNi; ++i) B.Grid.Node[i][j] = Vector2D(xy[j * NNi + i], xy[NNi * NNj + j * NNi + i]);
    std::vector<Euler2D_pState>* wo[4] = {&B.WoW, &B.WoE, &B.WoS, &B.WoN};
    const int L[4] = {NCj, NCj, NCi, NCi};
    for (int e = 0; e < 4; ++e) {
      std::vector<double> w(4 * L[e]);
      rd(w.data(), 8, w.size());
      for (int k = 0; k < L[e]; ++k) (*wo[e])[k] = Euler2D_pState(w[k], w[L[e] + k], w[2 * L[e] + k], w[3 * L[e] + k]);
    }
    std::vector<double> W(4 * NCi * NCj);
    rd(W.data(), 8, W.size());
    const int s = NCi * NCj;
    for (int j = 0; j < NCj; ++j)
      for (int i = 0; i < NCi; ++i) {
        const int q = j * NCi + i;
        B.W[i][j] = Euler2D_pState(W[q], W[s + q], W[2 * s + q], W[3 * s + q]);
        B.U[i][j] = B.W[i][j].U();
      }
  }
  fclose(f);
  return ok;
}

// The restart test modes (no deck):
//   host_driver restart_write CASE PREFIX NSTEPS TIME   Write_QuadTree + Write_Restart_Solution
//   host_driver restart_read PREFIX OUT                 Read_QuadTree + Read_Restart_Solution; OUT in
//                                                       the layout of the reference harness's
//                                                       restart_read
static int restart_modes(int argc, char** argv) {
  const std::string mode = argv[1];
  Euler2D_Input_Parameters IP;
  std::vector<Euler2D_Quad_Block> blocks;
  std::vector<int> neighbour;
  if (mode == "grid_write") {
    if (!read_case(argv[2], blocks, neighbour, IP)) return 2;
    if (Write_Multi_Block_Grid(argv[3], blocks, IP)) return 5;
    printf("ok\n");
    return 0;
  }
  if (mode == "grid_read") {
    // nodes X, Y of every block, then BC codes W E S N, then neighbours [nblk][8]
    std::string type;
    if (Read_Multi_Block_Grid(argv[2], blocks, neighbour, &type)) return 5;
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 10;
    for (const Euler2D_Quad_Block& B : blocks) {
      for (int j = 0; j < B.Grid.NNj; ++j)
        for (int i = 0; i < B.Grid.NNi; ++i) fwrite(&B.Grid.Node[i][j].x, 8, 1, f);
      for (int j = 0; j < B.Grid.NNj; ++j)
        for (int i = 0; i < B.Grid.NNi; ++i) fwrite(&B.Grid.Node[i][j].y, 8, 1, f);
    }
    for (const Euler2D_Quad_Block& B : blocks) {
      fwrite(B.Grid.BCtypeW.data(), 4, B.NCj, f);
      fwrite(B.Grid.BCtypeE.data(), 4, B.NCj, f);
      fwrite(B.Grid.BCtypeS.data(), 4, B.NCi, f);
      fwrite(B.Grid.BCtypeN.data(), 4, B.NCi, f);
    }
    fwrite(neighbour.data(), 4, neighbour.size(), f);
    fclose(f);
    printf("ok %s %zu\n", type.c_str(), blocks.size());
    return 0;
  }
  if (mode == "restart_write") {
    if (argc < 6 || !read_case(argv[2], blocks, neighbour, IP)) return 2;
    IP.Restart_File_Name = std::string(argv[3]) + ".soln";
    if (Write_QuadTree(blocks, neighbour, IP) || Write_Restart_Solution(blocks, IP, atoi(argv[4]), atof(argv[5]), 1.5))
      return 5;
    printf("ok\n");
    return 0;
  }
  IP.Restart_File_Name = std::string(argv[2]) + ".soln";
  int nsteps = 0;
  double time = 0.0, cpu = 0.0;
  if (Read_QuadTree(blocks, neighbour, IP) || Read_Restart_Solution(blocks, IP, nsteps, time, cpu)) return 5;
  FILE* f = fopen(argv[3], "wb");
  if (!f) return 10;
  const int hdr[2] = {nsteps, static_cast<int>(blocks.size())};
  fwrite(hdr, 4, 2, f);
  fwrite(&time, 8, 1, f);
  fwrite(&cpu, 8, 1, f);
  for (size_t b = 0; b < blocks.size(); ++b) {
    const Euler2D_Quad_Block& B = blocks[b];
    const int* nb = &neighbour[8 * b];
    const int rec[9] = {static_cast<int>(b), nb[0] >= 0, nb[1] >= 0, nb[2] >= 0, nb[3] >= 0, nb[0], nb[1], nb[2], nb[3]};
    fwrite(rec, 4, 9, f);
    for (int j = 0; j < B.NCj; ++j) fwrite(&B.Grid.BCtypeW[j], 4, 1, f);
    for (int j = 0; j < B.NCj; ++j) fwrite(&B.Grid.BCtypeE[j], 4, 1, f);
    for (int i = 0; i < B.NCi; ++i) fwrite(&B.Grid.BCtypeS[i], 4, 1, f);
    for (int i = 0; i < B.NCi; ++i) fwrite(&B.Grid.BCtypeN[i], 4, 1, f);
    for (int j = 0; j < B.Grid.NNj; ++j)
      for (int i = 0; i < B.Grid.NNi; ++i) fwrite(&B.Grid.Node[i][j].x, 8, 1, f);
    for (int j = 0; j < B.Grid.NNj; ++j)
      for (int i = 0; i < B.Grid.NNi; ++i) fwrite(&B.Grid.Node[i][j].y, 8, 1, f);
    const std::vector<Euler2D_pState>* wo[4] = {&B.WoW, &B.WoE, &B.WoS, &B.WoN};
    for (int e = 0; e < 4; ++e)
      for (int v = 1; v <= 4; ++v)
        for (const Euler2D_pState& w : *wo[e]) fwrite(&w[v], 8, 1, f);
    for (int v = 1; v <= 4; ++v)
      for (int j = 0; j < B.NCj; ++j)
        for (int i = 0; i < B.NCi; ++i) fwrite(&B.U[i][j][v], 8, 1, f);
  }
  fclose(f);
  printf("ok %d\n", nsteps);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: host_driver parse|run|residual1 DECK OUT [STATE_OUT]\n");
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "restart_write" || mode == "restart_read" || mode == "grid_write" || mode == "grid_read")
    return restart_modes(argc, argv);
  Euler2D_Input_Parameters IP;
  const int line = IP.Process_Input_Control_Parameter_File(argv[2]);
  if (line) {
    printf("error line %d\n", line);
    return 3;
  }
  std::vector<Euler2D_Quad_Block> blocks;
  std::vector<int> neighbour;
  if (Create_Initial_Solution_Blocks(IP, blocks, neighbour)) {
    printf("error blocks\n");
    return 4;
  }
  if (mode == "parse" || mode == "run") {
    if (Write_Case_File(argv[3], blocks, neighbour, IP)) return 5;
  }
  if (mode == "run") {
    if (argc < 5) return 2;
    Euler2D_Device_Blocks dev(blocks, neighbour, IP);
    if (!dev.handle()) return 6;
    std::vector<double> hist;
    if (IP.Maximum_Number_of_Time_Steps > 0 && dev.explicit_steps(IP.Maximum_Number_of_Time_Steps, &hist)) return 7;
    std::vector<e2d_nks_step> nh;
    if (IP.NKS.max_newton > 0 && dev.nks(IP.NKS, &nh)) return 8;
    if (dev.download()) return 9;
    FILE* f = fopen(argv[4], "wb");
    if (!f) return 10;
    write_W(f, blocks);
    fclose(f);
  }
  if (mode == "residual1") {
    // ghost cells of every block from the multi-block exchange + BCs
    Euler2D_Device_Blocks dev(blocks, neighbour, IP);
    if (!dev.handle() || dev.residual() || dev.download()) return 11;
    std::vector<Euler2D_Quad_Block> multi = blocks;  // dUdt of the multi-block residual
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 10;
    for (size_t b = 0; b < blocks.size(); ++b) {
      Euler2D_Quad_Block one = blocks[b];
      if (dUdt_Residual_Evaluation(one, IP)) return 12;
      const double dtmin = CFL(one, IP);
      if (dtmin <= 0.0) return 13;
      write_R(f, one);
      write_R(f, multi[b]);
      for (int j = 0; j < one.NCj; ++j)
        for (int i = 0; i < one.NCi; ++i) fwrite(&one.dt[i][j], sizeof(double), 1, f);
      fwrite(&dtmin, sizeof(double), 1, f);
      const double l2 = L2_Norm_Residual(one);
      fwrite(&l2, sizeof(double), 1, f);
    }
    fclose(f);
  }
  printf("ok %zu %.17g %.17g %.17g %d %d %d\n", IP.Ignored.size(), IP.Wo.d, IP.Wo.v.x, IP.Wo.p,
         IP.NKS.block_preconditioner, IP.NKS.ilu_level_of_fill, IP.NKS.jacobian_order);
  return 0;
}

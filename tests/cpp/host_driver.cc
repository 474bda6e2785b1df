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

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: host_driver parse|run|residual1 DECK OUT [STATE_OUT]\n");
    return 2;
  }
  const std::string mode = argv[1];
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
  printf("ok %zu %.17g %.17g %.17g\n", IP.Ignored.size(), IP.Wo.d, IP.Wo.v.x, IP.Wo.p);
  return 0;
}

// cffc_euler2d.hpp — C++ host surface of the B200 Euler2D library: the
// reference's Euler2D types and entry points by name, backed by the C ABI of
// cffc_e2d.h (libcffc_e2d.so).  A caller of the reference's Euler2D path
// includes this header instead of Euler2DQuad.h / Euler2DInput.h and keeps
// its calls:
//
//   Euler2D_pState / Euler2D_cState        src_2D/Euler2D/Euler2DState.h:131, :655
//   Euler2D_Quad_Block (W, U, dUdt, dt, Grid, WoN/S/E/W)
//                                          src_2D/Euler2D/Euler2DQuad.h:180-880
//   Euler2D_Input_Parameters + deck parser src_2D/Euler2D/Euler2DInput.h:41,
//                                          Euler2DInput.cc:1759-3920,
//                                          NewtonKrylovSchwarz2D/NKSInput2D.h:378-640
//   dUdt_Residual_Evaluation(block, IP)    Euler2DQuadSingleBlock.cc:5095
//   CFL, L1/L2/Max_Norm_Residual           Euler2DQuadSingleBlock.cc:3019, :3111-3167
//   Euler2DQuadSolver(file, batch_flag)    Euler2DQuadSolvers.cc:26
//
// Multi-block work (ghost exchange, explicit stepping, Newton-Krylov) runs on
// a Euler2D_Device_Blocks set: the blocks are packed into the library's SoA
// layout once, advanced on the GPU, and unpacked back on request.
#ifndef CFFC_EULER2D_HPP
#define CFFC_EULER2D_HPP

#include <istream>
#include <string>
#include <vector>

#include "cffc_e2d.h"

namespace cffc_b200 {

struct Vector2D {
  double x = 0.0, y = 0.0;
  Vector2D() = default;
  Vector2D(double a, double b) : x(a), y(b) {}
};

class Euler2D_cState;

// Primitive state (rho, u, v, p); gamma = 1.4, R = R_universal / M_air
// = 8.314511 / 0.028964 J/(kg K)
// (Euler2DState.h:972-977).  operator[] is 1-based as in the reference.
class Euler2D_pState {
 public:
  double d = 1.0;
  Vector2D v;
  double p = 1.0;
  static double g, gm1, gm1i, R;
  Euler2D_pState() = default;
  Euler2D_pState(double rho, double u, double vv, double pre) : d(rho), v(u, vv), p(pre) {}
  double a() const;   // sound speed sqrt(g p / d)
  double h() const;   // specific total enthalpy
  double E() const;   // total energy per unit volume
  Euler2D_cState U() const;
  double& operator[](int index);
  const double& operator[](int index) const;
};

// Conserved state (rho, rho u, rho v, E).
class Euler2D_cState {
 public:
  double d = 1.0;
  Vector2D dv;
  double E = 1.0;
  Euler2D_cState() = default;
  Euler2D_cState(double rho, double mx, double my, double e) : d(rho), dv(mx, my), E(e) {}
  double e() const;   // specific internal energy
  Euler2D_pState W() const;
  double& operator[](int index);
  const double& operator[](int index) const;
};

// Grid of one block: nodes (NNi x NNj incl. ghost nodes) and the BC type of
// every boundary cell (Grid2D_Quad_Block_HO::Node, BCtypeN/S/E/W).
struct Grid2D_Quad_Block {
  int NNi = 0, NNj = 0, Nghost = 0;
  std::vector<std::vector<Vector2D>> Node;   // Node[i][j]
  std::vector<int> BCtypeN, BCtypeS;         // [NCi]
  std::vector<int> BCtypeE, BCtypeW;         // [NCj]
};

// One solution block with the reference's index conventions: cells
// i in [0, NCi), interior [ICl, ICu] (ICl = Nghost), same for j.
class Euler2D_Quad_Block {
 public:
  int NCi = 0, ICl = 0, ICu = 0, NCj = 0, JCl = 0, JCu = 0, Nghost = 0;
  std::vector<std::vector<Euler2D_pState>> W;   // W[i][j]
  std::vector<std::vector<Euler2D_cState>> U;   // U[i][j]
  std::vector<std::vector<Euler2D_cState>> dUdt; // dUdt[i][j] (stage 0)
  std::vector<std::vector<double>> dt;
  std::vector<Euler2D_pState> WoN, WoS;         // [NCi] BC reference states
  std::vector<Euler2D_pState> WoE, WoW;         // [NCj]
  Grid2D_Quad_Block Grid;
  void allocate(int Ni, int Nj, int Ng);        // interior cells Ni x Nj
};

// The input parameters of the path (the deck keywords listed in
// Parse_Next_Input_Control_Parameter below); values in the deck's units
// (Pressure in kPa, Time_Max in ms), stored in SI as the reference does.
struct Euler2D_Input_Parameters {
  std::string Time_Integration_Type = "Explicit_Euler";
  int i_Time_Integration = E2D_TIME_EXPLICIT_EULER;
  int N_Stage = 1;
  double Residual_Smoothing_Epsilon = 0.0;  // > 0 turns implicit residual smoothing on
  int Residual_Smoothing_Gauss_Seidel_Iterations = 2;
  int Freeze_Limiter = 0;
  double Freeze_Limiter_Residual_Level = 1e-4;
  double CFL_Number = 0.5;
  int Time_Accurate = 0;
  int Local_Time_Stepping = 0;
  int Maximum_Number_of_Time_Steps = 100;
  double Time_Max = 0.0;
  std::string Reconstruction_Type = "Least_Squares";
  std::string Limiter_Type = "Venkatakrishnan";
  int i_Limiter = E2D_LIMITER_VENKATAKRISHNAN;
  std::string Flux_Function_Type = "Roe";
  int i_Flux_Function = E2D_FLUX_ROE;
  std::string ICs_Type = "Uniform";
  std::string Grid_Type = "Rectangular_Box";
  double Box_Width = 1.0, Box_Height = 1.0;
  double Bump_Height = 0.1;
  int Number_of_Cells_Idir = 100, Number_of_Cells_Jdir = 100;
  int Number_of_Blocks_Idir = 1, Number_of_Blocks_Jdir = 1;
  int Number_of_Blocks_Per_Processor = 0;  // 0: the block count (the quadtree's capacity)
  int Number_of_Ghost_Cells = 2;
  double Mach_Number = 0.0, Flow_Angle = 0.0;
  double Pressure = 101325.0, Temperature = 288.16;
  Euler2D_pState Wo;               // freestream (from Pressure, Temperature, Mach, angle)
  std::string Output_File_Name = "outputfile.dat";
  std::string Restart_File_Name = "restartfile.soln";  // the keyword's value + ".soln"
  std::string Grid_File_Name = "gridfile.grid";        // Grid_File_Name keyword + ".grid"
  std::string Grid_Definition_File_Name = "gridfile.griddef";
  std::string Gas_Type = "AIR";
  int Restart_Solution_Save_Frequency = 1000;
  std::vector<std::string> Commands;  // commands after Execute (Write_Restart, Write_Output, ...)
  int Precision = E2D_PREC_FP64;   // GPU_Precision keyword (library extension)
  e2d_nks_params NKS{};            // Maximum_Number_of_NKS_Iterations, GMRES_*, NKS_*
  std::vector<std::string> Ignored; // keywords of the reference outside this path
  int Line_Number = 0;
  Euler2D_Input_Parameters();
  void set_freestream();  // Wo from Pressure and Temperature, then set_velocity()
  void set_velocity();    // Wo.v from Mach_Number and Flow_Angle at Wo's sound speed
  // Reads a whole deck up to Execute / Terminate; returns 0 or the
  // (positive) line number of the first invalid entry.
  int Process_Input_Control_Parameter_File(const std::string& path);
};

// One multi-block set resident on the GPU.  neighbour[8*b + k] is the
// reference's same-resolution neighbour of block b in the order W E S N SW
// SE NW NE (-1: none).
class Euler2D_Device_Blocks {
 public:
  Euler2D_Device_Blocks(std::vector<Euler2D_Quad_Block>& blocks, const std::vector<int>& neighbour,
                        const Euler2D_Input_Parameters& IP, int device = 0);
  ~Euler2D_Device_Blocks();
  Euler2D_Device_Blocks(const Euler2D_Device_Blocks&) = delete;
  Euler2D_Device_Blocks& operator=(const Euler2D_Device_Blocks&) = delete;
  int upload();                         // W of the host blocks -> device (U = U(W))
  int upload_conserved();               // U of the host blocks -> device (W = W(U)), as after a restart
  int download();                       // device W, U -> host blocks
  int residual();                       // ghost fill + dUdt_Residual_Evaluation
  int explicit_steps(int n, std::vector<double>* hist);  // hist: n x (dt, L1, L2, Max)
  int nks(const e2d_nks_params& p, std::vector<e2d_nks_step>* hist);
  e2d_handle* handle() { return h_; }
 private:
  std::vector<Euler2D_Quad_Block>& blocks_;
  e2d_handle* h_ = nullptr;
  int nci_ = 0, ncj_ = 0, ng_ = 0;
};

int Parse_Next_Input_Control_Parameter(Euler2D_Input_Parameters& IP, std::istream& in, const std::string& code);

// Grid and initial solution for the deck's Grid_Type and ICs_Type (Uniform /
// Constant: the freestream everywhere).  Rectangular_Box and Periodic_Box
// span [-W/2, W/2] x [-H/2, H/2] with uniform cells (reflecting walls, or
// periodic wrap-around); Sine_Squared_Bump_Channel (a library grid, not the
// reference's spline-built Bump_Channel_Flow) is [-1.5, 1.5] x [0, 1] over a
// Bump_Height * sin^2 bump on |x| <= 0.5 with characteristic inflow/outflow.
int Create_Initial_Solution_Blocks(const Euler2D_Input_Parameters& IP, std::vector<Euler2D_Quad_Block>& blocks,
                                   std::vector<int>& neighbour);

// Writes the block set as a case file (the binary layout read by
// cffc_b200.cases.read_case and the oracle harness): dimensions, scheme,
// and per block neighbours, BC codes, nodes, BC reference states and W.
int Write_Case_File(const std::string& path, const std::vector<Euler2D_Quad_Block>& blocks,
                    const std::vector<int>& neighbour, const Euler2D_Input_Parameters& IP);

// Single-block residual with the caller's ghost cells (the reference's
// caller fills them); dUdt is written back into SolnBlk.dUdt.
int dUdt_Residual_Evaluation(Euler2D_Quad_Block& SolnBlk, const Euler2D_Input_Parameters& IP);

double CFL(Euler2D_Quad_Block& SolnBlk, const Euler2D_Input_Parameters& IP);
double L1_Norm_Residual(const Euler2D_Quad_Block& SolnBlk);
double L2_Norm_Residual(const Euler2D_Quad_Block& SolnBlk);
double Max_Norm_Residual(const Euler2D_Quad_Block& SolnBlk);

// ---- grid data files ------------------------------------------------------
// The reference's multi-block grid data file (Write_Multi_Block_Grid_Using_IP /
// Read_Multi_Block_Grid_Using_IP, Grid/HO_Grid2DQuadMultiBlock.h:3160-3210):
// the Grid_Type line, its i_Grid code, "nbi nbj", then every block's grid
// (j outer, i inner) as the restart files hold it.  Reading keeps nodes and
// BC codes (cell data and boundary splines are dropped) and wires the
// nbi x nbj root blocks as the reference does (periodic for Periodic_Box).
// Grid_Type Read_From_Data_File builds the initial blocks from
// Grid_File_Name.  Return 0, or 1 when the file cannot be opened or parsed.
int Write_Multi_Block_Grid(const std::string& path, const std::vector<Euler2D_Quad_Block>& blocks,
                           const Euler2D_Input_Parameters& IP);
int Read_Multi_Block_Grid(const std::string& path, std::vector<Euler2D_Quad_Block>& blocks,
                          std::vector<int>& neighbour, std::string* grid_type = nullptr, int* nbi = nullptr,
                          int* nbj = nullptr);

// ---- restart files -------------------------------------------------------
// The reference's checkpoint format: PREFIX_quadtree.tree (the block tree,
// Write_QuadTree / Read_QuadTree, AMR/AMR.h:163-340) and one
// PREFIX_blkNNNNNN.soln per block, NNNNNN the global block number
// (Write_Restart_Solution / Read_Restart_Solution,
// Euler2DQuadMultiBlock.cc:145-300), PREFIX = Restart_File_Name up to its
// first '.' or ' '.  Files written here are the reference's byte for byte
// for a block set without boundary splines (the reference's own writer
// prints 16 significant digits, so a round trip moves a value by at most
// one unit in its 16th digit).  Blocks are numbered b = j * nbi + i over the
// Number_of_Blocks_Idir x Number_of_Blocks_Jdir roots, one CPU.  Reading
// takes any tree whose used blocks all sit at one refinement level (no
// resolution changes) and files with or without boundary splines, whose
// data is skipped.  Return 0, or 1 when a file cannot be opened or parsed.
int Write_QuadTree(const std::vector<Euler2D_Quad_Block>& blocks, const std::vector<int>& neighbour,
                   const Euler2D_Input_Parameters& IP);
int Write_Restart_Solution(const std::vector<Euler2D_Quad_Block>& blocks, const Euler2D_Input_Parameters& IP,
                           int Number_of_Time_Steps, double Time, double CPU_Time);
// Fills neighbour (indexed by global block number), sizes blocks, and sets
// the root layout Number_of_Blocks_Idir/Jdir and Number_of_Blocks_Per_Processor
// from the tree.
int Read_QuadTree(std::vector<Euler2D_Quad_Block>& blocks, std::vector<int>& neighbour,
                  Euler2D_Input_Parameters& IP);
// Reads every block of the tree; as the reference does, adds the stored
// step count to Maximum_Number_of_Time_Steps.
int Read_Restart_Solution(std::vector<Euler2D_Quad_Block>& blocks, Euler2D_Input_Parameters& IP,
                          int& Number_of_Time_Steps, double& Time, double& CPU_Time);

// Whole solve from a deck: grid and ICs (or, for ICs_Type Restart, the
// restart files), explicit steps (restart files every
// Restart_Solution_Save_Frequency steps), then Newton-Krylov when
// Maximum_Number_of_NKS_Iterations > 0; writes Output_File_Name, and the
// restart files when the deck's commands after Execute hold Write_Restart.
int Euler2DQuadSolver(const char* Input_File_Name_ptr, int batch_flag);

}  // namespace cffc_b200

#endif

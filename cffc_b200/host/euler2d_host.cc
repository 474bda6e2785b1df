// euler2d_host.cc — the C++ host surface of include/cffc_euler2d.hpp: the
// reference's Euler2D state and block types, the input-deck parser of the
// path, grid / initial-solution builders, and the solver driver, all on top
// of the C ABI of cffc_e2d.h.  Host-side only: no CUDA code here.
#include "cffc_euler2d.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <istream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace cffc_b200 {

namespace {
constexpr double HALF = 0.5;
constexpr double PI = 3.14159265358979323846;
constexpr int INVALID_INPUT_CODE = -1, EXECUTE_CODE = 1, TERMINATE_CODE = 2;
}  // namespace

// ---- states (Euler2DState.h:1055-1095, :1741-1760, :3414-3430) -------------
// gm1 = g - 1 and gm1i = 1/gm1 as Euler2D_pState::setgas derives them (the
// double g - 1 is not the double nearest 0.4)
double Euler2D_pState::g = 1.4;
double Euler2D_pState::gm1 = 1.4 - 1.0;
double Euler2D_pState::gm1i = 1.0 / (1.4 - 1.0);
double Euler2D_pState::R = 8.314511 / (28.9640 * 0.001);  // R_UNIVERSAL / (MOLE_WT_AIR * MILLI)

double Euler2D_pState::a() const { return std::sqrt(g * p / d); }
double Euler2D_pState::h() const { return g * p / (gm1 * d) + HALF * (v.x * v.x + v.y * v.y); }
double Euler2D_pState::E() const { return p * gm1i + HALF * d * (v.x * v.x + v.y * v.y); }
Euler2D_cState Euler2D_pState::U() const { return Euler2D_cState(d, d * v.x, d * v.y, E()); }
double& Euler2D_pState::operator[](int index) {
  switch (index) {
    case 1: return d;
    case 2: return v.x;
    case 3: return v.y;
    default: return p;
  }
}
const double& Euler2D_pState::operator[](int index) const {
  return const_cast<Euler2D_pState*>(this)->operator[](index);
}

double Euler2D_cState::e() const { return E / d - HALF * (dv.x * dv.x + dv.y * dv.y) / (d * d); }
Euler2D_pState Euler2D_cState::W() const {
  return Euler2D_pState(d, dv.x / d, dv.y / d,
                        Euler2D_pState::gm1 * (E - HALF * (dv.x * dv.x + dv.y * dv.y) / d));
}
double& Euler2D_cState::operator[](int index) {
  switch (index) {
    case 1: return d;
    case 2: return dv.x;
    case 3: return dv.y;
    default: return E;
  }
}
const double& Euler2D_cState::operator[](int index) const {
  return const_cast<Euler2D_cState*>(this)->operator[](index);
}

// ---- block (Euler2D_Quad_Block::allocate, Euler2DQuad.h:655-760) -----------
void Euler2D_Quad_Block::allocate(int Ni, int Nj, int Ng) {
  Nghost = Ng;
  NCi = Ni + 2 * Ng; ICl = Ng; ICu = Ni + Ng - 1;
  NCj = Nj + 2 * Ng; JCl = Ng; JCu = Nj + Ng - 1;
  W.assign(NCi, std::vector<Euler2D_pState>(NCj));
  U.assign(NCi, std::vector<Euler2D_cState>(NCj));
  dUdt.assign(NCi, std::vector<Euler2D_cState>(NCj, Euler2D_cState(0, 0, 0, 0)));
  dt.assign(NCi, std::vector<double>(NCj, 0.0));
  WoN.assign(NCi, Euler2D_pState()); WoS.assign(NCi, Euler2D_pState());
  WoE.assign(NCj, Euler2D_pState()); WoW.assign(NCj, Euler2D_pState());
  Grid.Nghost = Ng;
  Grid.NNi = NCi + 1; Grid.NNj = NCj + 1;
  Grid.Node.assign(Grid.NNi, std::vector<Vector2D>(Grid.NNj));
  Grid.BCtypeN.assign(NCi, E2D_BC_NONE); Grid.BCtypeS.assign(NCi, E2D_BC_NONE);
  Grid.BCtypeE.assign(NCj, E2D_BC_NONE); Grid.BCtypeW.assign(NCj, E2D_BC_NONE);
}

// ---- input deck --------------------------------------------------------------
Euler2D_Input_Parameters::Euler2D_Input_Parameters() {
  // NKS_Input_Parameters defaults (NKSInput2D.h:125-172)
  NKS.max_newton = 0;
  NKS.gmres_restart = 30;
  NKS.max_gmres = 100;
  NKS.overall_tol = 1e-5;
  NKS.cfl0 = 1.0;
  NKS.gmres_tol_initial = 1e-5;
  NKS.gmres_tol_final = 1e-5;
  NKS.epsilon0 = 1e-6;
  NKS.min_ratio = 1e-10;
  // freestream defaults (Set_Default_Input_Parameters, Euler2DInput.cc:304-313):
  // the standard atmosphere, its temperature, Mach 0.8 along x
  Wo = Euler2D_pState(1.225, 0.0, 0.0, 101325.00);
  Pressure = Wo.p;
  Temperature = Wo.p / (Wo.d * Euler2D_pState::R);
  Mach_Number = 0.80;
  Flow_Angle = 0.0;
  set_velocity();
}

// Wo.v from Mach_Number and Flow_Angle at the current sound speed (the update
// every freestream keyword makes, Euler2DInput.cc:2558-2611).
void Euler2D_Input_Parameters::set_velocity() {
  Wo.v.x = Mach_Number * Wo.a() * std::cos(2.0 * PI * Flow_Angle / 360.00);
  Wo.v.y = Mach_Number * Wo.a() * std::sin(2.0 * PI * Flow_Angle / 360.00);
}

// Wo = (Pressure / (R Temperature), 0, 0, Pressure), then its velocity (the
// Pressure and Temperature keywords).
void Euler2D_Input_Parameters::set_freestream() {
  Wo = Euler2D_pState(Pressure / (Euler2D_pState::R * Temperature), 0.0, 0.0, Pressure);
  set_velocity();
}

namespace {

// Get_Next_Input_Control_Parameter (Euler2DInput.cc:100-144): the first
// token (up to blank, tab or '=') of the next line that is neither empty nor
// a '#' comment.
bool next_token(std::istream& in, int& line, std::string& tok) {
  std::string buf;
  while (std::getline(in, buf)) {
    ++line;
    size_t i = buf.find_first_not_of(" \t");
    if (i == std::string::npos || buf[i] == '#' || buf[i] == '\r') continue;
    size_t e = buf.find_first_of(" \t=\r", i);
    tok = buf.substr(i, e == std::string::npos ? std::string::npos : e - i);
    return true;
  }
  return false;
}

// A numeric value on the next line (IP.Input_File >> value; getline).
template <class T> bool next_value(std::istream& in, int& line, T& v) {
  std::string buf;
  if (!std::getline(in, buf)) return false;
  ++line;
  std::istringstream ss(buf);
  return static_cast<bool>(ss >> v);
}

}  // namespace

// Parse_Next_Input_Control_Parameter (Euler2DInput.cc:1759-3920,
// NKSInput2D.h:378-640) for the keywords of this path.  Returns 0 for a
// keyword taken, EXECUTE_CODE / TERMINATE_CODE, or INVALID_INPUT_CODE.
int Parse_Next_Input_Control_Parameter(Euler2D_Input_Parameters& IP, std::istream& in, const std::string& code) {
  int& L = IP.Line_Number;
  std::string s;
  auto str = [&](std::string& dst) { return next_token(in, L, dst) ? 0 : INVALID_INPUT_CODE; };
  if (code == "Execute") return EXECUTE_CODE;
  if (code == "Terminate") return TERMINATE_CODE;
  if (code == "Continue" || code == "Write_Output" || code == "Write_Output_Cells") return 0;
  if (code == "Time_Integration_Type") {
    if (str(IP.Time_Integration_Type)) return INVALID_INPUT_CODE;
    // Euler2DInput.cc:1782-1794; multigrid and the implicit schemes are
    // outside this path
    const std::string& t = IP.Time_Integration_Type;
    if (t == "Explicit_Euler") { IP.i_Time_Integration = E2D_TIME_EXPLICIT_EULER; IP.N_Stage = 1; }
    else if (t == "Explicit_Predictor_Corrector") { IP.i_Time_Integration = E2D_TIME_PREDICTOR_CORRECTOR; IP.N_Stage = 2; }
    else if (t == "Explicit_Runge_Kutta") { IP.i_Time_Integration = E2D_TIME_RUNGE_KUTTA; IP.N_Stage = 4; }
    else if (t == "Multistage_Optimal_Smoothing") { IP.i_Time_Integration = E2D_TIME_OPTIMAL_SMOOTHING; IP.N_Stage = 4; }
    else return INVALID_INPUT_CODE;
    return 0;
  }
  if (code == "Reconstruction_Type") {
    if (str(IP.Reconstruction_Type)) return INVALID_INPUT_CODE;
    return IP.Reconstruction_Type == "Least_Squares" ? 0 : INVALID_INPUT_CODE;
  }
  if (code == "Limiter_Type") {
    if (str(IP.Limiter_Type)) return INVALID_INPUT_CODE;
    const std::string& t = IP.Limiter_Type;
    if (t == "One") IP.i_Limiter = E2D_LIMITER_ONE;
    else if (t == "Zero") IP.i_Limiter = E2D_LIMITER_ZERO;
    else if (t == "Barth_Jespersen") IP.i_Limiter = E2D_LIMITER_BARTH_JESPERSEN;
    else if (t == "Venkatakrishnan") IP.i_Limiter = E2D_LIMITER_VENKATAKRISHNAN;
    else return INVALID_INPUT_CODE;
    return 0;
  }
  if (code == "Flux_Function_Type") {
    // the names of Euler2DInput.cc:1850-1876; the preconditioned and moving-frame
    // variants are outside this path
    if (str(IP.Flux_Function_Type)) return INVALID_INPUT_CODE;
    static const std::pair<const char*, int> names[] = {
        {"Godunov", E2D_FLUX_GODUNOV}, {"Roe", E2D_FLUX_ROE},         {"Rusanov", E2D_FLUX_RUSANOV},
        {"HLLE", E2D_FLUX_HLLE},       {"Linde", E2D_FLUX_LINDE},     {"HLLC", E2D_FLUX_HLLC},
        {"VanLeer", E2D_FLUX_VANLEER}, {"AUSM", E2D_FLUX_AUSM},       {"AUSM+", E2D_FLUX_AUSMPLUS}};
    for (const auto& n : names)
      if (IP.Flux_Function_Type == n.first) {
        IP.i_Flux_Function = n.second;
        return 0;
      }
    return INVALID_INPUT_CODE;
  }
  if (code == "ICs_Type") {
    if (str(IP.ICs_Type)) return INVALID_INPUT_CODE;
    const std::string& t = IP.ICs_Type;
    return (t == "Uniform" || t == "Constant" || t == "Restart") ? 0 : INVALID_INPUT_CODE;
  }
  if (code == "Grid_Type") {
    // any of the reference's grid names: a restart run (ICs_Type Restart)
    // takes its grid from the restart files; otherwise
    // Create_Initial_Solution_Blocks builds Rectangular_Box, Periodic_Box and
    // Sine_Squared_Bump_Channel and rejects the rest
    return str(IP.Grid_Type);
  }
  if (code == "Output_File_Name") {  // Euler2DInput.cc:2157-2174: names every output file
    std::string v;
    if (str(v)) return INVALID_INPUT_CODE;
    IP.Output_File_Name = v + ".dat";
    IP.Grid_File_Name = v + ".grid";
    IP.Grid_Definition_File_Name = v + ".griddef";
    IP.Restart_File_Name = v + ".soln";
    return 0;
  }
  if (code == "Grid_File_Name") {  // Euler2DInput.cc:2176-2184
    if (str(IP.Grid_File_Name)) return INVALID_INPUT_CODE;
    IP.Grid_Definition_File_Name = IP.Grid_File_Name + ".griddef";
    IP.Grid_File_Name += ".grid";
    return 0;
  }
  if (code == "Restart_File_Name") {  // Euler2DInput.cc:2186-2191
    if (str(IP.Restart_File_Name)) return INVALID_INPUT_CODE;
    IP.Restart_File_Name += ".soln";
    return 0;
  }
  if (code == "GPU_Precision") {
    if (str(s)) return INVALID_INPUT_CODE;
    if (s == "FP64") IP.Precision = E2D_PREC_FP64;
    else if (s == "FP64_Exact") IP.Precision = E2D_PREC_FP64_EXACT;
    else if (s == "FP32") IP.Precision = E2D_PREC_FP32;
    else return INVALID_INPUT_CODE;
    return 0;
  }
  // numeric keywords: (name, pointer, validity)
  auto num_i = [&](int& v, int lo) { return (next_value(in, L, v) && v >= lo) ? 0 : INVALID_INPUT_CODE; };
  auto num_d = [&](double& v, bool positive) {
    return (next_value(in, L, v) && (!positive || v > 0.0)) ? 0 : INVALID_INPUT_CODE;
  };
  if (code == "N_Stage") return num_i(IP.N_Stage, 1);  // the scheme's stage counts are checked at e2d_create
  if (code == "CFL_Number") return num_d(IP.CFL_Number, true);
  if (code == "Residual_Smoothing_Epsilon") {  // Euler2DInput.cc:2958-2969 (<= 0: off)
    int rc = num_d(IP.Residual_Smoothing_Epsilon, false);
    if (!rc && IP.Residual_Smoothing_Epsilon <= 0.0) IP.Residual_Smoothing_Epsilon = 0.0;
    return rc;
  }
  if (code == "Residual_Smoothing_Gauss_Seidel_Iterations") {
    int rc = num_i(IP.Residual_Smoothing_Gauss_Seidel_Iterations, -1000000);
    if (!rc && IP.Residual_Smoothing_Gauss_Seidel_Iterations < 0) IP.Residual_Smoothing_Gauss_Seidel_Iterations = 0;
    return rc;
  }
  if (code == "Freeze_Limiter") return num_i(IP.Freeze_Limiter, 0);
  if (code == "Freeze_Limiter_Residual_Level") return num_d(IP.Freeze_Limiter_Residual_Level, false);
  if (code == "Time_Accurate") return num_i(IP.Time_Accurate, 0);
  if (code == "Restart_Solution_Save_Frequency") return num_i(IP.Restart_Solution_Save_Frequency, 1);
  if (code == "Local_Time_Stepping") {
    int rc = num_i(IP.Local_Time_Stepping, 0);
    if (IP.Local_Time_Stepping > 1) IP.Local_Time_Stepping = 1;  // scalar local time stepping
    return rc;
  }
  if (code == "Maximum_Number_of_Time_Steps") return num_i(IP.Maximum_Number_of_Time_Steps, 0);
  if (code == "Time_Max") {
    int rc = num_d(IP.Time_Max, false);
    IP.Time_Max = IP.Time_Max / 1000.0;  // ms -> s
    return rc;
  }
  if (code == "Box_Width") return num_d(IP.Box_Width, true);
  if (code == "Box_Height") return num_d(IP.Box_Height, true);
  if (code == "Bump_Height") return num_d(IP.Bump_Height, false);
  if (code == "Number_of_Cells_Idir") return num_i(IP.Number_of_Cells_Idir, 1);
  if (code == "Number_of_Cells_Jdir") return num_i(IP.Number_of_Cells_Jdir, 1);
  if (code == "Number_of_Blocks_Idir") return num_i(IP.Number_of_Blocks_Idir, 1);
  if (code == "Number_of_Blocks_Jdir") return num_i(IP.Number_of_Blocks_Jdir, 1);
  if (code == "Number_of_Blocks_Per_Processor") return num_i(IP.Number_of_Blocks_Per_Processor, 1);
  if (code == "Number_of_Ghost_Cells") {
    int rc = num_i(IP.Number_of_Ghost_Cells, 1);
    return rc ? rc : (IP.Number_of_Ghost_Cells == 2 ? 0 : INVALID_INPUT_CODE);
  }
  if (code == "Mach_Number") {
    int rc = num_d(IP.Mach_Number, false);
    if (!rc) IP.set_velocity();
    return rc;
  }
  if (code == "Flow_Angle") {
    int rc = num_d(IP.Flow_Angle, false);
    if (!rc) IP.set_velocity();
    return rc;
  }
  if (code == "Pressure") {
    int rc = num_d(IP.Pressure, true);
    IP.Pressure = IP.Pressure * 1000.0;  // kPa -> Pa
    IP.set_freestream();
    return rc;
  }
  if (code == "Temperature") {
    int rc = num_d(IP.Temperature, true);
    IP.set_freestream();
    return rc;
  }
  // NKS_Input_Parameters::Parse_Next_Input_Control_Parameter (NKSInput2D.h:378-640)
  e2d_nks_params& N = IP.NKS;
  if (code == "Maximum_Number_of_NKS_Iterations") return num_i(N.max_newton, 0);
  if (code == "NKS_Overall_Tolerance") return num_d(N.overall_tol, false);
  if (code == "NKS_Finite_Time_Step_Initial_CFL") return num_d(N.cfl0, true);
  if (code == "Maximum_Number_of_GMRES_Iterations") return num_i(N.max_gmres, 1);
  if (code == "GMRES_Restart") return num_i(N.gmres_restart, 1);
  if (code == "GMRES_Tolerance") {
    int rc = num_d(N.gmres_tol_initial, true);
    N.gmres_tol_final = N.gmres_tol_initial;  // backward compatible keyword
    return rc;
  }
  if (code == "GMRES_Initial_Tolerance") return num_d(N.gmres_tol_initial, true);
  if (code == "GMRES_Final_Tolerance") return num_d(N.gmres_tol_final, true);
  if (code == "GMRES_Epsilon_Naught") return num_d(N.epsilon0, true);
  if (code == "NKS_Min_Finite_Time_Step_Norm_Ratio") return num_d(N.min_ratio, true);
  if (code == "GMRES_Block_Preconditioner") {
    // "Diagonal" is block Jacobi; "ILUK" and any other value ILU(k)
    std::string v;
    if (str(v)) return INVALID_INPUT_CODE;
    N.block_preconditioner = v == "Diagonal" ? E2D_PRECON_BLOCK_JACOBI : E2D_PRECON_BLOCK_ILUK;
    return 0;
  }
  if (code == "GMRES_Overlap") {
    // Schwarz overlap: only 0 (no overlap, the reference's default) is built
    int ov = 0;
    return (num_i(ov, 0) || ov != 0) ? INVALID_INPUT_CODE : 0;
  }
  if (code == "NKS_Finite_Time_Step" || code == "GMRES_Normalization") {
    // both on by default in the reference; OFF (or 0) runs are not built
    std::string v;
    if (str(v)) return INVALID_INPUT_CODE;
    return (v == "OFF" || v == "0") ? INVALID_INPUT_CODE : 0;
  }
  if (code == "GMRES_ILUK_Level_of_Fill") {
    int rc = num_i(N.ilu_level_of_fill, 0);
    return (rc || N.ilu_level_of_fill > 16) ? INVALID_INPUT_CODE : 0;
  }
  if (code == "Jacobian_Order") {
    // Euler2D has the first-order HLLE and the source-terms-only Jacobians;
    // the Roe, AUSM+up and second-order diamond-path ones stop the
    // reference's run (no Euler2D specialization) and are rejected here; an
    // unknown name falls back to first-order HLLE, as the reference's does.
    std::string v;
    if (str(v)) return INVALID_INPUT_CODE;
    if (v == "Source_Terms_Only") N.jacobian_order = E2D_JACOBIAN_SOURCE_TERMS_ONLY;
    else if (v == "First_Order_Inviscid_Roe" || v == "First_Order_Inviscid_AUSM_plus_up" ||
             v.rfind("Second_Order_Diamond_Path_with_", 0) == 0)
      return INVALID_INPUT_CODE;
    else N.jacobian_order = E2D_JACOBIAN_FIRST_ORDER_HLLE;
    return 0;
  }
  // Any other keyword belongs to parts of the reference outside this path:
  // its value line is skipped and the keyword recorded.
  IP.Ignored.push_back(code);
  std::string skip;
  std::getline(in, skip);
  ++L;
  return 0;
}

int Euler2D_Input_Parameters::Process_Input_Control_Parameter_File(const std::string& path) {
  std::ifstream in(path);
  if (!in.good()) return -1;
  Line_Number = 0;
  std::string code;
  while (next_token(in, Line_Number, code)) {
    const int rc = Parse_Next_Input_Control_Parameter(*this, in, code);
    if (rc == TERMINATE_CODE) break;
    if (rc == EXECUTE_CODE) {
      // the commands that follow (Write_Restart, Write_Output, ...) up to
      // Terminate, for the driver to carry out after the solve
      while (next_token(in, Line_Number, code) && code != "Terminate") Commands.push_back(code);
      break;
    }
    if (rc == INVALID_INPUT_CODE) return Line_Number > 0 ? Line_Number : 1;
  }
  return 0;
}

// ---- grids and initial solution -----------------------------------------------
int Create_Initial_Solution_Blocks(const Euler2D_Input_Parameters& IP, std::vector<Euler2D_Quad_Block>& blocks,
                                   std::vector<int>& neighbour) {
  const int nbi = IP.Number_of_Blocks_Idir, nbj = IP.Number_of_Blocks_Jdir, ng = IP.Number_of_Ghost_Cells;
  const std::string& t = IP.Grid_Type;
  if (t == "Read_From_Data_File") {  // the reference's grid data file (Grid_File_Name)
    if (Read_Multi_Block_Grid(IP.Grid_File_Name, blocks, neighbour)) return 1;
    for (Euler2D_Quad_Block& B : blocks) {
      for (auto* wo : {&B.WoN, &B.WoS, &B.WoE, &B.WoW})
        for (auto& w : *wo) w = IP.Wo;
      for (int i = 0; i < B.NCi; ++i)
        for (int j = 0; j < B.NCj; ++j) {
          B.W[i][j] = IP.Wo;
          B.U[i][j] = IP.Wo.U();
        }
    }
    return 0;
  }
  if (t != "Rectangular_Box" && t != "Periodic_Box" && t != "Sine_Squared_Bump_Channel") return 1;
  if (IP.Number_of_Cells_Idir % nbi || IP.Number_of_Cells_Jdir % nbj) return 1;
  const int nci = IP.Number_of_Cells_Idir / nbi, ncj = IP.Number_of_Cells_Jdir / nbj;
  const int Nx = IP.Number_of_Cells_Idir, Ny = IP.Number_of_Cells_Jdir;
  const bool periodic = IP.Grid_Type == "Periodic_Box";
  const bool bump = IP.Grid_Type == "Sine_Squared_Bump_Channel";
  int bcW = E2D_BC_REFLECTION, bcE = E2D_BC_REFLECTION, bcS = E2D_BC_REFLECTION, bcN = E2D_BC_REFLECTION;
  // Periodic_Box: BC_PERIODIC on the edges of a direction with one block,
  // BC_NONE otherwise (Grid/HO_Grid2DQuadMultiBlock.h:1299-1330); the blocks
  // are wired across the box edges only with several blocks in both
  // directions (AMR/QuadTree.cc:363)
  if (periodic) {
    bcW = bcE = nbi == 1 ? E2D_BC_PERIODIC : E2D_BC_NONE;
    bcS = bcN = nbj == 1 ? E2D_BC_PERIODIC : E2D_BC_NONE;
  }
  const bool wrap = periodic && nbi > 1 && nbj > 1;
  if (bump) bcW = bcE = E2D_BC_CHARACTERISTIC;
  // node map of global node indices (ghost nodes continue the same map)
  auto node = [&](int I, int J) -> Vector2D {
    const double x = -0.5 * IP.Box_Width + IP.Box_Width * double(I) / double(Nx);
    if (!bump) return Vector2D(x, -0.5 * IP.Box_Height + IP.Box_Height * double(J) / double(Ny));
    // channel [-1.5, 1.5] x [0, 1] over a sin^2 bump on |x| <= 0.5
    const double xb = -1.5 + 3.0 * double(I) / double(Nx);
    const double yw = std::fabs(xb) <= 0.5 ? IP.Bump_Height * std::pow(std::sin(PI * (xb + 0.5)), 2) : 0.0;
    const double eta = double(J) / double(Ny);
    return Vector2D(xb, yw + eta * (1.0 - yw));
  };
  static const int off[8][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
  blocks.assign(size_t(nbi) * nbj, Euler2D_Quad_Block());
  neighbour.assign(size_t(8) * nbi * nbj, -1);
  for (int bj = 0; bj < nbj; ++bj)
    for (int bi = 0; bi < nbi; ++bi) {
      const int b = bj * nbi + bi;
      Euler2D_Quad_Block& B = blocks[b];
      B.allocate(nci, ncj, ng);
      for (int k = 0; k < 8; ++k) {
        int ni = bi + off[k][0], nj = bj + off[k][1];
        if (wrap) { ni = (ni + nbi) % nbi; nj = (nj + nbj) % nbj; }
        if (ni >= 0 && ni < nbi && nj >= 0 && nj < nbj) neighbour[8 * b + k] = nj * nbi + ni;
      }
      for (int i = 0; i < B.Grid.NNi; ++i)
        for (int j = 0; j < B.Grid.NNj; ++j) B.Grid.Node[i][j] = node(bi * nci + i - ng, bj * ncj + j - ng);
      if (bi == 0) std::fill(B.Grid.BCtypeW.begin(), B.Grid.BCtypeW.end(), bcW);
      if (bi == nbi - 1) std::fill(B.Grid.BCtypeE.begin(), B.Grid.BCtypeE.end(), bcE);
      if (bj == 0) std::fill(B.Grid.BCtypeS.begin(), B.Grid.BCtypeS.end(), bcS);
      if (bj == nbj - 1) std::fill(B.Grid.BCtypeN.begin(), B.Grid.BCtypeN.end(), bcN);
      for (auto& w : B.WoN) w = IP.Wo;
      for (auto& w : B.WoS) w = IP.Wo;
      for (auto& w : B.WoE) w = IP.Wo;
      for (auto& w : B.WoW) w = IP.Wo;
      // ICs_Type Uniform / Constant: the freestream everywhere (ICs,
      // Euler2DQuadSingleBlock.cc:1689)
      for (int i = 0; i < B.NCi; ++i)
        for (int j = 0; j < B.NCj; ++j) {
          B.W[i][j] = IP.Wo;
          B.U[i][j] = IP.Wo.U();
        }
    }
  return 0;
}

// ---- device block set --------------------------------------------------------
namespace {

struct Packed {
  std::vector<int32_t> neighbour, bcw, bce, bcs, bcn;
  std::vector<double> X, Y, wow, woe, wos, won;
  e2d_blocks_desc desc{};
};

void pack_blocks(const std::vector<Euler2D_Quad_Block>& blocks, const std::vector<int>& neighbour, Packed& P) {
  const int nblk = int(blocks.size());
  const Euler2D_Quad_Block& B0 = blocks[0];
  const int NCi = B0.NCi, NCj = B0.NCj, NNi = NCi + 1, NNj = NCj + 1;
  P.neighbour.assign(neighbour.begin(), neighbour.end());
  P.bcw.resize(size_t(nblk) * NCj); P.bce.resize(size_t(nblk) * NCj);
  P.bcs.resize(size_t(nblk) * NCi); P.bcn.resize(size_t(nblk) * NCi);
  P.X.resize(size_t(nblk) * NNi * NNj); P.Y.resize(P.X.size());
  P.wow.resize(size_t(nblk) * 4 * NCj); P.woe.resize(P.wow.size());
  P.wos.resize(size_t(nblk) * 4 * NCi); P.won.resize(P.wos.size());
  for (int b = 0; b < nblk; ++b) {
    const Euler2D_Quad_Block& B = blocks[b];
    for (int j = 0; j < NCj; ++j) {
      P.bcw[size_t(b) * NCj + j] = B.Grid.BCtypeW[j];
      P.bce[size_t(b) * NCj + j] = B.Grid.BCtypeE[j];
      for (int v = 1; v <= 4; ++v) {
        P.wow[(size_t(b) * 4 + v - 1) * NCj + j] = B.WoW[j][v];
        P.woe[(size_t(b) * 4 + v - 1) * NCj + j] = B.WoE[j][v];
      }
    }
    for (int i = 0; i < NCi; ++i) {
      P.bcs[size_t(b) * NCi + i] = B.Grid.BCtypeS[i];
      P.bcn[size_t(b) * NCi + i] = B.Grid.BCtypeN[i];
      for (int v = 1; v <= 4; ++v) {
        P.wos[(size_t(b) * 4 + v - 1) * NCi + i] = B.WoS[i][v];
        P.won[(size_t(b) * 4 + v - 1) * NCi + i] = B.WoN[i][v];
      }
    }
    for (int j = 0; j < NNj; ++j)
      for (int i = 0; i < NNi; ++i) {
        P.X[(size_t(b) * NNj + j) * NNi + i] = B.Grid.Node[i][j].x;
        P.Y[(size_t(b) * NNj + j) * NNi + i] = B.Grid.Node[i][j].y;
      }
  }
  e2d_blocks_desc& d = P.desc;
  d.nblk = nblk; d.nci = NCi - 2 * B0.Nghost; d.ncj = NCj - 2 * B0.Nghost; d.ng = B0.Nghost;
  d.neighbour = P.neighbour.data();
  d.bc_w = P.bcw.data(); d.bc_e = P.bce.data(); d.bc_s = P.bcs.data(); d.bc_n = P.bcn.data();
  d.node_x = P.X.data(); d.node_y = P.Y.data();
  d.wo_w = P.wow.data(); d.wo_e = P.woe.data(); d.wo_s = P.wos.data(); d.wo_n = P.won.data();
}

e2d_scheme scheme_of(const Euler2D_Input_Parameters& IP) {
  e2d_scheme s{};
  s.limiter = IP.i_Limiter;
  s.flux = IP.i_Flux_Function;
  s.n_stage = IP.N_Stage;
  s.local_dt = IP.Local_Time_Stepping ? 1 : 0;
  s.precision = IP.Precision;
  s.time_integration = IP.i_Time_Integration;
  s.rs_iterations = IP.Residual_Smoothing_Gauss_Seidel_Iterations;
  s.freeze_limiter = IP.Freeze_Limiter ? 1 : 0;
  s.cfl = IP.CFL_Number;
  s.gamma = Euler2D_pState::g;
  s.rs_epsilon = IP.Residual_Smoothing_Epsilon;
  s.freeze_level = IP.Freeze_Limiter_Residual_Level;
  return s;
}

// host blocks <-> SoA [nblk][4][NCj][NCi]
void gather_W(const std::vector<Euler2D_Quad_Block>& blocks, std::vector<double>& W) {
  const int NCi = blocks[0].NCi, NCj = blocks[0].NCj;
  W.resize(blocks.size() * 4 * size_t(NCi) * NCj);
  for (size_t b = 0; b < blocks.size(); ++b)
    for (int v = 1; v <= 4; ++v)
      for (int j = 0; j < NCj; ++j)
        for (int i = 0; i < NCi; ++i) W[((b * 4 + v - 1) * NCj + j) * NCi + i] = blocks[b].W[i][j][v];
}

void gather_U(const std::vector<Euler2D_Quad_Block>& blocks, std::vector<double>& U) {
  const int NCi = blocks[0].NCi, NCj = blocks[0].NCj;
  U.resize(blocks.size() * 4 * size_t(NCi) * NCj);
  for (size_t b = 0; b < blocks.size(); ++b)
    for (int v = 1; v <= 4; ++v)
      for (int j = 0; j < NCj; ++j)
        for (int i = 0; i < NCi; ++i) U[((b * 4 + v - 1) * NCj + j) * NCi + i] = blocks[b].U[i][j][v];
}

}  // namespace

Euler2D_Device_Blocks::Euler2D_Device_Blocks(std::vector<Euler2D_Quad_Block>& blocks, const std::vector<int>& neighbour,
                                             const Euler2D_Input_Parameters& IP, int device)
    : blocks_(blocks) {
  if (blocks.empty()) return;
  Packed P;
  pack_blocks(blocks, neighbour, P);
  const e2d_scheme s = scheme_of(IP);
  int err = 0;
  h_ = e2d_create(&P.desc, &s, device, &err);
  nci_ = P.desc.nci; ncj_ = P.desc.ncj; ng_ = P.desc.ng;
  if (h_) upload();
}

Euler2D_Device_Blocks::~Euler2D_Device_Blocks() {
  if (h_) e2d_destroy(h_);
}

int Euler2D_Device_Blocks::upload() {
  if (!h_) return E2D_ERR_ARG;
  std::vector<double> W;
  gather_W(blocks_, W);
  return e2d_set_state(h_, W.data());
}

int Euler2D_Device_Blocks::upload_conserved() {
  if (!h_) return E2D_ERR_ARG;
  std::vector<double> U;
  gather_U(blocks_, U);
  return e2d_set_conserved(h_, U.data());
}

int Euler2D_Device_Blocks::download() {
  if (!h_) return E2D_ERR_ARG;
  const int NCi = blocks_[0].NCi, NCj = blocks_[0].NCj;
  const size_t n = blocks_.size() * 4 * size_t(NCi) * NCj;
  std::vector<double> W(n), U(n);
  const int rc = e2d_get_state(h_, W.data(), U.data());
  if (rc) return rc;
  for (size_t b = 0; b < blocks_.size(); ++b)
    for (int j = 0; j < NCj; ++j)
      for (int i = 0; i < NCi; ++i) {
        Euler2D_Quad_Block& B = blocks_[b];
        for (int v = 1; v <= 4; ++v) {
          const size_t q = ((b * 4 + v - 1) * NCj + j) * NCi + i;
          B.W[i][j][v] = W[q];
          B.U[i][j][v] = U[q];
        }
      }
  return 0;
}

int Euler2D_Device_Blocks::residual() {
  if (!h_) return E2D_ERR_ARG;
  const int NCi = blocks_[0].NCi, NCj = blocks_[0].NCj;
  std::vector<double> R(blocks_.size() * 4 * size_t(NCi) * NCj);
  const int rc = e2d_residual(h_, R.data());
  if (rc) return rc;
  for (size_t b = 0; b < blocks_.size(); ++b)
    for (int v = 1; v <= 4; ++v)
      for (int j = 0; j < NCj; ++j)
        for (int i = 0; i < NCi; ++i) blocks_[b].dUdt[i][j][v] = R[((b * 4 + v - 1) * NCj + j) * NCi + i];
  return 0;
}

int Euler2D_Device_Blocks::explicit_steps(int n, std::vector<double>* hist) {
  if (!h_) return E2D_ERR_ARG;
  if (hist) hist->assign(size_t(4) * (n > 0 ? n : 1), 0.0);
  return e2d_rk_steps(h_, n, hist ? hist->data() : nullptr);
}

int Euler2D_Device_Blocks::nks(const e2d_nks_params& p, std::vector<e2d_nks_step>* hist) {
  if (!h_) return E2D_ERR_ARG;
  std::vector<e2d_nks_step> local(p.max_newton > 0 ? p.max_newton : 1);
  int n = 0;
  const int rc = e2d_nks(h_, &p, local.data(), &n);
  if (hist) hist->assign(local.begin(), local.begin() + n);
  return rc;
}

int Write_Case_File(const std::string& path, const std::vector<Euler2D_Quad_Block>& blocks,
                    const std::vector<int>& neighbour, const Euler2D_Input_Parameters& IP) {
  if (blocks.empty()) return E2D_ERR_ARG;
  Packed P;
  pack_blocks(blocks, neighbour, P);
  std::vector<double> W;
  gather_W(blocks, W);
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return E2D_ERR_ARG;
  const e2d_blocks_desc& d = P.desc;
  const e2d_scheme s = scheme_of(IP);
  const int NCi = d.nci + 2 * d.ng, NCj = d.ncj + 2 * d.ng, NNi = NCi + 1, NNj = NCj + 1;
  const int32_t head[14] = {0x43443245, 2, d.nblk, d.nci, d.ncj, d.ng, s.limiter, s.flux, s.n_stage, s.local_dt, 1,
                            IP.Number_of_Blocks_Idir, IP.Number_of_Blocks_Jdir,
                            IP.Grid_Type == "Periodic_Box" ? 1 : 0};
  const double headf[4] = {s.cfl, s.rs_epsilon, s.freeze_level, 0.0};
  const int32_t head2[4] = {s.time_integration, s.rs_iterations, s.freeze_limiter, 0};
  fwrite(head, sizeof(int32_t), 14, f);
  fwrite(headf, sizeof(double), 4, f);
  fwrite(head2, sizeof(int32_t), 4, f);
  for (int b = 0; b < d.nblk; ++b) {
    fwrite(P.neighbour.data() + 8 * b, sizeof(int32_t), 8, f);
    fwrite(P.bcw.data() + size_t(b) * NCj, sizeof(int32_t), NCj, f);
    fwrite(P.bce.data() + size_t(b) * NCj, sizeof(int32_t), NCj, f);
    fwrite(P.bcs.data() + size_t(b) * NCi, sizeof(int32_t), NCi, f);
    fwrite(P.bcn.data() + size_t(b) * NCi, sizeof(int32_t), NCi, f);
    fwrite(P.X.data() + size_t(b) * NNi * NNj, sizeof(double), size_t(NNi) * NNj, f);
    fwrite(P.Y.data() + size_t(b) * NNi * NNj, sizeof(double), size_t(NNi) * NNj, f);
    fwrite(P.wow.data() + size_t(b) * 4 * NCj, sizeof(double), size_t(4) * NCj, f);
    fwrite(P.woe.data() + size_t(b) * 4 * NCj, sizeof(double), size_t(4) * NCj, f);
    fwrite(P.wos.data() + size_t(b) * 4 * NCi, sizeof(double), size_t(4) * NCi, f);
    fwrite(P.won.data() + size_t(b) * 4 * NCi, sizeof(double), size_t(4) * NCi, f);
    fwrite(W.data() + size_t(b) * 4 * NCi * NCj, sizeof(double), size_t(4) * NCi * NCj, f);
  }
  return fclose(f) == 0 ? 0 : E2D_ERR_ARG;
}

// ---- single-block entry points ----------------------------------------------
int dUdt_Residual_Evaluation(Euler2D_Quad_Block& SolnBlk, const Euler2D_Input_Parameters& IP) {
  std::vector<Euler2D_Quad_Block> one(1, SolnBlk);
  std::vector<int> nb(8, -1);
  Euler2D_Device_Blocks dev(one, nb, IP);
  if (!dev.handle()) return E2D_ERR_CUDA;
  int rc = dev.residual();
  if (rc) return rc;
  SolnBlk.dUdt = one[0].dUdt;
  return 0;
}

// CFL (Euler2DQuadSingleBlock.cc:3019-3080): the device evaluates every
// interior cell's step into SolnBlk.dt; returns the block minimum (or a
// negative library error).
double CFL(Euler2D_Quad_Block& SolnBlk, const Euler2D_Input_Parameters& IP) {
  std::vector<Euler2D_Quad_Block> one(1, SolnBlk);
  std::vector<int> nb(8, -1);
  Euler2D_Device_Blocks dev(one, nb, IP);
  if (!dev.handle()) return E2D_ERR_CUDA;
  const int NCi = SolnBlk.NCi, NCj = SolnBlk.NCj;
  std::vector<double> dt(size_t(NCi) * NCj);
  double dtmin = 0.0;
  const int rc = e2d_cfl(dev.handle(), dt.data(), &dtmin);
  if (rc) return rc;
  for (int j = 0; j < NCj; ++j)
    for (int i = 0; i < NCi; ++i) SolnBlk.dt[i][j] = dt[size_t(j) * NCi + i];
  return dtmin;
}

double L1_Norm_Residual(const Euler2D_Quad_Block& B) {
  double s = 0.0;
  for (int j = B.JCl; j <= B.JCu; ++j)
    for (int i = B.ICl; i <= B.ICu; ++i) s += std::fabs(B.dUdt[i][j].d);
  return s;
}
double L2_Norm_Residual(const Euler2D_Quad_Block& B) {
  double s = 0.0;
  for (int j = B.JCl; j <= B.JCu; ++j)
    for (int i = B.ICl; i <= B.ICu; ++i) s += B.dUdt[i][j].d * B.dUdt[i][j].d;
  return std::sqrt(s);
}
double Max_Norm_Residual(const Euler2D_Quad_Block& B) {
  double m = 0.0;
  for (int j = B.JCl; j <= B.JCu; ++j)
    for (int i = B.ICl; i <= B.ICu; ++i) m = std::fmax(m, std::fabs(B.dUdt[i][j].d));
  return m;
}

// ---- restart files --------------------------------------------------------------
namespace {

// Restart_File_Name up to its first ' ' or '.' (Euler2DQuadMultiBlock.cc:160-168).
std::string restart_prefix(const Euler2D_Input_Parameters& IP) {
  return IP.Restart_File_Name.substr(0, IP.Restart_File_Name.find_first_of(" ."));
}
std::string soln_file(const Euler2D_Input_Parameters& IP, int gblknum) {
  char ext[32];
  snprintf(ext, sizeof(ext), "%.6d.soln", gblknum);
  return restart_prefix(IP) + "_blk" + ext;
}
std::string tree_file(const Euler2D_Input_Parameters& IP) { return restart_prefix(IP) + "_quadtree.tree"; }

// quadCentroid (Math.h:311-351) on (SW, SE, NE, NW): the cell centroid and
// area Grid2D_Quad_Block_HO::Update_Cells stores and the restart file lists.
void quad_centroid(const Vector2D& p0, const Vector2D& p1, const Vector2D& p2, const Vector2D& p3, Vector2D& c,
                   double& area) {
  const Vector2D p[4] = {p0, p1, p2, p3};
  double atmp = 0.0, xt = 0.0, yt = 0.0;
  for (int k = 0; k < 4; ++k) {
    const Vector2D& a = p[(k + 3) % 4];
    const Vector2D& b = p[k];
    const double ai = a.x * b.y - b.x * a.y;
    atmp += ai;
    xt += (b.x + a.x) * ai;
    yt += (b.y + a.y) * ai;
  }
  area = 0.5 * atmp;
  if (atmp != 0.0) {
    c.x = xt / (3.0 * atmp);
    c.y = yt / (3.0 * atmp);
  } else {
    c.x = c.y = 0.0;
  }
}

// Stream forms of the reference's types (Vector2D, Euler2D_pState /
// cState: a leading blank, scientific; Math/Vector2D.h:433,
// Euler2DState.h:1349, 1724).
void put_vec(std::ostream& o, double x, double y) {
  o.setf(std::ios::scientific);
  o << " " << x << " " << y;
  o.unsetf(std::ios::scientific);
}
void put_state(std::ostream& o, double a, double b, double c, double d) {
  o.setf(std::ios::scientific);
  o << " " << a << " " << b << " " << c << " " << d;
  o.unsetf(std::ios::scientific);
}

// operator<<(ostream&, Grid2D_Quad_Block_HO) (Grid/HO_Grid2DQuad.cc:
// 13763-13990) of a first-order geometry without boundary splines or
// stretching; it leaves the stream at precision 15.
void put_grid(std::ostream& o, const Euler2D_Quad_Block& B) {
  const Grid2D_Quad_Block& G = B.Grid;
  const int ng = B.Nghost, NCi = B.NCi, NCj = B.NCj;
  o << G.NNi << " " << ng << " " << G.NNi - ng - 1 << "\n";
  o << G.NNj << " " << ng << " " << G.NNj - ng - 1 << "\n";
  o << ng << "\n" << 0 << "\n" << 0 << "\n";
  o << NCi << " " << B.ICl << " " << B.ICu << "\n";
  o << NCj << " " << B.JCl << " " << B.JCu << "\n";
  o.precision(15);
  for (int j = 0; j < G.NNj; ++j)
    for (int i = 0; i < G.NNi; ++i) {
      put_vec(o, G.Node[i][j].x, G.Node[i][j].y);
      o << "\n";
    }
  for (int j = 0; j < NCj; ++j)
    for (int i = 0; i < NCi; ++i) {
      Vector2D c;
      double A;
      quad_centroid(G.Node[i][j], G.Node[i + 1][j], G.Node[i + 1][j + 1], G.Node[i][j + 1], c, A);
      o << " " << i << " " << j;
      put_vec(o, c.x, c.y);
      o.setf(std::ios::scientific);
      o << " " << A << "\n";
      o.unsetf(std::ios::scientific);
      // geometric moments of order 0: the single moment (0, 0) = 1
      // (TaylorDerivatives2D.h:143-150, 808-817)
      o << " ";
      o.width(4);
      o << 0 << std::endl;
      o.width(4);
      o << 0;
      o.width(4);
      o << 0;
      o.precision(15);
      o.width(25);
      o << 1.0 << std::endl;
      o << "\n";
    }
  for (int i = 0; i < NCi; ++i) o << G.BCtypeN[i] << " " << G.BCtypeS[i] << "\n";
  for (int j = 0; j < NCj; ++j) o << G.BCtypeE[j] << " " << G.BCtypeW[j] << "\n";
  for (int k = 0; k < 12; ++k) o << 0 << "\n" << 0 << "\n";  // no boundary splines
  o.setf(std::ios::scientific);
  o << 0.0 << " " << 0.0 << " " << 0.0 << " " << 0.0 << "\n";
  o << 0.0 << " " << 0.0 << " " << 0.0 << " " << 0.0 << "\n";
  o << 0 << " " << 1.0 << " " << 1.0 << "\n";
  o << 0 << " " << 1.0 << " " << 1.0 << "\n";
  o.unsetf(std::ios::scientific);
  o << 1 << " " << 1 << " " << 1 << " " << 1 << "\n";
}

// One block in the layout of operator<<(ostream&, Euler2D_Quad_Block)
// (Euler2DQuad.h:1306-1336).
void put_block(std::ostream& o, const Euler2D_Quad_Block& B) {
  const int ng = B.Nghost, NCi = B.NCi, NCj = B.NCj;
  put_grid(o, B);
  o << NCi << " " << B.ICl << " " << B.ICu << " " << ng << "\n";
  o << NCj << " " << B.JCl << " " << B.JCu << "\n";
  o << 0 << "\n";  // Axisymmetric
  for (int j = 0; j < NCj; ++j)
    for (int i = 0; i < NCi; ++i) {
      const Euler2D_cState& U = B.U[i][j];
      put_state(o, U.d, U.dv.x, U.dv.y, U.E);
      o << "\n";
    }
  for (int j = 0; j < NCj; ++j) {
    put_state(o, B.WoW[j].d, B.WoW[j].v.x, B.WoW[j].v.y, B.WoW[j].p);
    o << "\n";
    put_state(o, B.WoE[j].d, B.WoE[j].v.x, B.WoE[j].v.y, B.WoE[j].p);
    o << "\n";
  }
  for (int i = 0; i < NCi; ++i) {
    put_state(o, B.WoS[i].d, B.WoS[i].v.x, B.WoS[i].v.y, B.WoS[i].p);
    o << "\n";
    put_state(o, B.WoN[i].d, B.WoN[i].v.x, B.WoN[i].v.y, B.WoN[i].p);
    o << "\n";
  }
  o << 0 << "\n";  // NumberOfHighOrderVariables
}

// Whitespace-separated reading, as the reference's istream >> with skipws.
template <class T> bool get(std::istream& in, T& v) { return static_cast<bool>(in >> v); }
bool skip(std::istream& in, long n) {
  std::string t;
  for (long k = 0; k < n; ++k)
    if (!(in >> t)) return false;
  return true;
}

// Spline2D_HO and its Spline2DInterval_HO list (Grid/HO_Spline2D.h:808-830,
// Grid/HO_Spline2DInterval.h:271-330): read and dropped.
bool skip_spline(std::istream& in) {
  long np, n;
  if (!get(in, np)) return false;
  if (np != 0 && !skip(in, 4 + 4 * np)) return false;
  if (!get(in, n)) return false;
  for (long k = 0; k < n; ++k) {
    long nsub, ngq;
    if (!get(in, nsub) || !get(in, ngq)) return false;
    // lengths; per Gauss point its position and normal; per contour-integral
    // point (3 per subinterval) its position and dy/ds
    if (!skip(in, nsub + 4 * nsub * ngq + 3 * 3 * nsub)) return false;
  }
  return true;
}

// operator>>(istream&, Grid2D_Quad_Block_HO) (Grid/HO_Grid2DQuad.cc:
// 14006-14200): nodes and BC codes kept, cell data and splines dropped;
// allocates the block.
bool get_grid(std::istream& in, Euler2D_Quad_Block& B) {
  int nni, inl, inu, nnj, jnl, jnu, ng, rec, bflag, nci, icl, icu, ncj, jcl, jcu;
  if (!(in >> nni >> inl >> inu >> nnj >> jnl >> jnu >> ng >> rec >> bflag)) return false;
  if (nni == 0 || nnj == 0) return false;
  if (!(in >> nci >> icl >> icu >> ncj >> jcl >> jcu)) return false;
  if (nci != nni - 1 || ncj != nnj - 1 || nci <= 2 * ng || ncj <= 2 * ng) return false;
  B.allocate(nci - 2 * ng, ncj - 2 * ng, ng);
  Grid2D_Quad_Block& G = B.Grid;
  for (int j = 0; j < nnj; ++j)
    for (int i = 0; i < nni; ++i)
      if (!(in >> G.Node[i][j].x >> G.Node[i][j].y)) return false;
  const long moments = long(rec + 1) * (rec + 2) / 2;
  for (int j = 0; j < ncj; ++j)
    for (int i = 0; i < nci; ++i) {
      int order;
      if (!skip(in, 5) || !get(in, order) || order != rec || !skip(in, 3 * moments)) return false;
    }
  for (int i = 0; i < nci; ++i)
    if (!(in >> G.BCtypeN[i] >> G.BCtypeS[i])) return false;
  for (int j = 0; j < ncj; ++j)
    if (!(in >> G.BCtypeE[j] >> G.BCtypeW[j])) return false;
  for (int k = 0; k < 12; ++k)
    if (!skip_spline(in)) return false;
  return skip(in, 8 + 6 + 4);  // Smin/Smax, stretching, orthogonality flags
}

// operator>>(istream&, Euler2D_Quad_Block) (Euler2DQuad.h:1338-1400).
bool get_block(std::istream& in, Euler2D_Quad_Block& B) {
  if (!get_grid(in, B)) return false;
  const int nci = B.NCi, ncj = B.NCj, ng = B.Nghost;
  int ni, il, iu, g2, nj, jl, ju, axi;
  if (!(in >> ni >> il >> iu >> g2 >> nj >> jl >> ju >> axi)) return false;
  if (ni != nci || nj != ncj || g2 != ng) return false;
  for (int j = 0; j < ncj; ++j)
    for (int i = 0; i < nci; ++i) {
      Euler2D_cState& U = B.U[i][j];
      if (!(in >> U.d >> U.dv.x >> U.dv.y >> U.E)) return false;
      B.W[i][j] = U.W();
    }
  for (int j = 0; j < ncj; ++j) {
    Euler2D_pState& w = B.WoW[j];
    Euler2D_pState& e = B.WoE[j];
    if (!(in >> w.d >> w.v.x >> w.v.y >> w.p >> e.d >> e.v.x >> e.v.y >> e.p)) return false;
  }
  for (int i = 0; i < nci; ++i) {
    Euler2D_pState& s = B.WoS[i];
    Euler2D_pState& n = B.WoN[i];
    if (!(in >> s.d >> s.v.x >> s.v.y >> s.p >> n.d >> n.v.x >> n.v.y >> n.p)) return false;
  }
  int n_ho;
  return get(in, n_ho) && n_ho == 0;  // high-order variables are outside this path
}

// One node of the block tree (QuadTreeBlock::read, AMR/QuadTree.h:357-385,
// with AdaptiveBlock2D operator>>, AMR/AdaptiveBlock.h:720-760).
struct TreeLeaf {
  int gblknum, cpu, blknum, level;
  int n[8];          // neighbour counts N S E W NW NE SE SW
  int ncpu[8], nblk[8], nlevel[8];
};
bool read_tree_node(std::istream& in, std::vector<TreeLeaf>& leaves) {
  int used, gbl, cpu, blk, di, dj, dg, sector, level;
  if (!(in >> used >> gbl >> cpu >> blk >> di >> dj >> dg >> sector >> level)) return false;
  TreeLeaf L{};
  L.gblknum = gbl; L.cpu = cpu; L.blknum = blk; L.level = level;
  for (int s = 0; s < 8; ++s) {
    if (!get(in, L.n[s])) return false;
    for (int k = 0; k < L.n[s]; ++k) {
      int c, b, i, j, g, sec, lev;
      if (!(in >> c >> b >> i >> j >> g >> sec >> lev)) return false;
      if (k == 0) { L.ncpu[s] = c; L.nblk[s] = b; L.nlevel[s] = lev; }
    }
  }
  int children;
  if (!get(in, children)) return false;
  if (used) leaves.push_back(L);
  if (!used && children > 0)
    for (int k = 0; k < 4; ++k)
      if (!read_tree_node(in, leaves)) return false;
  return true;
}

// AdaptiveBlock2D_Info of a same-level root block on CPU 0 (AMR/AdaptiveBlock.h:502-509).
void put_info(std::ostream& o, int blknum, const Euler2D_Quad_Block& B) {
  o << " " << 0 << " " << blknum << " " << B.ICu - B.ICl + 1 << " " << B.JCu - B.JCl + 1 << " " << B.Nghost
    << " " << -1 << " " << 0;
}

}  // namespace

namespace {
// The nbi x nbj root layout of a block set numbered b = j * nbi + i: the
// deck's, or (for a grid read from a file) the run of east neighbours from
// block 0.
bool root_layout(const std::vector<int>& neighbour, int nblk, const Euler2D_Input_Parameters& IP, int& nbi,
                 int& nbj) {
  nbi = IP.Number_of_Blocks_Idir;
  nbj = IP.Number_of_Blocks_Jdir;
  if (nbi * nbj == nblk) return true;
  if (neighbour.size() != size_t(8) * nblk) return false;
  nbi = 1;
  for (int b = 0; neighbour[8 * b + 1] > b; b = neighbour[8 * b + 1]) ++nbi;
  nbj = nblk / nbi;
  return nbi * nbj == nblk;
}

// i_Grid codes of the grid names this library builds or reads (CFD/CFD.h:800-860).
int grid_code(const std::string& t) {
  if (t == "Rectangular_Box") return 2;
  if (t == "Bump_Channel_Flow") return 16;
  if (t == "Periodic_Box") return 55;
  return 10001;  // GRID_READ_FROM_GRID_DATA_FILE
}
}  // namespace

int Write_Multi_Block_Grid(const std::string& path, const std::vector<Euler2D_Quad_Block>& blocks,
                           const Euler2D_Input_Parameters& IP) {
  const int nbi = IP.Number_of_Blocks_Idir, nbj = IP.Number_of_Blocks_Jdir;
  if (blocks.empty() || size_t(nbi) * nbj != blocks.size()) return 1;
  std::ofstream o(path);
  if (!o.good()) return 1;
  o << IP.Grid_Type << "\n" << grid_code(IP.Grid_Type) << "\n";
  o << nbi << " " << nbj << "\n";
  for (const Euler2D_Quad_Block& B : blocks) {
    o.precision(14);  // Grid2D_Quad_Block_HO::Write_Quad_Block
    put_grid(o, B);
    o.precision(6);
  }
  return o.good() ? 0 : 1;
}

int Read_Multi_Block_Grid(const std::string& path, std::vector<Euler2D_Quad_Block>& blocks,
                          std::vector<int>& neighbour, std::string* grid_type, int* nbi_out, int* nbj_out) {
  std::ifstream in(path);
  if (!in.good()) return 1;
  std::string type;
  int code, nbi, nbj;
  std::getline(in, type);
  if (!(in >> code >> nbi >> nbj) || nbi < 1 || nbj < 1) return 1;
  if (grid_type) *grid_type = type;
  if (nbi_out) *nbi_out = nbi;
  if (nbj_out) *nbj_out = nbj;
  blocks.assign(size_t(nbi) * nbj, Euler2D_Quad_Block());
  for (Euler2D_Quad_Block& B : blocks)
    if (!get_grid(in, B)) return 1;
  for (const Euler2D_Quad_Block& B : blocks)
    if (B.NCi != blocks[0].NCi || B.NCj != blocks[0].NCj) return 1;
  // root blocks of the layout (Find_Neighbours_of_Root_Solution_Blocks,
  // AMR/QuadTree.cc:363, with the periodic-box wiring of GRID_PERIODIC_BOX)
  // (several blocks in both directions)
  const bool periodic = code == 55 && nbi > 1 && nbj > 1;
  static const int off[8][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
  neighbour.assign(size_t(8) * nbi * nbj, -1);
  for (int bj = 0; bj < nbj; ++bj)
    for (int bi = 0; bi < nbi; ++bi)
      for (int k = 0; k < 8; ++k) {
        int ni = bi + off[k][0], nj = bj + off[k][1];
        if (periodic) { ni = (ni + nbi) % nbi; nj = (nj + nbj) % nbj; }
        if (ni >= 0 && ni < nbi && nj >= 0 && nj < nbj) neighbour[8 * (bj * nbi + bi) + k] = nj * nbi + ni;
      }
  return 0;
}

int Write_QuadTree(const std::vector<Euler2D_Quad_Block>& blocks, const std::vector<int>& neighbour,
                   const Euler2D_Input_Parameters& IP) {
  const int nblk = static_cast<int>(blocks.size());
  int nbi, nbj;
  if (!root_layout(neighbour, nblk, IP, nbi, nbj)) return 1;
  std::ofstream o(tree_file(IP));
  if (!o.good()) return 1;
  o << nbi << " " << nbj << " " << 1 << " "
    << std::max(nblk, IP.Number_of_Blocks_Per_Processor) << "\n";
  // neighbour slots in the tree's order N S E W NW NE SE SW (ours: W E S N SW SE NW NE)
  static const int slot[8] = {3, 2, 1, 0, 6, 7, 5, 4};
  for (int b = 0; b < nblk; ++b) {
    o << " " << 1 << " " << b;
    put_info(o, b, blocks[b]);
    for (int s = 0; s < 8; ++s) {
      const int nb = neighbour[8 * b + slot[s]];
      o << "\n " << (nb >= 0 ? 1 : 0);
      if (nb >= 0) {
        o << " ";
        put_info(o, nb, blocks[nb]);
      }
    }
    o << "\n" << " " << 0 << "\n";
  }
  return o.good() ? 0 : 1;
}

int Write_Restart_Solution(const std::vector<Euler2D_Quad_Block>& blocks, const Euler2D_Input_Parameters& IP,
                           int Number_of_Time_Steps, double Time, double CPU_Time) {
  for (size_t b = 0; b < blocks.size(); ++b) {
    std::ofstream o(soln_file(IP, static_cast<int>(b)));
    if (!o.good()) return 1;
    o.setf(std::ios::scientific);
    o.precision(14);
    o << Number_of_Time_Steps << " " << Time << " ";
    o << " " << CPU_Time << "\n";
    o.unsetf(std::ios::scientific);
    o << IP.Gas_Type << "\n";
    o.precision(14);
    put_block(o, blocks[b]);
    if (!o.good()) return 1;
  }
  return 0;
}

int Read_QuadTree(std::vector<Euler2D_Quad_Block>& blocks, std::vector<int>& neighbour,
                  Euler2D_Input_Parameters& IP) {
  std::ifstream in(tree_file(IP));
  if (!in.good()) return 1;
  int nri, nrj, ncpu, nblk;
  if (!(in >> nri >> nrj >> ncpu >> nblk) || nri < 1 || nrj < 1) return 1;
  IP.Number_of_Blocks_Idir = nri;
  IP.Number_of_Blocks_Jdir = nrj;
  IP.Number_of_Blocks_Per_Processor = nblk;
  std::vector<TreeLeaf> leaves;
  for (int r = 0; r < nri * nrj; ++r)
    if (!read_tree_node(in, leaves)) return 1;
  const int n = static_cast<int>(leaves.size());
  std::vector<int> order(n, -1);  // gblknum -> leaf
  for (int k = 0; k < n; ++k) {
    const int g = leaves[k].gblknum;
    if (g < 0 || g >= n || order[g] >= 0 || leaves[k].level != leaves[0].level) return 1;
    order[g] = k;
  }
  auto find = [&](int cpu, int blk) {
    for (int k = 0; k < n; ++k)
      if (leaves[k].cpu == cpu && leaves[k].blknum == blk) return leaves[k].gblknum;
    return -1;
  };
  static const int slot[8] = {3, 2, 1, 0, 6, 7, 5, 4};  // tree side -> W E S N SW SE NW NE
  neighbour.assign(size_t(8) * n, -1);
  for (int g = 0; g < n; ++g) {
    const TreeLeaf& L = leaves[order[g]];
    for (int s = 0; s < 8; ++s) {
      if (L.n[s] == 0) continue;
      if (L.n[s] != 1 || L.nlevel[s] != L.level) return 1;  // a resolution change
      const int nb = find(L.ncpu[s], L.nblk[s]);
      if (nb < 0) return 1;
      neighbour[8 * g + slot[s]] = nb;
    }
  }
  blocks.assign(n, Euler2D_Quad_Block());
  return 0;
}

int Read_Restart_Solution(std::vector<Euler2D_Quad_Block>& blocks, Euler2D_Input_Parameters& IP,
                          int& Number_of_Time_Steps, double& Time, double& CPU_Time) {
  for (size_t b = 0; b < blocks.size(); ++b) {
    std::ifstream in(soln_file(IP, static_cast<int>(b)));
    if (!in.good()) return 1;
    int nsteps;
    double t, cpu;
    std::string rest, gas;
    if (!(in >> nsteps >> t >> cpu)) return 1;
    std::getline(in, rest);
    std::getline(in, gas);
    if (b == 0) {
      Number_of_Time_Steps = nsteps;
      IP.Maximum_Number_of_Time_Steps += nsteps;
      Time = t;
      CPU_Time = cpu;
      if (gas != IP.Gas_Type) IP.Gas_Type = gas;
    }
    if (!get_block(in, blocks[b])) return 1;
  }
  return 0;
}

// ---- solver driver (Euler2DQuadSolver, Euler2DQuadSolvers.cc:26-1100) --------
int Euler2DQuadSolver(const char* Input_File_Name_ptr, int batch_flag) {
  Euler2D_Input_Parameters IP;
  int rc = IP.Process_Input_Control_Parameter_File(Input_File_Name_ptr);
  if (rc) {
    if (!batch_flag) fprintf(stderr, "Euler2DQuadSolver: error reading %s at line %d\n", Input_File_Name_ptr, rc);
    return rc > 0 ? rc : E2D_ERR_ARG;
  }
  std::vector<Euler2D_Quad_Block> blocks;
  std::vector<int> neighbour;
  int number_of_time_steps = 0;
  double Time = 0.0, cpu_time = 0.0;
  const bool restart = IP.ICs_Type == "Restart";
  if (restart) {  // Euler2DQuadSolvers.cc:223-270
    if (Read_QuadTree(blocks, neighbour, IP) ||
        Read_Restart_Solution(blocks, IP, number_of_time_steps, Time, cpu_time))
      return E2D_ERR_ARG;
  } else if ((rc = Create_Initial_Solution_Blocks(IP, blocks, neighbour))) {
    return E2D_ERR_ARG;
  }
  Euler2D_Device_Blocks dev(blocks, neighbour, IP);
  if (!dev.handle()) return E2D_ERR_CUDA;
  if (restart && (rc = dev.upload_conserved())) return rc;
  const std::clock_t c0 = std::clock();
  auto save = [&]() -> bool {  // Write_QuadTree + Write_Restart_Solution of the current state
    if (dev.download()) return true;
    const double cpu = cpu_time + double(std::clock() - c0) / CLOCKS_PER_SEC;
    return Write_QuadTree(blocks, neighbour, IP) != 0 ||
           Write_Restart_Solution(blocks, IP, number_of_time_steps, Time, cpu) != 0;
  };
  // the explicit loop in chunks that end where the reference saves restart
  // files (every Restart_Solution_Save_Frequency steps, not at its first step)
  std::vector<double> hist;
  const int first = number_of_time_steps, freq = IP.Restart_Solution_Save_Frequency;
  while (number_of_time_steps < IP.Maximum_Number_of_Time_Steps) {
    const int n = std::min(IP.Maximum_Number_of_Time_Steps - number_of_time_steps,
                           freq - number_of_time_steps % freq);
    std::vector<double> h;
    if ((rc = dev.explicit_steps(n, &h))) return rc;
    for (int k = 0; k < n; ++k) Time += IP.CFL_Number * h[4 * k];
    hist.insert(hist.end(), h.begin(), h.begin() + 4 * n);
    number_of_time_steps += n;
    if (number_of_time_steps % freq == 0 && number_of_time_steps > first && save()) return E2D_ERR_ARG;
  }
  // ghost exchange and BCs of the final explicit state (Euler2DQuadSolvers.cc:901-925)
  if (number_of_time_steps > first && (rc = e2d_fill_ghosts(dev.handle()))) return rc;
  std::vector<e2d_nks_step> nks_hist;
  if (IP.NKS.max_newton > 0) {
    if ((rc = dev.nks(IP.NKS, &nks_hist))) return rc;
  }
  if ((rc = dev.download())) return rc;
  // commands after Execute (Euler2DQuadSolvers.cc:1317-1360 for Write_Restart)
  for (const std::string& c : IP.Commands)
    if (c == "Write_Restart" && save()) return E2D_ERR_ARG;
  // cell-centred output: one zone per block (x, y of the cell centroid
  // average of its nodes; rho, u, v, p)
  FILE* f = fopen(IP.Output_File_Name.c_str(), "w");
  if (!f) return E2D_ERR_ARG;
  fprintf(f, "TITLE = \"Euler2D solution\"\nVARIABLES = \"x\" \"y\" \"rho\" \"u\" \"v\" \"p\"\n");
  for (size_t b = 0; b < blocks.size(); ++b) {
    const Euler2D_Quad_Block& B = blocks[b];
    fprintf(f, "ZONE T = \"Block %zu\" I = %d J = %d F = POINT\n", b, B.ICu - B.ICl + 1, B.JCu - B.JCl + 1);
    for (int j = B.JCl; j <= B.JCu; ++j)
      for (int i = B.ICl; i <= B.ICu; ++i) {
        const auto& N = B.Grid.Node;
        const double x = 0.25 * (N[i][j].x + N[i + 1][j].x + N[i + 1][j + 1].x + N[i][j + 1].x);
        const double y = 0.25 * (N[i][j].y + N[i + 1][j].y + N[i + 1][j + 1].y + N[i][j + 1].y);
        const Euler2D_pState& w = B.W[i][j];
        fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", x, y, w.d, w.v.x, w.v.y, w.p);
      }
  }
  fclose(f);
  if (!batch_flag) {
    if (!hist.empty())
      printf("explicit: %d steps, last L2 = %.10g\n", IP.Maximum_Number_of_Time_Steps, hist[hist.size() - 2]);
    for (size_t k = 0; k < nks_hist.size(); ++k)
      printf("Newton Step %zu L2norm = %.10g L2norm_ratio = %.10g CFL = %.10g GMRES = %d\n", k + 1, nks_hist[k].l2,
             nks_hist[k].ratio, nks_hist[k].cfl, nks_hist[k].gmres_iters);
  }
  return 0;
}

}  // namespace cffc_b200

// C entry of the deck-driven solve (for callers without C++ linkage).
extern "C" int e2d_solver_run(const char* input_file, int batch_flag) {
  if (!input_file) return E2D_ERR_ARG;
  return cffc_b200::Euler2DQuadSolver(input_file, batch_flag);
}

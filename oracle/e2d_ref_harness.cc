// e2d_ref_harness: drives the compiled CFFC reference (oracle/_ref/libcffc_ref.a)
// on a block set described by an e2d case file, and writes what the
// reference computes.  Test infrastructure only: it generates golden vectors,
// pins the C restatement (oracle/e2d_oracle.c) and times the reference's CPU
// path.  The product never links or runs it.
//
// The block set is handed to the reference as its initial multi-block mesh:
// one Grid2D_Quad_Block_HO per block with the case's nodes (ghost nodes
// included) and BC types, geometry from Grid2D_Quad_Block_HO::Update_Cells
// (src_2D/Grid/HO_Grid2DQuad.cc:9832).  The reference's own
// Create_Initial_Solution_Blocks (src_2D/AMR/AMR.h:40) then builds the
// quadtree, the neighbour lists (periodic-box wiring, src_2D/AMR/QuadTree.cc:363,
// when the case is periodic) and the message buffers, so every step below is
// the reference's own code:
//   residual   Send_All_Messages (AMR/AdaptiveBlock2D_MessagePassing.h:7883),
//              BCs (Euler2DQuadMultiBlock.cc:937),
//              dUdt_Residual_Evaluation (Euler2DQuadSingleBlock.cc:5095)
//   explicit   the explicit loop of Euler2DQuadSolvers.cc:657-898 with the
//              multi-block CFL, Set_Global_TimeStep, L1/L2/Max norms,
//              dUdt_Multistage_Explicit, Update_Solution_Multistage_Explicit
//   nks        Newton_Krylov_Schwarz_Solver (NewtonKrylovSchwarz2D/NKS2D.h:136)
// The "time" mode runs the explicit step with the reference's per-block
// routines on POSIX threads (blocks are independent between ghost
// exchanges, as on the reference's MPI ranks) and a restated same-resolution
// exchange, a plain copy of the neighbours' two edge layers of U followed by
// W = U.W() (Euler2D_Quad_Block::LoadSendBuffer/UnloadReceiveBuffer,
// src_2D/Euler2D/Euler2DQuad.h:1570-1650); the golden tests show the two agree.
//
// usage:
//   e2d_ref_harness residual CASE OUT
//   e2d_ref_harness explicit CASE NSTEPS OUT
//   e2d_ref_harness nks      CASE OUT MAX_NEWTON GMRES_RESTART MAX_GMRES CFL0 OVERALL_TOL [GMRES_TOL
//                            [ILUK|Diagonal LEVEL]]
//   e2d_ref_harness precon   CASE OUT CFL ILUK|Diagonal LEVEL VFILE
//   e2d_ref_harness time     CASE NSTEPS THREADS      (prints one JSON line)
//   e2d_ref_harness restart_write CASE PREFIX NSTEPS TIME  (Write_QuadTree + Write_Restart_Solution)
//   e2d_ref_harness restart_read  CASE PREFIX OUT [GRIDFILE]
//   e2d_ref_harness grid_write    CASE GRIDFILE
//   e2d_ref_harness solve    DECK                      (Euler2DQuadSolver in batch mode)
//
// Case file (little endian), shared with cffc_b200/cases.py:
//   int32 magic 0x43443245, version 1 or 2
//   int32 nblk, nci, ncj, ng
//   int32 limiter, flux, n_stage, local_dt, time_accurate, nbi, nbj, periodic
//   f64   cfl, rs_epsilon, freeze_level, 0         (version 1: cfl, 0, 0, 0)
//   int32 time_integration, rs_iterations, freeze_limiter, 0   (version 2 only)
//   per block (b = bj * nbi + bi):
//     int32 neighbour[8]           W, E, S, N, SW, SE, NW, NE (-1 = none)
//     int32 bcW[NCj], bcE[NCj], bcS[NCi], bcN[NCi]      reference BC codes
//     f64   X[NNj][NNi], Y[NNj][NNi]                    nodes incl. ghosts
//     f64   WoW[4][NCj], WoE[4][NCj], WoS[4][NCi], WoN[4][NCi]
//     f64   W[4][NCj][NCi]                              (rho, u, v, p)
// with NCi = nci + 2 ng, NNi = NCi + 1 (likewise j).  Arrays are [var][j][i].
#include <pthread.h>
#include <time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include "Euler2D/Euler2DQuad.h"
#include "Euler2D/Euler2DInput.h"
#include "AMR/AMR.h"
#include "NewtonKrylovSchwarz2D/NKS2D.h"
#include "Euler2D/Euler2DQuadNKS.h"

namespace {

struct BlockData {
  int neigh[8];
  std::vector<int> bcw, bce, bcs, bcn;
  std::vector<double> X, Y, wow, woe, wos, won, W;
};

struct Case {
  int nblk, nci, ncj, ng, NCi, NCj, NNi, NNj;
  int limiter, flux, n_stage, local_dt, time_accurate, nbi, nbj, periodic;
  double cfl;
  // version 2: scheme, residual smoothing and limiter freezing
  int time_integration = 0, rs_iterations = 2, freeze_limiter = 0;
  double rs_epsilon = 0.0, freeze_level = 1e-4;
  std::vector<BlockData> data;
};

template <class T> void rd(FILE* f, T* p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}
template <class T> void wr(FILE* f, const T* p, size_t n) { fwrite(p, sizeof(T), n, f); }

void read_case(const char* path, Case& c) {
  FILE* f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  int hdr[2], dims[4], opts[8];
  double dopts[4];
  rd(f, hdr, 2);
  if (hdr[0] != 0x43443245 || (hdr[1] != 1 && hdr[1] != 2)) { fprintf(stderr, "bad case file\n"); exit(2); }
  rd(f, dims, 4); rd(f, opts, 8); rd(f, dopts, 4);
  if (hdr[1] == 2) {
    int opts2[4];
    rd(f, opts2, 4);
    c.time_integration = opts2[0]; c.rs_iterations = opts2[1]; c.freeze_limiter = opts2[2];
    c.rs_epsilon = dopts[1]; c.freeze_level = dopts[2];
  }
  c.nblk = dims[0]; c.nci = dims[1]; c.ncj = dims[2]; c.ng = dims[3];
  c.NCi = c.nci + 2 * c.ng; c.NCj = c.ncj + 2 * c.ng; c.NNi = c.NCi + 1; c.NNj = c.NCj + 1;
  c.limiter = opts[0]; c.flux = opts[1]; c.n_stage = opts[2]; c.local_dt = opts[3];
  c.time_accurate = opts[4]; c.nbi = opts[5]; c.nbj = opts[6]; c.periodic = opts[7];
  c.cfl = dopts[0];
  if (c.nbi * c.nbj != c.nblk) { fprintf(stderr, "case has no structured block layout\n"); exit(2); }
  c.data.resize(c.nblk);
  for (int b = 0; b < c.nblk; ++b) {
    BlockData& d = c.data[b];
    rd(f, d.neigh, 8);
    d.bcw.resize(c.NCj); d.bce.resize(c.NCj); d.bcs.resize(c.NCi); d.bcn.resize(c.NCi);
    rd(f, &d.bcw[0], c.NCj); rd(f, &d.bce[0], c.NCj); rd(f, &d.bcs[0], c.NCi); rd(f, &d.bcn[0], c.NCi);
    d.X.resize(c.NNi * c.NNj); d.Y.resize(c.NNi * c.NNj);
    rd(f, &d.X[0], d.X.size()); rd(f, &d.Y[0], d.Y.size());
    d.wow.resize(4 * c.NCj); d.woe.resize(4 * c.NCj); d.wos.resize(4 * c.NCi); d.won.resize(4 * c.NCi);
    rd(f, &d.wow[0], d.wow.size()); rd(f, &d.woe[0], d.woe.size());
    rd(f, &d.wos[0], d.wos.size()); rd(f, &d.won[0], d.won.size());
    d.W.resize(4 * c.NCi * c.NCj);
    rd(f, &d.W[0], d.W.size());
  }
  fclose(f);
}

void set_input(const Case& c, Euler2D_Input_Parameters& IP) {
  Set_Default_Input_Parameters(IP);
  IP.i_Reconstruction = RECONSTRUCTION_LEAST_SQUARES;
  IP.i_Limiter = c.limiter;
  IP.i_Flux_Function = c.flux;
  // scheme code 0 runs as the Runge-Kutta family (N_Stage 1 or 2)
  IP.i_Time_Integration = c.time_integration == 0 ? TIME_STEPPING_EXPLICIT_RUNGE_KUTTA : c.time_integration;
  IP.N_Stage = c.n_stage;
  IP.Residual_Smoothing = c.rs_epsilon > 0.0 ? 1 : 0;
  IP.Residual_Smoothing_Epsilon = c.rs_epsilon;
  IP.Residual_Smoothing_Gauss_Seidel_Iterations = c.rs_iterations;
  IP.Freeze_Limiter = c.freeze_limiter;
  IP.Freeze_Limiter_Residual_Level = c.freeze_level;
  IP.CFL_Number = c.cfl;
  IP.Local_Time_Stepping = c.local_dt ? SCALAR_LOCAL_TIME_STEPPING : GLOBAL_TIME_STEPPING;
  IP.Time_Accurate = c.time_accurate;
  IP.Axisymmetric = 0;
  IP.Number_of_Ghost_Cells = c.ng;
  IP.Number_of_Blocks_Idir = c.nbi;
  IP.Number_of_Blocks_Jdir = c.nbj;
  IP.Number_of_Processors = 1;
  IP.Number_of_Blocks_Per_Processor = c.nblk;
  IP.Maximum_Refinement_Level = 1;
  IP.Minimum_Refinement_Level = 1;
  IP.i_Grid = c.periodic ? GRID_PERIODIC_BOX : GRID_RECTANGULAR_BOX;
}

// Fills one block's state from the case.
void load_state(const Case& c, const BlockData& d, Euler2D_Quad_Block& B) {
  const int s = c.NCi * c.NCj;
  for (int j = 0; j < c.NCj; ++j)
    for (int i = 0; i < c.NCi; ++i) {
      const int q = j * c.NCi + i;
      B.W[i][j] = Euler2D_pState(d.W[q], d.W[s + q], d.W[2 * s + q], d.W[3 * s + q]);
      B.U[i][j] = U(B.W[i][j]);
    }
  Euler2D_pState* Wo_dst[4] = {B.WoW, B.WoE, B.WoS, B.WoN};
  const std::vector<double>* Wo_src[4] = {&d.wow, &d.woe, &d.wos, &d.won};
  const int Wo_len[4] = {c.NCj, c.NCj, c.NCi, c.NCi};
  for (int e = 0; e < 4; ++e) {
    const std::vector<double>& w = *Wo_src[e];
    const int L = Wo_len[e];
    for (int k = 0; k < L; ++k) Wo_dst[e][k] = Euler2D_pState(w[k], w[L + k], w[2 * L + k], w[3 * L + k]);
  }
  B.Freeze_Limiter = OFF;
  B.Axisymmetric = 0;
}

void set_grid(const Case& c, const BlockData& d, Grid2D_Quad_Block_HO& G) {
  for (int j = 0; j < c.NNj; ++j)
    for (int i = 0; i < c.NNi; ++i) {
      G.Node[i][j].X.x = d.X[j * c.NNi + i];
      G.Node[i][j].X.y = d.Y[j * c.NNi + i];
    }
  for (int j = 0; j < c.NCj; ++j) { G.BCtypeW[j] = d.bcw[j]; G.BCtypeE[j] = d.bce[j]; }
  for (int i = 0; i < c.NCi; ++i) { G.BCtypeS[i] = d.bcs[i]; G.BCtypeN[i] = d.bcn[i]; }
  G.Schedule_Interior_Mesh_Update();
  G.Schedule_Ghost_Cells_Update();
  G.Update_Cells();
}

// GMRES_Block_Preconditioner and GMRES_ILUK_Level_of_Fill as the deck
// keywords set them (NKSInput2D.h:523-536).
void set_block_preconditioner(NKS_Input_Parameters& N, const char* kind, const char* level) {
  N.GMRES_Block_Preconditioner = strcmp(kind, "Diagonal") ? Block_ILUK : Block_Jacobi;
  N.GMRES_ILUK_Level_of_Fill = atoi(level);
}

// The reference's own multi-block set-up.  order[b] = solution block index
// of case block b.
struct RefSet {
  Euler2D_Input_Parameters IP;
  QuadTreeBlock_DataStructure QuadTree;
  AdaptiveBlockResourceList Global;
  AdaptiveBlock2D_List Local;
  Euler2D_Quad_Block* Soln;
  std::vector<int> order;
  bool first_step = true;
};

void build_reference_blocks(const Case& c, RefSet& R) {
  set_input(c, R.IP);
  Grid2D_Quad_Block_HO** M = new Grid2D_Quad_Block_HO*[c.nbi];
  for (int bi = 0; bi < c.nbi; ++bi) M[bi] = new Grid2D_Quad_Block_HO[c.nbj];
  for (int bj = 0; bj < c.nbj; ++bj)
    for (int bi = 0; bi < c.nbi; ++bi) {
      M[bi][bj].allocate(c.nci, c.ncj, c.ng);
      set_grid(c, c.data[bj * c.nbi + bi], M[bi][bj]);
    }
  R.Soln = NULL;
  R.Soln = Create_Initial_Solution_Blocks(M, R.Soln, R.IP, R.QuadTree, R.Global, R.Local);
  if (!R.Soln) { fprintf(stderr, "Create_Initial_Solution_Blocks failed\n"); exit(3); }
  R.order.resize(c.nblk);
  for (int bj = 0; bj < c.nbj; ++bj)
    for (int bi = 0; bi < c.nbi; ++bi) {
      const int n = R.QuadTree.Roots[bi][bj].block.info.blknum;
      R.order[bj * c.nbi + bi] = n;
      load_state(c, c.data[bj * c.nbi + bi], R.Soln[n]);
    }
}

void dump_p(FILE* f, Euler2D_Quad_Block& B, Euler2D_pState** A) {
  std::vector<double> o(4 * B.NCi * B.NCj);
  const int s = B.NCi * B.NCj;
  for (int j = 0; j < B.NCj; ++j)
    for (int i = 0; i < B.NCi; ++i)
      for (int v = 0; v < 4; ++v) o[v * s + j * B.NCi + i] = A[i][j][v + 1];
  wr(f, &o[0], o.size());
}

void dump_c(FILE* f, Euler2D_Quad_Block& B, int which) {
  std::vector<double> o(4 * B.NCi * B.NCj);
  const int s = B.NCi * B.NCj;
  for (int j = 0; j < B.NCj; ++j)
    for (int i = 0; i < B.NCi; ++i)
      for (int v = 0; v < 4; ++v) {
        double x = which < 0 ? B.U[i][j][v + 1] : B.dUdt[i][j][which][v + 1];
        o[v * s + j * B.NCi + i] = x;
      }
  wr(f, &o[0], o.size());
}

double wall_seconds() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct StepLog { double dt, l1, l2, lmax; };

// One explicit multistage step in the order of Euler2DQuadSolvers.cc:657-898.
int explicit_step_reference(RefSet& R, StepLog& log) {
  Euler2D_Input_Parameters& IP = R.IP;
  double dTime = CFL(R.Soln, R.Local, IP);
  if (!IP.Local_Time_Stepping) Set_Global_TimeStep(R.Soln, R.Local, dTime);
  double l1 = L1_Norm_Residual(R.Soln, R.Local);
  double l2 = L2_Norm_Residual(R.Soln, R.Local);
  l2 = sqrt(sqr(l2));
  double lmax = Max_Norm_Residual(R.Soln, R.Local);
  log.dt = dTime; log.l1 = l1; log.l2 = l2; log.lmax = lmax;
  // limiter freezing (Euler2DQuadSolvers.cc:794-803)
  if (!R.first_step && IP.Freeze_Limiter && l2 <= IP.Freeze_Limiter_Residual_Level) Freeze_Limiters(R.Soln, R.Local);
  for (int stage = 1; stage <= IP.N_Stage; ++stage) {
    int err = Send_All_Messages(R.Soln, R.Local, NUM_VAR_EULER2D, OFF);
    if (err) return err;
    BCs(R.Soln, R.Local, IP);
    err = dUdt_Multistage_Explicit(R.Soln, R.Global, R.Local, IP, stage);
    if (err) return err;
    err = Send_Conservative_Flux_Corrections(R.Soln, R.Local, NUM_VAR_EULER2D);
    if (err) return err;
    Apply_Boundary_Flux_Corrections_Multistage_Explicit(R.Soln, R.Local, IP, stage);
    if (IP.Residual_Smoothing) Residual_Smoothing(R.Soln, R.Local, IP, stage);
    err = Update_Solution_Multistage_Explicit(R.Soln, R.Local, IP, stage);
    if (err) return err;
  }
  R.first_step = false;
  return 0;
}

// ---- threaded timing mode (per-block reference routines, restated exchange)
struct TimedSet {
  const Case* c;
  Euler2D_Input_Parameters IP;
  std::vector<Euler2D_Quad_Block*> blk;
};
int n_threads = 1;

void exchange_restated(TimedSet& T) {
  const Case& c = *T.c;
  const int g = c.ng;
  for (int b = 0; b < c.nblk; ++b) {
    Euler2D_Quad_Block& B = *T.blk[b];
    const int* nb = c.data[b].neigh;
    const int ICl = B.ICl, ICu = B.ICu, JCl = B.JCl, JCu = B.JCu;
    for (int k = 0; k < 8; ++k) {
      if (nb[k] < 0) continue;
      Euler2D_Quad_Block& S = *T.blk[nb[k]];
      int i0, i1, j0, j1, di, dj;
      const int wi = (k == 0 || k == 4 || k == 6), ei = (k == 1 || k == 5 || k == 7);
      const int sj = (k == 2 || k == 4 || k == 5), nj = (k == 3 || k == 6 || k == 7);
      if (wi) { i0 = ICl - g; i1 = ICl - 1; di = (S.ICu + 1) - ICl; }
      else if (ei) { i0 = ICu + 1; i1 = ICu + g; di = S.ICl - (ICu + 1); }
      else { i0 = ICl; i1 = ICu; di = 0; }
      if (sj) { j0 = JCl - g; j1 = JCl - 1; dj = (S.JCu + 1) - JCl; }
      else if (nj) { j0 = JCu + 1; j1 = JCu + g; dj = S.JCl - (JCu + 1); }
      else { j0 = JCl; j1 = JCu; dj = 0; }
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
          B.U[i][j] = S.U[i + di][j + dj];
          B.W[i][j] = B.U[i][j].W();
        }
    }
  }
}

struct ParJob { TimedSet* T; void (*fn)(TimedSet&, int, void*); void* arg; int t, nt; };
void* par_worker(void* p) {
  ParJob* j = (ParJob*)p;
  for (int b = j->t; b < j->T->c->nblk; b += j->nt) j->fn(*j->T, b, j->arg);
  return 0;
}
void parallel_blocks(TimedSet& T, void (*fn)(TimedSet&, int, void*), void* arg) {
  const int nt = n_threads < T.c->nblk ? n_threads : T.c->nblk;
  std::vector<pthread_t> th(nt);
  std::vector<ParJob> jobs(nt);
  for (int t = 0; t < nt; ++t) {
    ParJob j = {&T, fn, arg, t, nt};
    jobs[t] = j;
    if (t > 0) pthread_create(&th[t], 0, par_worker, &jobs[t]);
  }
  par_worker(&jobs[0]);
  for (int t = 1; t < nt; ++t) pthread_join(th[t], 0);
}
struct CflArg { double* dt; };
void cfl_block(TimedSet& T, int b, void* a) { ((CflArg*)a)->dt[b] = CFL(*T.blk[b], T.IP); }
struct StageArg { int stage; int* err; };
void stage_block(TimedSet& T, int b, void* a) {
  StageArg* x = (StageArg*)a;
  BCs(*T.blk[b], T.IP);
  int e = dUdt_Multistage_Explicit(*T.blk[b], x->stage, T.IP);
  if (!e) e = Update_Solution_Multistage_Explicit(*T.blk[b], x->stage, T.IP) ? 1 : 0;
  x->err[b] = e;
}

int explicit_step_threaded(TimedSet& T) {
  const int nb = T.c->nblk;
  std::vector<double> dtb(nb);
  CflArg ca = {&dtb[0]};
  parallel_blocks(T, cfl_block, &ca);
  double dtmin = MILLION;
  for (int b = 0; b < nb; ++b) dtmin = min(dtmin, dtb[b]);
  if (!T.IP.Local_Time_Stepping)
    for (int b = 0; b < nb; ++b) Set_Global_TimeStep(*T.blk[b], dtmin);
  std::vector<int> errb(nb, 0);
  for (int stage = 1; stage <= T.IP.N_Stage; ++stage) {
    exchange_restated(T);
    StageArg sa = {stage, &errb[0]};
    parallel_blocks(T, stage_block, &sa);
    for (int b = 0; b < nb; ++b)
      if (errb[b]) return errb[b];
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 3 && !strcmp(argv[1], "solve")) {
    // the reference's own deck-driven solver, as its command line runs it
    // (Euler2DQuadSolver, Euler2DQuadSolvers.cc:26), in batch mode, after
    // the process set-up of its main (one processor, Euler2D.cc)
    CFFC_Initialize_MPI(argc, argv);
    return Euler2DQuadSolver(argv[2], 1);
  }
  if (argc < 4) {
    fprintf(stderr, "usage: %s residual|explicit|nks|time CASE ... | solve DECK\n", argv[0]);
    return 2;
  }
  Case c;
  read_case(argv[2], c);
  const char* mode = argv[1];

  if (!strcmp(mode, "residual")) {
    RefSet R;
    build_reference_blocks(c, R);
    Send_All_Messages(R.Soln, R.Local, NUM_VAR_EULER2D, OFF);
    BCs(R.Soln, R.Local, R.IP);
    for (int b = 0; b < c.nblk; ++b) dUdt_Residual_Evaluation(R.Soln[R.order[b]], R.IP);
    FILE* f = fopen(argv[3], "wb");
    for (int b = 0; b < c.nblk; ++b) {
      Euler2D_Quad_Block& B = R.Soln[R.order[b]];
      dump_p(f, B, B.W);
      dump_c(f, B, 0);
      dump_p(f, B, B.dWdx);
      dump_p(f, B, B.dWdy);
      dump_p(f, B, B.phi);
    }
    fclose(f);
    return 0;
  }

  if (!strcmp(mode, "explicit")) {
    const int nsteps = atoi(argv[3]);
    RefSet R;
    build_reference_blocks(c, R);
    Send_All_Messages(R.Soln, R.Local, NUM_VAR_EULER2D, OFF);
    BCs(R.Soln, R.Local, R.IP);
    std::vector<StepLog> hist(nsteps);
    int err = 0, n = 0;
    for (; n < nsteps && !err; ++n) err = explicit_step_reference(R, hist[n]);
    if (err) fprintf(stderr, "explicit step %d failed (error %d)\n", n, err);
    FILE* f = fopen(argv[4], "wb");
    int hdr[2] = {n, err};
    wr(f, hdr, 2);
    for (int k = 0; k < n; ++k) wr(f, &hist[k].dt, 4);
    for (int b = 0; b < c.nblk; ++b) {
      dump_c(f, R.Soln[R.order[b]], -1);
      dump_c(f, R.Soln[R.order[b]], 0);
    }
    fclose(f);
    return err ? 1 : 0;
  }

  if (!strcmp(mode, "precon")) {
    // The Newton step's preconditioner alone: dt as the Newton loop sets it
    // (NKS2D.h:913-930), then per block Create_Preconditioner,
    // Update_Jacobian_and_Preconditioner and Apply_Preconditioner
    // (Block_Preconditioner2D.h:261, 352, 787) on the vectors of VFILE
    // ([nblk][NCj][NCi][4] doubles, GMRES_Block::index order); OUT gets z.
    if (argc < 8) { fprintf(stderr, "precon CASE OUT CFL ILUK|Diagonal LEVEL VFILE\n"); return 2; }
    RefSet R;
    build_reference_blocks(c, R);
    set_block_preconditioner(R.IP.NKS_IP, argv[5], argv[6]);
    Send_All_Messages(R.Soln, R.Local, NUM_VAR_EULER2D, OFF);
    BCs(R.Soln, R.Local, R.IP);
    const double cfl = atof(argv[4]);
    double dTime = CFL(R.Soln, R.Local, R.IP);
    if (R.IP.Local_Time_Stepping == GLOBAL_TIME_STEPPING) {
      Set_Global_TimeStep(R.Soln, R.Local, dTime * cfl);
    } else {
      for (int b = 0; b < c.nblk; ++b) {
        Euler2D_Quad_Block& B = R.Soln[R.order[b]];
        for (int i = 0; i < B.NCi; ++i)
          for (int j = 0; j < B.NCj; ++j) B.dt[i][j] *= cfl;
      }
    }
    const int n = 4 * (c.nci + 2 * c.ng) * (c.ncj + 2 * c.ng);
    std::vector<double> v(size_t(n) * c.nblk), z(size_t(n) * c.nblk, 0.0);
    FILE* fv = fopen(argv[7], "rb");
    if (!fv || fread(v.data(), sizeof(double), v.size(), fv) != v.size()) { fprintf(stderr, "bad VFILE\n"); return 2; }
    fclose(fv);
    for (int b = 0; b < c.nblk; ++b) {
      Block_Preconditioner<Euler2D_pState, Euler2D_Quad_Block, Euler2D_Input_Parameters> P;
      P.Create_Preconditioner(R.Soln[R.order[b]], R.IP, NUM_VAR_EULER2D);
      P.Update_Jacobian_and_Preconditioner(0.0);
      P.Apply_Preconditioner(n, 1, &v[size_t(b) * n], n, &z[size_t(b) * n], n);
    }
    FILE* f = fopen(argv[3], "wb");
    wr(f, z.data(), z.size());
    fclose(f);
    return 0;
  }

  if (!strcmp(mode, "nks")) {
    if (argc < 9) { fprintf(stderr, "nks CASE OUT MAX_NEWTON RESTART MAX_GMRES CFL0 TOL\n"); return 2; }
    RefSet R;
    build_reference_blocks(c, R);
    NKS_Input_Parameters& N = R.IP.NKS_IP;
    N.Maximum_Number_of_NKS_Iterations = atoi(argv[4]);
    N.GMRES_Restart = atoi(argv[5]);
    N.Maximum_Number_of_GMRES_Iterations = atoi(argv[6]);
    N.Finite_Time_Step_Initial_CFL = atof(argv[7]);
    N.Overall_Tolerance = atof(argv[8]);
    if (argc > 9) N.GMRES_Initial_Tolerance = N.GMRES_Final_Tolerance = atof(argv[9]);
    if (argc > 11) set_block_preconditioner(N, argv[10], argv[11]);
    Send_All_Messages(R.Soln, R.Local, NUM_VAR_EULER2D, OFF);
    BCs(R.Soln, R.Local, R.IP);
    std::string hist_path = std::string(argv[3]) + ".hist";
    std::ofstream hist(hist_path.c_str());
    CPUTime cpu;
    int nexp = 0;
    double ptime = 0.0;
    const double t0 = wall_seconds();
    int err = Newton_Krylov_Schwarz_Solver<Euler2D_pState, Euler2D_Quad_Block, Euler2D_Input_Parameters>(
        cpu, hist, nexp, ptime, R.Soln, R.QuadTree, R.Global, R.Local, R.IP);
    const double t1 = wall_seconds();
    hist.close();
    fprintf(stderr, "nks: error %d, %.3f s\n", err, t1 - t0);
    FILE* f = fopen(argv[3], "wb");
    int hdr[2] = {err, 0};
    wr(f, hdr, 2);
    const double secs = t1 - t0;
    wr(f, &secs, 1);
    for (int b = 0; b < c.nblk; ++b) dump_c(f, R.Soln[R.order[b]], -1);
    fclose(f);
    return err ? 1 : 0;
  }

  if (!strcmp(mode, "restart_write")) {
    // Write_Restart_Solution + Write_QuadTree (Euler2DQuadMultiBlock.cc:218,
    // AMR/AMR.h:296) of the case's block set, PREFIX_blkNNNNNN.soln and
    // PREFIX_quadtree.tree, with time step count NSTEPS and time TIME.
    if (argc < 6) { fprintf(stderr, "restart_write CASE PREFIX NSTEPS TIME\n"); return 2; }
    RefSet R;
    build_reference_blocks(c, R);
    snprintf(R.IP.Restart_File_Name, sizeof(R.IP.Restart_File_Name), "%s.soln", argv[3]);
    CPUTime cpu;
    cpu.cput = 1.5;
    int err = Write_Restart_Solution(R.Soln, R.Local, R.IP, atoi(argv[4]), atof(argv[5]), cpu);
    err = err || Write_QuadTree(R.QuadTree, R.IP);
    return err ? 1 : 0;
  }

  if (!strcmp(mode, "grid_write")) {
    // the grid data file of the case's blocks in the layout of
    // Write_Multi_Block_Grid_Using_IP (Grid/HO_Grid2DQuadMultiBlock.h:3160):
    // grid type line, i_Grid, "nbi nbj", Write_Quad_Block of every block
    std::ofstream out(argv[3]);
    out << (c.periodic ? "Periodic_Box" : "Rectangular_Box") << "\n"
        << (c.periodic ? GRID_PERIODIC_BOX : GRID_RECTANGULAR_BOX) << "\n";
    out << c.nbi << " " << c.nbj << "\n";
    for (int bj = 0; bj < c.nbj; ++bj)
      for (int bi = 0; bi < c.nbi; ++bi) {
        Grid2D_Quad_Block_HO G;
        G.allocate(c.nci, c.ncj, c.ng);
        set_grid(c, c.data[bj * c.nbi + bi], G);
        G.Write_Quad_Block(out);
      }
    return out.good() ? 0 : 1;
  }

  if (!strcmp(mode, "restart_read")) {
    // Read_QuadTree + Read_Restart_Solution (AMR/AMR.h:169,
    // Euler2DQuadMultiBlock.cc:145) of PREFIX; the case file gives the grid
    // type (periodic wiring) and the block count.  OUT: int32 nsteps, int32
    // nblk, f64 time, f64 cpu time, then per root block (j outer, i inner):
    // int32 gblknum, nW, nE, nS, nN and the local numbers of the first
    // neighbour on each side (-1: none), int32 BCtypeW/E/S/N, f64 nodes X, Y,
    // f64 WoW/E/S/N [4][n], f64 U [4][NCj][NCi].
    if (argc < 5) { fprintf(stderr, "restart_read CASE PREFIX OUT\n"); return 2; }
    Euler2D_Input_Parameters IP;
    set_input(c, IP);
    snprintf(IP.Restart_File_Name, sizeof(IP.Restart_File_Name), "%s.soln", argv[3]);
    QuadTreeBlock_DataStructure QT;
    AdaptiveBlockResourceList Global;
    AdaptiveBlock2D_List Local;
    Euler2D_Quad_Block* Soln = new Euler2D_Quad_Block[c.nblk];
    int nsteps = 0;
    double time = 0.0;
    CPUTime cpu;
    if (Read_QuadTree(QT, Global, Local, IP)) { fprintf(stderr, "Read_QuadTree failed\n"); return 1; }
    if (Read_Restart_Solution(Soln, Local, IP, nsteps, time, cpu)) { fprintf(stderr, "Read_Restart_Solution failed\n"); return 1; }
    if (argc > 5) {
      // restart_read CASE PREFIX OUT GRIDFILE: also the blocks' grids as a
      // grid data file of type Bump_Channel_Flow (Write_Quad_Block per root)
      std::ofstream g(argv[5]);
      g << "Bump_Channel_Flow\n" << GRID_BUMP_CHANNEL_FLOW << "\n" << QT.NRi << " " << QT.NRj << "\n";
      for (int bj = 0; bj < QT.NRj; ++bj)
        for (int bi = 0; bi < QT.NRi; ++bi) Soln[QT.Roots[bi][bj].block.info.blknum].Grid.Write_Quad_Block(g);
    }
    FILE* f = fopen(argv[4], "wb");
    int hdr[2] = {nsteps, c.nblk};
    wr(f, hdr, 2);
    wr(f, &time, 1);
    wr(f, &cpu.cput, 1);
    for (int bj = 0; bj < QT.NRj; ++bj)
      for (int bi = 0; bi < QT.NRi; ++bi) {
        const int n = QT.Roots[bi][bj].block.info.blknum;
        const AdaptiveBlock2D& A = Local.Block[n];
        Euler2D_Quad_Block& B = Soln[n];
        int nb[9] = {A.gblknum, A.nW, A.nE, A.nS, A.nN,
                     A.nW ? A.infoW[0].blknum : -1, A.nE ? A.infoE[0].blknum : -1,
                     A.nS ? A.infoS[0].blknum : -1, A.nN ? A.infoN[0].blknum : -1};
        wr(f, nb, 9);
        std::vector<int> bc;
        for (int j = 0; j < B.NCj; ++j) bc.push_back(B.Grid.BCtypeW[j]);
        for (int j = 0; j < B.NCj; ++j) bc.push_back(B.Grid.BCtypeE[j]);
        for (int i = 0; i < B.NCi; ++i) bc.push_back(B.Grid.BCtypeS[i]);
        for (int i = 0; i < B.NCi; ++i) bc.push_back(B.Grid.BCtypeN[i]);
        wr(f, &bc[0], bc.size());
        std::vector<double> xy;
        for (int j = 0; j < B.NCj + 1; ++j)
          for (int i = 0; i < B.NCi + 1; ++i) xy.push_back(B.Grid.Node[i][j].X.x);
        for (int j = 0; j < B.NCj + 1; ++j)
          for (int i = 0; i < B.NCi + 1; ++i) xy.push_back(B.Grid.Node[i][j].X.y);
        wr(f, &xy[0], xy.size());
        Euler2D_pState* Wo[4] = {B.WoW, B.WoE, B.WoS, B.WoN};
        const int L[4] = {B.NCj, B.NCj, B.NCi, B.NCi};
        for (int e = 0; e < 4; ++e) {
          std::vector<double> w(4 * L[e]);
          for (int k = 0; k < L[e]; ++k)
            for (int v = 0; v < 4; ++v) w[v * L[e] + k] = Wo[e][k][v + 1];
          wr(f, &w[0], w.size());
        }
        dump_c(f, B, -1);
      }
    fclose(f);
    return 0;
  }

  if (!strcmp(mode, "time")) {
    const int nsteps = atoi(argv[3]);
    n_threads = argc > 4 ? atoi(argv[4]) : 1;
    if (n_threads < 1) n_threads = 1;
    TimedSet T;
    T.c = &c;
    set_input(c, T.IP);
    T.blk.resize(c.nblk);
    for (int b = 0; b < c.nblk; ++b) {
      T.blk[b] = new Euler2D_Quad_Block;
      T.blk[b]->allocate(c.nci, c.ncj, c.ng);
      set_grid(c, c.data[b], T.blk[b]->Grid);
      load_state(c, c.data[b], *T.blk[b]);
    }
    exchange_restated(T);
    for (int b = 0; b < c.nblk; ++b) BCs(*T.blk[b], T.IP);
    const double t0 = wall_seconds();
    int err = 0, n = 0;
    for (; n < nsteps && !err; ++n) err = explicit_step_threaded(T);
    const double s = wall_seconds() - t0;
    const double cells = double(c.nblk) * c.nci * c.ncj;
    printf("{\"seconds\": %.6f, \"steps\": %d, \"cells\": %.0f, \"threads\": %d, "
           "\"mcell_updates_per_s\": %.6f, \"error\": %d}\n",
           s, n, cells, n_threads, cells * n / s * 1e-6, err);
    return err ? 1 : 0;
  }
  fprintf(stderr, "unknown mode %s\n", mode);
  return 2;
}

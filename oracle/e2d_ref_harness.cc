// e2d_ref_harness: drives the compiled CFFC reference (oracle/_ref/libcffc_ref.a)
// on a block set described by an e2d case file, and writes what the
// reference computes.  Test infrastructure only: it generates golden vectors,
// pins the C restatement (oracle/e2d_oracle.c) and times the reference's CPU
// path.  The product never links or runs it.
//
// Every numerical step is the reference's own per-block routine:
//   BCs                                src_2D/Euler2D/Euler2DQuadSingleBlock.cc:2354
//   dUdt_Residual_Evaluation           src_2D/Euler2D/Euler2DQuadSingleBlock.cc:5095
//                                      -> Euler2DQuad.cc:814
//   dUdt_Multistage_Explicit           Euler2DQuadSingleBlock.cc:5117 -> Euler2DQuad.cc:1235
//   Update_Solution_Multistage_Explicit Euler2DQuadSingleBlock.cc:5300
//   CFL / Set_Global_TimeStep          Euler2DQuadSingleBlock.cc:3019, :3089
//   L1/L2/Max_Norm_Residual            Euler2DQuadSingleBlock.cc:3111-3167
//   Grid2D_Quad_Block_HO::Update_Cells src_2D/Grid/HO_Grid2DQuad.cc:9832
// The one step restated here is the same-resolution ghost exchange between
// blocks, a plain copy of the neighbours' two edge layers of U followed by
// W = U.W(), as Euler2D_Quad_Block::LoadSendBuffer / UnloadReceiveBuffer do
// (src_2D/Euler2D/Euler2DQuad.h:1570-1650) for Send_All_Messages
// (src_2D/AMR/AdaptiveBlock2D_MessagePassing.h:7883).
//
// usage:
//   e2d_ref_harness residual CASE OUT
//   e2d_ref_harness explicit CASE NSTEPS OUT [threads]
//   e2d_ref_harness time     CASE NSTEPS THREADS      (prints one JSON line)
//
// Case file (little endian), shared with cffc_b200/case_io.py:
//   int32 magic 0x43443245, version 1
//   int32 nblk, nci, ncj, ng
//   int32 limiter, flux, n_stage, local_dt, time_accurate, 0, 0, 0
//   f64   cfl, 0, 0, 0
//   per block:
//     int32 neighbour[8]           W, E, S, N, SW, SE, NW, NE (-1 = none)
//     int32 bcW[NCj], bcE[NCj], bcS[NCi], bcN[NCi]      reference BC codes
//     f64   X[NNj][NNi], Y[NNj][NNi]                    nodes incl. ghosts
//     f64   WoW[4][NCj], WoE[4][NCj], WoS[4][NCi], WoN[4][NCi]
//     f64   W[4][NCj][NCi]                              (rho, u, v, p)
// with NCi = nci + 2 ng, NNi = NCi + 1 (likewise j).  Arrays are [var][j][i].
#include <time.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <pthread.h>

#include "Euler2D/Euler2DQuad.h"
#include "Euler2D/Euler2DInput.h"

namespace {

struct Case {
  int nblk, nci, ncj, ng;
  int limiter, flux, n_stage, local_dt, time_accurate;
  double cfl;
  std::vector<int> neigh;  // nblk * 8
  std::vector<Euler2D_Quad_Block*> blk;  // the reference block has no public copy
};

template <class T> void rd(FILE* f, T* p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}
template <class T> void wr(FILE* f, const T* p, size_t n) { fwrite(p, sizeof(T), n, f); }

void set_input(const Case& c, Euler2D_Input_Parameters& IP) {
  Set_Default_Input_Parameters(IP);
  IP.i_Reconstruction = RECONSTRUCTION_LEAST_SQUARES;
  IP.i_Limiter = c.limiter;
  IP.i_Flux_Function = c.flux;
  IP.i_Time_Integration = TIME_STEPPING_EXPLICIT_RUNGE_KUTTA;
  IP.N_Stage = c.n_stage;
  IP.CFL_Number = c.cfl;
  IP.Local_Time_Stepping = c.local_dt ? SCALAR_LOCAL_TIME_STEPPING : GLOBAL_TIME_STEPPING;
  IP.Time_Accurate = c.time_accurate;
  IP.Axisymmetric = 0;
  IP.Number_of_Ghost_Cells = c.ng;
}

void read_case(const char* path, Case& c) {
  FILE* f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  int hdr[2], dims[4], opts[8];
  double dopts[4];
  rd(f, hdr, 2);
  if (hdr[0] != 0x43443245 || hdr[1] != 1) { fprintf(stderr, "bad case file\n"); exit(2); }
  rd(f, dims, 4); rd(f, opts, 8); rd(f, dopts, 4);
  c.nblk = dims[0]; c.nci = dims[1]; c.ncj = dims[2]; c.ng = dims[3];
  c.limiter = opts[0]; c.flux = opts[1]; c.n_stage = opts[2];
  c.local_dt = opts[3]; c.time_accurate = opts[4]; c.cfl = dopts[0];
  c.neigh.resize(8 * c.nblk);
  c.blk.resize(c.nblk);
  for (int b = 0; b < c.nblk; ++b) c.blk[b] = new Euler2D_Quad_Block;
  const int NCi = c.nci + 2 * c.ng, NCj = c.ncj + 2 * c.ng;
  const int NNi = NCi + 1, NNj = NCj + 1;
  std::vector<double> X(NNi * NNj), Y(NNi * NNj), Wo(4 * (NCi > NCj ? NCi : NCj));
  std::vector<double> W(4 * NCi * NCj);
  for (int b = 0; b < c.nblk; ++b) {
    Euler2D_Quad_Block& B = *c.blk[b];
    B.allocate(c.nci, c.ncj, c.ng);
    rd(f, &c.neigh[8 * b], 8);
    rd(f, B.Grid.BCtypeW, NCj); rd(f, B.Grid.BCtypeE, NCj);
    rd(f, B.Grid.BCtypeS, NCi); rd(f, B.Grid.BCtypeN, NCi);
    rd(f, &X[0], X.size()); rd(f, &Y[0], Y.size());
    for (int j = 0; j < NNj; ++j)
      for (int i = 0; i < NNi; ++i) {
        B.Grid.Node[i][j].X.x = X[j * NNi + i];
        B.Grid.Node[i][j].X.y = Y[j * NNi + i];
      }
    B.Grid.Schedule_Interior_Mesh_Update();
    B.Grid.Schedule_Ghost_Cells_Update();
    B.Grid.Update_Cells();
    Euler2D_pState* Wo_dst[4] = {B.WoW, B.WoE, B.WoS, B.WoN};
    const int Wo_len[4] = {NCj, NCj, NCi, NCi};
    for (int e = 0; e < 4; ++e) {
      rd(f, &Wo[0], 4 * Wo_len[e]);
      for (int k = 0; k < Wo_len[e]; ++k)
        Wo_dst[e][k] = Euler2D_pState(Wo[k], Wo[Wo_len[e] + k], Wo[2 * Wo_len[e] + k],
                                      Wo[3 * Wo_len[e] + k]);
    }
    rd(f, &W[0], W.size());
    for (int j = 0; j < NCj; ++j)
      for (int i = 0; i < NCi; ++i) {
        const int q = j * NCi + i, s = NCi * NCj;
        B.W[i][j] = Euler2D_pState(W[q], W[s + q], W[2 * s + q], W[3 * s + q]);
        B.U[i][j] = U(B.W[i][j]);
      }
    B.Freeze_Limiter = OFF;
    B.Axisymmetric = 0;
  }
  fclose(f);
}

// Same-resolution ghost exchange (see the header comment).
void exchange(Case& c) {
  const int g = c.ng;
  for (int b = 0; b < c.nblk; ++b) {
    Euler2D_Quad_Block& B = *c.blk[b];
    const int* nb = &c.neigh[8 * b];
    const int ICl = B.ICl, ICu = B.ICu, JCl = B.JCl, JCu = B.JCu;
    for (int k = 0; k < 8; ++k) {
      if (nb[k] < 0) continue;
      Euler2D_Quad_Block& S = *c.blk[nb[k]];
      // ghost index range in this block and the source offset in S
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

void fill_ghosts(Case& c, Euler2D_Input_Parameters& IP) {
  exchange(c);
  for (int b = 0; b < c.nblk; ++b) BCs(*c.blk[b], IP);
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

// Runs fn(block) for every block on n_threads POSIX threads (blocks are
// independent once their ghosts are filled; the reference runs them on
// separate MPI ranks the same way).
int n_threads = 1;
struct ParJob { Case* c; void (*fn)(Case&, int, void*); void* arg; int t, nt; };
void* par_worker(void* p) {
  ParJob* j = (ParJob*)p;
  for (int b = j->t; b < j->c->nblk; b += j->nt) j->fn(*j->c, b, j->arg);
  return 0;
}
void parallel_blocks(Case& c, void (*fn)(Case&, int, void*), void* arg) {
  const int nt = n_threads < c.nblk ? n_threads : c.nblk;
  std::vector<pthread_t> th(nt);
  std::vector<ParJob> jobs(nt);
  for (int t = 0; t < nt; ++t) {
    ParJob j = {&c, fn, arg, t, nt};
    jobs[t] = j;
    if (t > 0) pthread_create(&th[t], 0, par_worker, &jobs[t]);
  }
  par_worker(&jobs[0]);
  for (int t = 1; t < nt; ++t) pthread_join(th[t], 0);
}

struct StepLog { double dt, l1, l2, lmax; };

struct CflArg { Euler2D_Input_Parameters* IP; double* dt; };
void cfl_block(Case& c, int b, void* a) {
  CflArg* x = (CflArg*)a;
  x->dt[b] = CFL(*c.blk[b], *x->IP);
}
struct StageArg { Euler2D_Input_Parameters* IP; int stage; int* err; };
void stage_block(Case& c, int b, void* a) {
  StageArg* x = (StageArg*)a;
  BCs(*c.blk[b], *x->IP);
  int e = dUdt_Multistage_Explicit(*c.blk[b], x->stage, *x->IP);
  if (!e) e = Update_Solution_Multistage_Explicit(*c.blk[b], x->stage, *x->IP) ? 1 : 0;
  x->err[b] = e;
}

// One explicit multistage time step in the order of the reference's solver
// loop (src_2D/Euler2D/Euler2DQuadSolvers.cc:657-898).
int explicit_step(Case& c, Euler2D_Input_Parameters& IP, StepLog& log) {
  const int nb = c.nblk;
  double dtmin = MILLION;
  std::vector<double> dtb(nb);
  CflArg ca = {&IP, &dtb[0]};
  parallel_blocks(c, cfl_block, &ca);
  for (int b = 0; b < nb; ++b) dtmin = min(dtmin, dtb[b]);
  if (!IP.Local_Time_Stepping)
    for (int b = 0; b < nb; ++b) Set_Global_TimeStep(*c.blk[b], dtmin);
  double l1 = 0, l2 = 0, lmax = 0;
  for (int b = 0; b < nb; ++b) {
    l1 += L1_Norm_Residual(*c.blk[b], 1);
    l2 += sqr(L2_Norm_Residual(*c.blk[b], 1));
    lmax = max(lmax, Max_Norm_Residual(*c.blk[b], 1));
  }
  // multi-block L2 (Euler2DQuadMultiBlock.cc:1049) is squared, summed over
  // ranks and rooted again by the solver loop (Euler2DQuadSolvers.cc:690-693)
  log.dt = dtmin; log.l1 = l1; log.l2 = sqrt(sqr(sqrt(l2))); log.lmax = lmax;
  std::vector<int> errb(nb, 0);
  for (int stage = 1; stage <= IP.N_Stage; ++stage) {
    exchange(c);
    StageArg sa = {&IP, stage, &errb[0]};
    parallel_blocks(c, stage_block, &sa);
    for (int b = 0; b < nb; ++b)
      if (errb[b]) return errb[b];
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s residual|explicit|time CASE ...\n", argv[0]);
    return 2;
  }
  Case c;
  read_case(argv[2], c);
  Euler2D_Input_Parameters IP;
  set_input(c, IP);
  const char* mode = argv[1];

  if (!strcmp(mode, "residual")) {
    fill_ghosts(c, IP);
    for (int b = 0; b < c.nblk; ++b) dUdt_Residual_Evaluation(*c.blk[b], IP);
    FILE* f = fopen(argv[3], "wb");
    for (int b = 0; b < c.nblk; ++b) {
      Euler2D_Quad_Block& B = *c.blk[b];
      dump_p(f, B, B.W);
      dump_c(f, B, 0);
      dump_p(f, B, B.dWdx);
      dump_p(f, B, B.dWdy);
      dump_p(f, B, B.phi);
    }
    fclose(f);
    return 0;
  }

  if (!strcmp(mode, "explicit") || !strcmp(mode, "time")) {
    const int nsteps = atoi(argv[3]);
    const int timing = !strcmp(mode, "time");
    int threads = 1;
    if (timing && argc > 4) threads = atoi(argv[4]);
    if (!timing && argc > 5) threads = atoi(argv[5]);
    if (threads < 1) threads = 1;
    n_threads = threads;
    fill_ghosts(c, IP);
    std::vector<StepLog> hist(nsteps);
    const double t0 = wall_seconds();
    int err = 0, n = 0;
    for (; n < nsteps && !err; ++n) err = explicit_step(c, IP, hist[n]);
    const double t1 = wall_seconds();
    if (err) fprintf(stderr, "explicit step %d failed (error %d)\n", n, err);
    if (timing) {
      const double s = t1 - t0;
      const double cells = double(c.nblk) * c.nci * c.ncj;
      printf("{\"seconds\": %.6f, \"steps\": %d, \"cells\": %.0f, \"threads\": %d, "
             "\"mcell_updates_per_s\": %.6f, \"error\": %d}\n",
             s, n, cells, threads, cells * n / s * 1e-6, err);
      return err ? 1 : 0;
    }
    FILE* f = fopen(argv[4], "wb");
    int hdr[2] = {n, err};
    wr(f, hdr, 2);
    for (int k = 0; k < n; ++k) wr(f, &hist[k].dt, 4);
    for (int b = 0; b < c.nblk; ++b) {
      dump_c(f, *c.blk[b], -1);
      dump_c(f, *c.blk[b], 0);
    }
    fclose(f);
    return err ? 1 : 0;
  }
  fprintf(stderr, "unknown mode %s\n", mode);
  return 2;
}

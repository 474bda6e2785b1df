/*
 * cffc_e2d.h — C ABI of the B200 Euler2D finite-volume library
 * (libcffc_e2d.so, built from cffc_b200/csrc).
 *
 * This is the boundary a caller of the CFFC reference's Euler2D path binds
 * (cgo / ctypes / JNI / a C++ host layer): plain pointers and sizes, no
 * framework types.  Each entry point names the reference interface it
 * replaces (paths relative to the CFFC source tree).
 *
 * Data layout (host arrays passed in or out, and the device arrays behind a
 * handle): one record per block, SoA per variable, rows of i:
 *     cell arrays  [nblk][4][NCj][NCi]   NCi = nci + 2*ng, NCj = ncj + 2*ng
 *     node arrays  [nblk][NNj][NNi]      NNi = NCi + 1,   NNj = NCj + 1
 * Cell (i, j) of a block is the reference's SolnBlk.W[i][j] with the same
 * index origin (ghost cells at i < ICl = ng and i > ICu = ng + nci - 1), and
 * node (i, j) is Grid.Node[i][j].  Primitive variables are (rho, u, v, p),
 * conserved (rho, rho*u, rho*v, E).  All state is FP64 (the reference is
 * FP64); the FP32 reconstruction/flux variant is selected per handle.
 *
 * Conventions mirror the reference's error_flag: 0 = success; a positive
 * return is a reference-style failure (e.g. 1 + the linear index of the first
 * cell whose density or energy went non-positive, where
 * Update_Solution_Multistage_Explicit returns the cell's i index); negative
 * returns are library errors (E2D_ERR_*).  One CUDA stream per handle; a
 * handle is not thread-safe.  The library owns device memory; host buffers
 * belong to the caller.
 */
#ifndef CFFC_E2D_H
#define CFFC_E2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary-condition codes: the reference's values (src_2D/CFD/CFD.h:270-351). */
#define E2D_BC_NONE 0
#define E2D_BC_CONSTANT_EXTRAPOLATION 4001
#define E2D_BC_PERIODIC 6000
#define E2D_BC_REFLECTION 7001
#define E2D_BC_CHARACTERISTIC 8001
#define E2D_BC_FIXED 11000

/* Limiter codes (src_2D/CFD/CFD.h:750-762). */
#define E2D_LIMITER_ONE (-1)
#define E2D_LIMITER_ZERO 0
#define E2D_LIMITER_BARTH_JESPERSEN 8
#define E2D_LIMITER_VENKATAKRISHNAN 9

/* Flux function codes (src_2D/CFD/CFD.h:768-778). */
#define E2D_FLUX_GODUNOV 1  /* exact Riemann solver            */
#define E2D_FLUX_ROE 2      /* Roe with Harten's entropy fix   */
#define E2D_FLUX_RUSANOV 3
#define E2D_FLUX_HLLE 4
#define E2D_FLUX_LINDE 5    /* HLLL                            */
#define E2D_FLUX_HLLC 6
#define E2D_FLUX_VANLEER 8
#define E2D_FLUX_AUSM 9
#define E2D_FLUX_AUSMPLUS 10

/* Precision of reconstruction and flux evaluation. */
#define E2D_PREC_FP64 0       /* FP64, FMA contraction allowed                   */
#define E2D_PREC_FP32 1       /* FP32 reconstruction + flux, FP64 state/update   */
#define E2D_PREC_FP64_EXACT 2 /* FP64 in the reference's rounding order, no FMA:
                                 bit-identical to the reference's x86-64 build  */

/* Library error codes (negative returns). */
#define E2D_ERR_ARG (-1)      /* invalid argument or unsupported option     */
#define E2D_ERR_CUDA (-2)     /* a CUDA call failed                          */
#define E2D_ERR_NOMEM (-3)    /* device allocation failed                    */
#define E2D_ERR_NAN (-4)      /* NaN/Inf detected in a residual norm         */
#define E2D_ERR_GMRES (-5)    /* GMRES breakdown                             */

/* Block-set description: geometry, topology and boundary data of all blocks.
 * Mirrors what Euler2D_Quad_Block / Grid2D_Quad_Block_HO hold for the path
 * (src_2D/Euler2D/Euler2DQuad.h:140-599, src_2D/Grid/HO_Grid2DQuad.h:277-305):
 * nodes including ghost nodes, the per-edge BC type arrays BCtypeW/E/S/N and
 * reference states WoW/E/S/N.  neighbour[b*8 + k] gives the same-resolution
 * neighbour across edge/corner k = W, E, S, N, SW, SE, NW, NE (-1: none);
 * it is the block connectivity the reference keeps in its quadtree
 * (src_2D/AMR/QuadTree.cc:363). */
typedef struct e2d_blocks_desc {
  int32_t nblk, nci, ncj, ng; /* ng must be 2 (Euler2DQuad.h:655 asserts > 1) */
  const int32_t *neighbour;   /* [nblk][8]                                     */
  const int32_t *bc_w, *bc_e; /* [nblk][NCj]                                   */
  const int32_t *bc_s, *bc_n; /* [nblk][NCi]                                   */
  const double *node_x;       /* [nblk][NNj][NNi]                              */
  const double *node_y;       /* [nblk][NNj][NNi]                              */
  const double *wo_w, *wo_e;  /* [nblk][4][NCj] primitive reference states     */
  const double *wo_s, *wo_n;  /* [nblk][4][NCi]                                */
} e2d_blocks_desc;

/* Explicit time-stepping schemes (i_Time_Integration, src_2D/CFD/CFD.h:651-659)
 * and their stage counts:
 *   E2D_TIME_EXPLICIT_EULER / PREDICTOR_CORRECTOR / RUNGE_KUTTA: N_Stage 1, 2
 *     (residuals accumulated over the stages), 4 (classical RK4), 5
 *     (the reference's 5-stage coefficients);
 *   E2D_TIME_OPTIMAL_SMOOTHING: N_Stage 1-6, the optimally smoothing
 *     multistage coefficients of van Leer, Tai and Powell (CFD.cc:953).
 * Code 0 (the structure's zero value) is the Runge-Kutta family. */
#define E2D_TIME_EXPLICIT_EULER 0
#define E2D_TIME_PREDICTOR_CORRECTOR 3
#define E2D_TIME_OPTIMAL_SMOOTHING 7
#define E2D_TIME_RUNGE_KUTTA 8

/* Numerical scheme: the subset of Euler2D_Input_Parameters the path reads
 * (src_2D/Euler2D/Euler2DInput.h:41-120). */
typedef struct e2d_scheme {
  int32_t limiter;   /* i_Limiter                                         */
  int32_t flux;      /* i_Flux_Function: E2D_FLUX_* (all but Osher)       */
  int32_t n_stage;   /* N_Stage (see E2D_TIME_*)                          */
  int32_t local_dt;  /* Local_Time_Stepping: 0 global, 1 scalar local     */
  int32_t precision; /* E2D_PREC_*                                        */
  int32_t time_integration;  /* i_Time_Integration: E2D_TIME_*            */
  int32_t rs_iterations;     /* Residual_Smoothing_Gauss_Seidel_Iterations */
  int32_t freeze_limiter;    /* Freeze_Limiter: 0 off, 1 on               */
  double cfl;        /* CFL_Number                                        */
  double gamma;      /* specific-heat ratio g (GAMMA_AIR = 1.4)           */
  double rs_epsilon; /* Residual_Smoothing_Epsilon (> 0: smoothing on)    */
  double freeze_level;       /* Freeze_Limiter_Residual_Level             */
} e2d_scheme;

typedef struct e2d_handle e2d_handle;

/* Allocates device state for the block set and uploads geometry; computes
 * cell centroids/areas as Grid2D_Quad_Block_HO::Update_Cells does
 * (src_2D/Grid/HO_Grid2DQuad.cc:9832, Math.h:311 quadCentroid).  Replaces
 * Euler2D_Quad_Block::allocate + grid set-up (Euler2DQuad.h:655).
 * Returns NULL on failure with *err set. */
e2d_handle *e2d_create(const e2d_blocks_desc *desc, const e2d_scheme *scheme,
                       int device, int *err);

/* One handle over ncase independent cases (each its own block set, as
 * e2d_create takes it; block counts and block dimensions may differ).
 * Their blocks are laid end to end in case order; every entry point then
 * works on all cases at once, with per-case time-step minima, residual
 * norms, histories and Newton-Krylov solves, and gives each case the same
 * result bit for bit as a handle of that case alone.  Cases of different
 * block dimensions run as one batch per block shape behind this handle; the
 * host arrays (states, residuals, local time steps) are then each case's
 * array in its own shape, concatenated in case order, and
 * e2d_get_reconstruction, e2d_device_state, e2d_kernel_times and
 * e2d_block_precon_apply are not available (E2D_ERR_ARG); e2d_stage_config
 * reports the first shape's kernel.  No reference counterpart: the
 * reference runs one case per process. */
e2d_handle *e2d_create_batch(const e2d_blocks_desc *cases, int ncase, const e2d_scheme *scheme,
                             int device, int *err);

/* Number of cases of a handle (1 for e2d_create). */
int e2d_batch_cases(e2d_handle *h);

/* Releases the handle (Euler2D_Quad_Block::deallocate, Euler2DQuad.h:~700). */
void e2d_destroy(e2d_handle *h);

/* Uploads the primitive state W of every cell [nblk][4][NCj][NCi] (host
 * memory) and sets U = U(W); ghost values are kept until the next ghost fill.
 * Replaces the ICs / Uo assignment loops (Euler2DQuadSingleBlock.cc:1689). */
int e2d_set_state(e2d_handle *h, const double *W);

/* Uploads the conserved state U of every cell [nblk][4][NCj][NCi] and sets
 * W = W(U): the state a restart file holds (operator>> of
 * Euler2D_Quad_Block reads U and derives W, Euler2DQuad.h:1356-1362). */
int e2d_set_conserved(e2d_handle *h, const double *U);

/* Downloads W and/or U (either may be NULL). */
int e2d_get_state(e2d_handle *h, double *W, double *U);

/* Ghost exchange between blocks followed by the BCs of every block:
 * Send_All_Messages (src_2D/AMR/AdaptiveBlock2D_MessagePassing.h:7883) then
 * BCs (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:2354). */
int e2d_fill_ghosts(e2d_handle *h);

/* dUdt_Residual_Evaluation for all blocks (Euler2DQuadSingleBlock.cc:5095 ->
 * Euler2DQuad.cc:814): ghost fill, least-squares reconstruction with the
 * limiter, flux per face, flux divergence into dUdt.  dUdt (host, may be
 * NULL) receives [nblk][4][NCj][NCi] with zero ghost entries. */
int e2d_residual(e2d_handle *h, double *dUdt);

/* Gradients and limiter values of the last reconstruction (SolnBlk.dWdx,
 * dWdy, phi), each [nblk][4][NCj][NCi]; any may be NULL. */
int e2d_get_reconstruction(e2d_handle *h, double *dWdx, double *dWdy, double *phi);

/* n_steps explicit multistage time steps, each in the order of the
 * reference's explicit loop (src_2D/Euler2D/Euler2DQuadSolvers.cc:657-898):
 * CFL + global minimum, Set_Global_TimeStep (global dt), residual norms,
 * then per stage ghost fill, dUdt_Multistage_Explicit (Euler2DQuad.cc:1235)
 * and Update_Solution_Multistage_Explicit (Euler2DQuadSingleBlock.cc:5300).
 * hist (host, may be NULL) receives [n_steps][ncase][4] = dt_min, L1, L2,
 * Max of the density residual of each case as the loop computes them before
 * each step (ncase = 1 unless the handle is a batch). */
int e2d_rk_steps(e2d_handle *h, int n_steps, double *hist);

/* L1, L2 and max norms of the density residual dUdt[...][0][1] over all
 * interior cells (Euler2DQuadMultiBlock.cc:1017-1190); out receives
 * [ncase][3] (three values for a single case). */
int e2d_norms(e2d_handle *h, double *out);

/* CFL (Euler2DQuadSingleBlock.cc:3019-3080) of the current state: the
 * stability time step of every interior cell into dt (host, may be NULL;
 * [nblk][NCj][NCi], ghost entries untouched) and their minimum over all
 * blocks of each case into dtmin[ncase] (CFL of Euler2DQuadMultiBlock.cc:963
 * with CFFC_Minimum_MPI). */
int e2d_cfl(e2d_handle *h, double *dt, double *dtmin);

/* Deck-driven solve: Euler2DQuadSolver(char *Input_File_Name, int
 * batch_flag) (Euler2DQuadSolvers.cc:26) through the C++ host layer of
 * cffc_euler2d.hpp.  Returns 0, the line number of the first invalid deck
 * entry, or a library error. */
int e2d_solver_run(const char *input_file, int batch_flag);

/* Self-test of the tensor-core path the warm-start network uses (tcgen05,
 * BF16 operands in shared memory, FP32 accumulator in TMEM): D[128][N] =
 * A[128][K] * B[N][K]^T for host BF16 bit patterns A, B and host FP32 D;
 * 16 <= N <= 256 and 16 <= K <= 128, multiples of 16.  No reference
 * counterpart. */
int e2d_tc_selftest(const uint16_t *A, const uint16_t *B, float *D, int N, int K);

/* ---- Learned warm start (no reference counterpart) ---------------------
 * A per-cell network, 16 input features -> 128 -> 128 (tanh) -> 4 outputs,
 * evaluated and trained by tcgen05 kernels (BF16 operands, FP32
 * accumulation in TMEM).  The caller builds the features and targets (the
 * normalised converged state of cases the Newton-Krylov solver produced);
 * its prediction seeds e2d_set_state, and the solver then drives every case
 * to the same residual tolerance as from the freestream.
 * Parameters, flat FP32 (e2d_mlp_nparams() of them): W1[128][16], b1[128],
 * W2[128][128], b2[128], W3[16][128] (rows 4..15 unused), b3[16].
 * X, T, Y are device pointers: X[n][16], T[n][4], Y[n][4] FP32; stream is a
 * cudaStream_t or NULL. */
typedef struct e2d_mlp e2d_mlp;
e2d_mlp *e2d_mlp_create(uint64_t seed, int *err);  /* Glorot-uniform weights */
void e2d_mlp_destroy(e2d_mlp *m);
int e2d_mlp_nparams(void);
/* out (host, may be NULL) <- parameters; then parameters <- in (may be NULL) */
int e2d_mlp_params(e2d_mlp *m, float *out, const float *in);
int e2d_mlp_forward(e2d_mlp *m, const float *X, int n, float *Y, void *stream);
/* gradient of sum((Y - T)^2) / n into grad (host, may be NULL), loss (host) */
int e2d_mlp_gradient(e2d_mlp *m, const float *X, const float *T, int n, float *grad, double *loss,
                     void *stream);
/* steps of full-batch Adam (0.9, 0.999, 1e-8) at learning rate lr */
int e2d_mlp_train(e2d_mlp *m, const float *X, const float *T, int n, int steps, float lr, float *loss_hist,
                  void *stream);

/* Newton-Krylov-Schwarz parameters: the NKS_Input_Parameters fields the
 * Euler2D steady path reads (src_2D/NewtonKrylovSchwarz2D/NKSInput2D.h:128-172;
 * defaults in brackets).  The Frechet derivative is first order.  The
 * preconditioner (Block_Preconditioner, Block_Preconditioner2D.h:261-800)
 * is block Jacobi or BPKIT's ILU(k) on the approximate Jacobian, both with
 * exact inverses of the 4x4 diagonal blocks (LP_INVERSE).  Of the reference's
 * Jacobian orders, Euler2D provides the first-order HLLE Jacobian and the
 * source-terms-only one; the others end its run (they need specializations
 * Euler2D does not have) and are not offered here.  Zero-filled fields past
 * max_gmres select the reference's defaults. */
#define E2D_PRECON_BLOCK_JACOBI 0   /* GMRES_Block_Preconditioner Diagonal  */
#define E2D_PRECON_BLOCK_ILUK 1     /* GMRES_Block_Preconditioner ILUK      */
#define E2D_JACOBIAN_FIRST_ORDER_HLLE 0  /* First_Order_Inviscid_HLLE       */
#define E2D_JACOBIAN_SOURCE_TERMS_ONLY 1 /* Source_Terms_Only (-I/dt)       */
typedef struct e2d_nks_params {
  int32_t max_newton;        /* Maximum_Number_of_NKS_Iterations            */
  int32_t gmres_restart;     /* GMRES_Restart                       [30]    */
  int32_t max_gmres;         /* Maximum_Number_of_GMRES_Iterations          */
  int32_t block_preconditioner; /* E2D_PRECON_*                    [Jacobi] */
  double overall_tol;        /* Overall_Tolerance, L2 density drop [1e-5]   */
  double cfl0;               /* Finite_Time_Step_Initial_CFL        [1]     */
  double gmres_tol_initial;  /* GMRES_Initial_Tolerance             [1e-5]  */
  double gmres_tol_final;    /* GMRES_Final_Tolerance               [1e-5]  */
  double epsilon0;           /* Epsilon_Naught                      [1e-6]  */
  double min_ratio;          /* Min_Finite_Time_Step_Norm_Ratio     [1e-10] */
  /* Per case (host, may be NULL): the L2 the residual ratio, the tolerance
   * and the SER CFL are measured against instead of the first residual
   * (library extension; a warm-started case passes its freestream residual
   * so that it is driven to the same absolute level as a cold start). */
  const double *l2_reference;
  int32_t ilu_level_of_fill; /* GMRES_ILUK_Level_of_Fill, 0-16         [0]     */
  int32_t jacobian_order;    /* Jacobian_Order: E2D_JACOBIAN_*   [HLLE]    */
  /* Per case (host, may be NULL): the L2 the SER CFL ratio is measured
   * against, while the tolerance keeps l2_reference (library extension; a
   * warm-started case passes its own first residual, so its pseudo-time
   * step grows from the initial CFL as a cold start's does). */
  const double *cfl_reference;
} e2d_nks_params;

/* One Newton step of the history (the values the reference prints). */
typedef struct e2d_nks_step {
  double l1, l2, lmax;       /* density residual norms before the step      */
  double ratio;              /* L2 / L2 of the first step                   */
  double cfl;                /* finite-time-step CFL of the step            */
  double gmres_resid0, gmres_relres; /* initial residual, final ratio       */
  int32_t gmres_iters, gmres_restarts, gmres_failed, pad;
} e2d_nks_step;

/* Steady solve by pseudo-transient Newton-Krylov: the Newton loop of
 * Internal_Newton_Krylov_Schwarz_Solver (NKS2D.h:412-1258) with SER CFL
 * (Finite_Time_Step, NKS2D.h:1316), the block-Jacobi or ILU(k)
 * preconditioner of Block_Preconditioner (Block_Preconditioner2D.h:352-800,
 * BPKIT BJacobi / BILUK with LP_INVERSE), right-preconditioned restarted matrix-free GMRES with modified
 * Gram-Schmidt (GMRES2D.h:790-1544) and Newton_Update with positivity
 * back-off (Euler2DQuadNKS.h:23-92).  hist (host, may be NULL) receives one
 * entry per Newton step evaluated, *n_steps their count.  Returns 0, or a
 * negative library error. */
int e2d_nks(e2d_handle *h, const e2d_nks_params *p, e2d_nks_step *hist, int *n_steps);

/* The Newton step's preconditioner on its own: each cell's dt is the
 * CFL-limited step (local or global, as the scheme says) times cfl, as the
 * Newton loop sets it (NKS2D.h:913-930); then
 * Block_Preconditioner::Update_Jacobian_and_Preconditioner and
 * Apply_Preconditioner (Block_Preconditioner2D.h:352, 787) for every block:
 * z = M^-1 v.  v and z are host arrays in the GMRES vector layout
 * [nblk][NCj][NCi][4] (ghost entries of v ignored, of z zero).  The state
 * is left as it was; dt is overwritten.  Returns 0 or a library error. */
int e2d_block_precon_apply(e2d_handle *h, const e2d_nks_params *p, double cfl, const double *v, double *z);

/* The level-of-fill pattern of the ILU(k) preconditioner for blocks of
 * nci x ncj cells, as BPKIT's symbolic_ilu (bpkit/src/SparseUtil.cc:198)
 * builds it on the reference's block matrix (ghost rows included), then
 * restricted to interior cells: row_ptr[nci*ncj + 1], col[*nnz] (interior
 * cell index y*nci + x, ascending per row; written only when *nnz <= cap),
 * levels[2] (may be NULL) the forward and backward dependency-level counts.
 * Host work only.  Returns 0 or a library error. */
int e2d_ilu_pattern(int32_t nci, int32_t ncj, int32_t level, int32_t *row_ptr, int32_t *col, int32_t cap,
                    int32_t *nnz, int32_t *levels);

/* Device status word: 0 or the first error a kernel recorded. */
int e2d_status(e2d_handle *h);

/* Device pointers of the resident state (for callers that keep data in HBM):
 * W, U, dUdt as [nblk][4][NCj][NCi] doubles. */
int e2d_device_state(e2d_handle *h, double **W, double **U, double **dUdt);

/* Runs the handle's work on the caller's CUDA stream (a cudaStream_t; NULL
 * restores the handle's own stream).  No reference counterpart: the
 * reference is single-threaded host code. */
int e2d_set_stream(e2d_handle *h, void *stream);

/* Runs n_steps explicit steps launch by launch with CUDA events around each
 * kernel and returns the mean device time in milliseconds per launch of each
 * kernel kind: out[0] ghost fill, out[1] RK stage 1, out[2] RK stage 2,
 * out[3] CFL, out[4] norms (partial + final), out[5] whole step.  The state
 * advances as with e2d_rk_steps.  Profiling aid; no reference counterpart. */
int e2d_kernel_times(e2d_handle *h, int n_steps, double out[6]);

/* Self-test of the fast FP64 path's Newton-refined reciprocal, reciprocal
 * square root and square root against IEEE division / sqrt on n device
 * inputs x (> 0): out[0..2] receive the largest relative errors (host).
 * No reference counterpart. */
int e2d_fastmath_check(const double *x, int n, double *out);

/* Switches the precision of the handle's reconstruction and flux
 * (E2D_PREC_*) for the calls that follow -- e.g. an FP32 Newton-Krylov
 * phase down to the single-precision residual floor, then FP64 to the final
 * tolerance on the same state.  No reference counterpart. */
int e2d_set_precision(e2d_handle *h, int precision);

/* The stage kernel the handle's autotuner chose when the handle was created:
 * *kernel 0 = the tiled kernel, 1 = the column-marching kernel with *rows
 * rows per chunk; *us the tuner's time of one explicit stage with it (0 when
 * no tuning ran: an odd block width or a degenerate edge, where the tiled
 * kernel is the only one).  Any pointer may be NULL.  The environment variable
 * CFFC_E2D_STAGE_KERNEL=tiled or =march, read when a handle is created,
 * fixes the kernel without tuning (the marching kernel still only where it
 * applies).  No reference counterpart. */
int e2d_stage_config(e2d_handle *h, int *kernel, int *rows, double *us);

/* The deep warm-start network (library extension, no reference
 * counterpart): 5 input features padded to 16, four hidden layers of 256
 * units with GELU (tanh form), 4 outputs; BF16 tcgen05 products with FP32
 * accumulation, layer by layer over batches of rows.  X: device [n][16]
 * FP32 (features 5..15 zero), T: device [n][4], Y: device [n][4].  Training
 * takes `steps` Adam steps on minibatches of `batch` rows drawn without
 * replacement per epoch (seeded); loss_hist (host, may be NULL) receives the
 * minibatch losses. */
typedef struct e2d_mlp_deep e2d_mlp_deep;
e2d_mlp_deep *e2d_mlp_deep_create(uint64_t seed, int *err);
void e2d_mlp_deep_destroy(e2d_mlp_deep *d);
int e2d_mlp_deep_nparams(void);
int e2d_mlp_deep_params(e2d_mlp_deep *d, float *out, const float *in);
int e2d_mlp_deep_forward(e2d_mlp_deep *d, const float *X, int n, float *Y, void *stream);
int e2d_mlp_deep_gradient(e2d_mlp_deep *d, const float *X, const float *T, int n, float *grad, double *loss,
                          void *stream);
int e2d_mlp_deep_train(e2d_mlp_deep *d, const float *X, const float *T, int n, int steps, int batch, float lr,
                       uint64_t seed, float *loss_hist, void *stream);

/* Largest block count e2d_residual_norms_static serves. */
#define E2D_NORMS_STATIC_MAX_BLOCKS 4096

/* L1, L2 and max norms of the density residual of a caller-owned device
 * array, computed without allocating any device memory.  No counterpart in
 * the reference: it is for callers that cannot allocate when they need the
 * norms (allocation may stall or synchronise the device mid-loop, their
 * process's allocator owns all device memory, or they forbid allocation
 * after start-up).  Same result as e2d_norms, within reduction-order
 * rounding.
 *   dUdt    device pointer, [nblk][4][NCj][NCi] with two ghost layers
 *           (NCi = nci + 4, NCj = ncj + 4); only interior density is read
 *   out     device pointer to 3 doubles: L1, L2, Max
 *   stream  cudaStream_t to run on (NULL: the default stream)
 * The scratch is a fixed device array of 3 * E2D_NORMS_STATIC_MAX_BLOCKS
 * doubles (96 KiB), held on every GPU that loads the library until exit;
 * nblk above E2D_NORMS_STATIC_MAX_BLOCKS is rejected with E2D_ERR_ARG.
 * The first call on a device looks up the array's device address (with that
 * device current); that lookup may load the library's device code, which
 * can allocate device memory, so make the first call at start-up, before
 * any stream capture.  Later calls allocate nothing.  All calls share the
 * array: calls that overlap on the GPU race. */
int e2d_residual_norms_static(const double *dUdt, int32_t nblk, int32_t nci, int32_t ncj,
                              double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CFFC_E2D_H */

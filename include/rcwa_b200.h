/*
 * rcwa_b200.h — C ABI of the B200 RCWA diffraction-efficiency engine.
 *
 * Plain C types only: pointers, sizes, and complex numbers as interleaved
 * double pairs.  Every entry point returns an RCWA_* status code.  All device
 * memory is owned by the engine; host buffers passed in are only read during
 * the call, host buffers passed out are written before the call returns.
 *
 * Each entry point names the reference interface it replaces
 * (Sirokujira/OpenRCWA paths, file:line).  Units are the caller's: lengths in
 * any unit (the .ofd bridge uses metres), wavenumbers in rad per that unit.
 */
#ifndef RCWA_B200_H
#define RCWA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define RCWA_OK            0
#define RCWA_ERR_INVALID   1  /* bad sizes / pointers / geometry                     */
#define RCWA_ERR_CUDA      2  /* CUDA runtime failure                                */
#define RCWA_ERR_NOCONV    3  /* eigenvalue QR exceeded its iteration budget         */
#define RCWA_ERR_SINGULAR  4  /* exactly zero pivot in an LU factorisation           */
#define RCWA_ERR_NONFINITE 5  /* NaN / Inf in a result                               */
#define RCWA_ERR_GRAZING   6  /* kz == 0 or incident kz ~ 0 (scatterPlaneWave early return,
                                 rcwa/RCWASolver.cpp:1843-1847,1898-1901)            */
#define RCWA_ERR_NOMEM     7  /* device allocation failed                            */
#define RCWA_ERR_NODEVICE  8  /* no usable CUDA device                               */
#define RCWA_ERR_UNSUPPORTED 9 /* a feature outside this engine's scope (see docs)  */

/* ---- Fourier rule options (rcwa/FourierSolver2D.h:8-13) ------------------- */
#define RCWA_CONTINUOUS_XY   0
#define RCWA_DISCONTINUOUS_X 1
#define RCWA_DISCONTINUOUS_Y 2

/* ---- precision of the batched solve ---------------------------------------- */
#define RCWA_PREC_FP64  0     /* every stage complex128                           */
#define RCWA_PREC_MIXED 1     /* cascade GEMMs (F, G, Rud, Tdd), modal V = Q W
                                 products and the updates between the 128-wide
                                 blocks of the interface and tau LU
                                 factorisations and solves in 3xTF32 on the
                                 tensor cores (FP32 accumulation within
                                 K-blocks of 256, FP64 across); the eigensolve,
                                 the LU panels and triangles, the half-spaces
                                 and the efficiency sums stay FP64.  Stacks
                                 with a metallic layer (Re eps < 0 in some
                                 cell) keep FP64 throughout: their cascade is
                                 too ill-conditioned for 3xTF32               */

typedef struct { double re, im; } rcwa_cplx;

typedef struct rcwa_engine rcwa_engine;
typedef struct rcwa_plan rcwa_plan;

/* A layer stack on one common cell grid: what RCWASolver(nX, nY) holds after
 * addLayer() of every layer (rcwa/RCWASolver.h:67-84, rcwa/Layer.h:29-31).
 * eps[l] is a (ncy-1) x (ncx-1) row-major grid, row = y strip, column = x
 * strip, exactly the Layer eps_ matrix.  Layer 0 is the incidence half-space,
 * layer n_layers-1 the transmission half-space.  A uniform half-space (every
 * cell equal) takes closed-form modes; one whose cells differ is solved like
 * a patterned layer, as the reference solves every layer type
 * (rcwa/RCWASolver.cpp:194-210), and its values at (0, 0) enter the
 * efficiencies (rcwa/RCWASolver.cpp:1823-1830).  thickness[l] is used
 * for 0 < l < n_layers-1 only (rcwa/RCWASolver.cpp:415-431).  mu, when not
 * NULL, is the relative permeability on the same grid (Layer(coordX, coordY,
 * eps, mu), rcwa/Layer.cpp:41-72): a layer with a cell whose mu differs from 1
 * by more than 1e-12 takes the magnetic branch of the wave equation
 * (rcwa/Layer.cpp:128-164,205-213); the half-spaces' mu enters their modes
 * and the efficiencies (rcwa/RCWASolver.cpp:1826-1907).  NULL: mu = 1. */
typedef struct {
  int nHx, nHy;              /* harmonics: 2*nHx+1 by 2*nHy+1 orders            */
  int ncx, ncy;              /* number of cell edges along x and y (>= 2)        */
  const double* cx;          /* [ncx] ascending; period Lx = cx[ncx-1]-cx[0]     */
  const double* cy;          /* [ncy] ascending                                  */
  int n_layers;              /* >= 2                                             */
  const rcwa_cplx* eps;      /* [n_layers][ncy-1][ncx-1]                         */
  const double* thickness;   /* [n_layers]                                       */
  const rcwa_cplx* mu;       /* [n_layers][ncy-1][ncx-1] or NULL                 */
} rcwa_stack;

/* One solve point: one RCWASolver::solve (rcwa/RCWASolver.cpp:139-148) of a
 * stack at one wavelength and Bloch wavevector (setBlochWavevector,
 * rcwa/RCWASolver.h:180). */
typedef struct {
  int stack;                 /* index into the stack array                       */
  double lambda;             /* vacuum wavelength                                */
  double kx0, ky0;           /* Bloch wavevector offsets                         */
} rcwa_point;

/* ---- engine ----------------------------------------------------------------- */
const char* rcwa_status_string(int status);
int rcwa_engine_create(int device, rcwa_engine** out);
/* Destroy every plan and surrogate network of the engine first: plans return
 * their device buffers to the engine's pool and workspace cache. */
void rcwa_engine_destroy(rcwa_engine* e);
/* Message of the last failure on this engine ("" if none). */
const char* rcwa_engine_last_error(const rcwa_engine* e);

/* Batched diffraction efficiencies.  Replaces, for every point, the sequence
 *   RCWASolver::solve                         rcwa/RCWASolver.cpp:139-148
 *   generateHorizontalPlaneWave(px, py, 0)    rcwa/RCWASolver.cpp:1778-1789
 *   scatterPlaneWave(c, 0, L-1, k0, REF, TRN) rcwa/RCWASolver.cpp:1792-1908
 *   R = REF.sum(), T = TRN.sum()              sol/rcwa_bridge.cpp:311-312
 * for n_exc incident transverse polarisation vectors per point.
 *   pxy        [n_pts][n_exc][2] complex (px, py), host
 *   R, T       [n_pts][n_exc], host
 *   ref_orders, trn_orders: NULL or per-point blocks of n_exc*N doubles, point
 *              p's block starting at sum_{q<p} n_exc*N_q (N = orders of the
 *              point's stack), order k = (2nHy+1)*(m+nHx) + (n+nHy); unmasked
 *              REF/TRN vectors as scatterPlaneWave returns them
 *   status     [n_pts] per-point RCWA_* code, host (may be NULL)
 * Returns RCWA_OK when the call itself ran; per-point failures are reported in
 * status (and the call returns the first non-zero point status). */
int rcwa_engine_solve_batch(rcwa_engine* e,
                            const rcwa_stack* stacks, int n_stacks,
                            const rcwa_point* pts, int n_pts,
                            int n_exc, const rcwa_cplx* pxy,
                            int precision,
                            double* R, double* T,
                            double* ref_orders, double* trn_orders,
                            int* status);

/* A layer stack whose patterned layers are given by their 2D Laurent
 * coefficient tables instead of a cell grid: F2D[p][q] =
 * (1/(Lx Ly)) integral of eps(x,y) exp(-i 2pi (m x/Lx + n y/Ly)), m = p - 2nHx,
 * n = q - 2nHy, the table layout of FourierSolver2D's ContinuousXY branch
 * (rcwa/FourierSolver2D.cpp:250-349).  All three convolution matrices of such a
 * layer are the table's block-Toeplitz matrix (the Laurent rule for every
 * tensor), e.g. the closed-form disk transform of circular pillars, which the
 * reference only approximates by staircasing (rcwa/RCWADriver.cpp:19-37).
 * Layers 0 and n_layers-1 are uniform half-spaces of permittivity eps_half[0]
 * and eps_half[1]. */
typedef struct {
  int nHx, nHy;              /* harmonics: 2*nHx+1 by 2*nHy+1 orders            */
  double Lx, Ly;             /* periods                                          */
  int n_layers;              /* >= 2                                             */
  const rcwa_cplx* eps_half; /* [2] incidence and transmission half-spaces      */
  const rcwa_cplx* f2d;      /* [n_layers-2][(4nHx+1)*(4nHy+1)] row-major        */
  const double* thickness;   /* [n_layers] (0 < l < n_layers-1 used)             */
} rcwa_table_stack;

/* rcwa_engine_solve_batch / rcwa_plan_create for Laurent-table stacks
 * (same points, outputs and precision modes). */
int rcwa_engine_solve_tables(rcwa_engine* e,
                             const rcwa_table_stack* stacks, int n_stacks,
                             const rcwa_point* pts, int n_pts,
                             int n_exc, const rcwa_cplx* pxy,
                             int precision,
                             double* R, double* T,
                             double* ref_orders, double* trn_orders,
                             int* status);
int rcwa_plan_create_tables(rcwa_engine* e,
                            const rcwa_table_stack* stacks, int n_stacks,
                            const rcwa_point* pts, int n_pts,
                            int n_exc, const rcwa_cplx* pxy, int precision,
                            rcwa_plan** out);

/* The same solve split in three so that a caller can keep the inputs resident
 * and time the device work alone: plan_create uploads the inputs and sizes the
 * workspace, plan_execute enqueues every kernel on `stream` (a cudaStream_t,
 * NULL = the engine's own stream) without synchronising, plan_results waits
 * and copies the outputs back (same layouts as rcwa_engine_solve_batch). */
int rcwa_plan_create(rcwa_engine* e,
                     const rcwa_stack* stacks, int n_stacks,
                     const rcwa_point* pts, int n_pts,
                     int n_exc, const rcwa_cplx* pxy, int precision,
                     rcwa_plan** out);
int rcwa_plan_execute(rcwa_plan* p, void* stream);
int rcwa_plan_results(rcwa_plan* p, double* R, double* T,
                      double* ref_orders, double* trn_orders, int* status);
/* Re-evaluate the efficiencies of an executed plan for new incident
 * polarisation vectors pxy [n_pts][n_exc][2] without solving again (the
 * scattering matrices stay on the device): the second and later
 * generateHorizontalPlaneWave + scatterPlaneWave pairs of one solve
 * (rcwa/RCWASolver.cpp:1778-1908).  Plans whose points needed more than one
 * device-memory chunk return RCWA_ERR_UNSUPPORTED.  Read the results with
 * rcwa_plan_results. */
int rcwa_plan_rescatter(rcwa_plan* p, const rcwa_cplx* pxy);

/* The scattering matrix of one point of an executed plan, as the
 * RCWASolver::Tdd() / Rud() accessors return it (rcwa/RCWASolver.h:141-142;
 * the RTCM cascade's final Tdd_ and Rud_, rcwa/RCWASolver.cpp:378-492, in the
 * modal basis of the uniform half-spaces, W = I):
 *   Rud, Tdd  NULL or host [n*n] row-major complex, n = 2*N of the point's
 *             stack (either may be NULL)
 * Waits for the plan's work.  Plans whose points needed more than one
 * device-memory chunk return RCWA_ERR_UNSUPPORTED (the engine reuses the
 * workspace chunk by chunk); a point index out of range RCWA_ERR_INVALID. */
int rcwa_plan_smatrix(rcwa_plan* p, int point, rcwa_cplx* Rud, rcwa_cplx* Tdd);

/* Number of engine kernel launches the last plan_execute enqueued. */
long long rcwa_plan_launch_count(const rcwa_plan* p);
/* Schedules the plan uses, per chunk: sched[6] = {matrix order n, points,
 * interface LU schedule, tau LU schedule, Schur crossover, product path}
 * (values as in rcwa_tuner_*; product path 1 for FP64 plans and for chunks
 * whose points all keep FP64 products).  Returns the number of chunks (chunk < 0 or
 * sched NULL: only the count), -1 for a bad plan or chunk. */
int rcwa_plan_schedule(const rcwa_plan* p, int chunk, int* sched);
/* Per-stage device time: with profiling on, plan_execute records CUDA events
 * between the stages on its stream; plan_stage_times waits and writes the
 * milliseconds of every stage of the last execution into ms[max_stages] and
 * returns the number of stages; rcwa_stage_name names stage i.  (The
 * reference only has commented-out host timers, rcwa/Layer.cpp:245-252.) */
int rcwa_plan_set_profiling(rcwa_plan* p, int on);
int rcwa_plan_stage_times(rcwa_plan* p, double* ms, int max_stages);
const char* rcwa_stage_name(int stage);
void rcwa_plan_destroy(rcwa_plan* p);

/* ---- stage entry points (host buffers in and out, synchronous) -------------- */

/* FourierSolver1D(x, d).solve(f, M, Ff)   rcwa/FourierSolver1D.cpp:11-41.
 * x[nxe] edges, f[nxe-1], Ff[M]. */
int rcwa_fourier1d(rcwa_engine* e, const double* x, int nxe, double d,
                   const rcwa_cplx* f, int M, rcwa_cplx* Ff);

/* FourierSolver2D(cx, cy).solve(f, nx, ny, opt, Ff)   rcwa/FourierSolver2D.cpp:12-351.
 * f[(ncy-1)*(ncx-1)] row-major (row = y), Ff[(nx*ny)^2] row-major. */
int rcwa_fourier2d(rcwa_engine* e, const double* cx, int ncx, const double* cy, int ncy,
                   const rcwa_cplx* f, int nx, int ny, int opt, rcwa_cplx* Ff);

/* Layer::solve for one patterned layer   rcwa/Layer.cpp:255-273 with
 * Layer::waveEqnCoeff (:75-253) and WaveEquationSolver::solve
 * (rcwa/WaveEquationSolver.cpp:24-37).  alpha/beta[nx*ny] are the diagonals
 * of Kx/Ky (RCWASolver::evaluateAlphaBeta, rcwa/RCWASolver.cpp:242-266).
 * Outputs (any may be NULL), n = 2*nx*ny:
 *   W, V [n*n] row-major: eigvecE / eigvecH (columns = modes, unit 2-norm)
 *   gamma [n]: Layer::gamma() = keff/k0
 *   eigenvalues [n]: eigenvalues of P*Q. */
int rcwa_layer_solve(rcwa_engine* e, const double* cx, int ncx, const double* cy, int ncy,
                     const rcwa_cplx* eps, int nx, int ny,
                     const double* alpha, const double* beta, double lambda,
                     rcwa_cplx* W, rcwa_cplx* V, rcwa_cplx* gamma, rcwa_cplx* eigenvalues);

/* Batched right eigenvectors of general complex matrices:
 * MKLEigenSolver<MatrixXcs>::compute (LAPACKE zgeev('N','V') branch,
 * rcwa/MKLEigenSolver.hpp:102-179).  A[batch][n*n] row-major, w[batch][n],
 * VR[batch][n*n] row-major (columns unit 2-norm), info[batch]. */
int rcwa_zgeev_batched(rcwa_engine* e, int n, int batch, const rcwa_cplx* A,
                       rcwa_cplx* w, rcwa_cplx* VR, int* info);

/* Failure-injection hook for tests of the RCWA_ERR_NOCONV path (no
 * counterpart in the reference, whose LAPACK zgeev has a fixed iteration
 * limit, rcwa/MKLEigenSolver.hpp:131): caps the QR sweeps of every later
 * eigensolve at `sweeps` (0 restores the built-in budget of 30*max(10, n)).
 * Process-wide; a plan captured into a CUDA graph keeps the cap that was set
 * when it was captured.  Returns RCWA_ERR_INVALID for a negative cap. */
int rcwa_set_qr_sweep_limit(int sweeps);

/* CTAs per matrix of the Hessenberg reduction and the multishift Schur
 * iteration (no reference counterpart: a scheduling choice of this engine).
 * A batch of large matrices (order >= 1024) that would leave half of the SMs
 * idle is given a thread-block cluster of up to 8 CTAs per matrix; every
 * element is computed by the same operations whatever the team size, so the
 * results are identical.  ctas = 0 restores the automatic choice, 1..8 forces
 * a size for every later eigensolve (matrices of order >= 64).  Process-wide;
 * a plan captured into a CUDA graph keeps the size chosen when it was
 * captured.  Returns RCWA_ERR_INVALID outside 0..8. */
int rcwa_set_eig_cluster(int ctas);
/* The team size rcwa_set_eig_cluster's setting gives a batch of `batch`
 * order-n matrices on the current device. */
int rcwa_eig_cluster_size(int n, int batch);
/* The same for the panel step of the LU factorisations (interface and tau
 * factorisations, rcwa_zgetrf stages): a batch of large matrices (order >=
 * 1024) that would leave half of the SMs idle factorises each 32-column
 * panel on a cluster of up to 8 CTAs per matrix, with identical factors.
 * ctas = 0: automatic, 1..8: forced; RCWA_ERR_INVALID outside 0..8. */
int rcwa_set_lu_cluster(int ctas);

/* Fields inside a solved stack, for one point of an executed single-chunk
 * plan: the mode amplitudes of every interior layer for the plane wave
 * (px, py) of generateHorizontalPlaneWave (RCWASolver::evaluateIntermediateField,
 * rcwa/RCWASolver.cpp:1505-1644), then one field component on a slice as
 * RCWASolver::saveFieldImage evaluates it before writing its CSV
 * (rcwa/RCWASolver.cpp:707-1012, no layer translation).  slice: 0 = XY at
 * depth coord, 1 = XZ at y = coord, 2 = YZ at x = coord, the depth measured
 * from the top of the first interior layer (the slice covers the interior
 * layers); component 0..5 = Ex, Ey, Ez, Hx, Hy, Hz; nres1 samples along x
 * (XY, XZ) or y (YZ), at cell centres from the grid's origin; field:
 * rows x nres1 complex, rows from rcwa_plan_field_rows (saveFieldImage's
 * nRes2 = max(1, (int)(nres1 L2 / L1))).  The stack needs an interior layer.
 * Allocates device scratch for the call (about 7 n^2 complex per interface)
 * and waits for it to finish. */
int rcwa_plan_field_rows(const rcwa_plan* plan, int point, int slice, int nres1, int* rows);
int rcwa_plan_field(rcwa_plan* plan, int point, rcwa_cplx px, rcwa_cplx py, int slice, double coord,
                    int component, int nres1, rcwa_cplx* field);
int rcwa_lu_cluster_size(int n, int batch);

/* Batched complex GEMM D = alpha*A*B + beta*C (row-major, host buffers
 * [batch][M*K], [batch][K*N], [batch][M*N]; C may be NULL when beta = 0), the
 * product kernel of the cascade: RCWA_PREC_FP64 on the FP64 tensor path,
 * RCWA_PREC_MIXED as 3xTF32 on the fifth-generation tensor cores.  No
 * counterpart in the reference (its Eigen products). */
int rcwa_zgemm_batched(rcwa_engine* e, int M, int N, int K, int batch, const rcwa_cplx* A, const rcwa_cplx* B,
                       const rcwa_cplx* C, rcwa_cplx alpha, rcwa_cplx beta, int precision, rcwa_cplx* D);

/* ---- Schedule autotuner ----------------------------------------------
 * No counterpart in the reference (its CPU path calls LAPACK with fixed
 * blocking).  A tuner is a table of schedule choices keyed by decision, matrix
 * order n and batch class (waves of one-CTA-per-matrix work: 1, 2, 3, 4 for
 * 4-7, 8 for 8 and more).  Decisions and their choices:
 *   RCWA_TUNE_LU       0: one CTA factors each matrix, 1: panel by panel,
 *                      2: 128-column blocks (1 inside each block, then one
 *                      K = 128 trailing update per block; n >= 256)
 *   RCWA_TUNE_SCHUR    active-block size below which the Schur iteration uses
 *                      single-shift sweeps (64, 96, 128, 192; only 64 for
 *                      n < 64 and n >= 512; default 128 for 64 <= n < 128,
 *                      else 64)
 *   RCWA_TUNE_PRODUCT  mixed plans' cascade products and their tile shape,
 *                      0: 3xTF32 on tcgen05 with 128 x 128 output tiles,
 *                      1: FP64 tensor path, 2: 3xTF32 on tcgen05 with
 *                      128 x 256 output tiles
 * Every choice computes the same quantities (LU: same pivoting rule; Schur:
 * same convergence tests; products: within the mixed tolerance), so a tuner
 * changes speed, not results beyond rounding.
 * rcwa_engine_set_tuner: mode RCWA_TUNING_OFF (built-in rules),
 * RCWA_TUNING_TABLE (the table, else the rules) or RCWA_TUNING_AUTO (the
 * table, else time every candidate on the device while the plan is created,
 * on seeded random matrices, and record the fastest).  The engine does not
 * own the tuner; keep it alive while the engine uses it.  The table calls are
 * host-only and thread-safe.  rcwa_tuner_get writes -1 for a missing entry;
 * rcwa_tuner_entry lists entries (cand/ms: 4 slots, unused -1 / 0); the file
 * format is text, one entry per line. */
#define RCWA_TUNE_LU      0
#define RCWA_TUNE_SCHUR   1
#define RCWA_TUNE_PRODUCT 2
#define RCWA_TUNING_OFF   0
#define RCWA_TUNING_TABLE 1
#define RCWA_TUNING_AUTO  2
typedef struct rcwa_tuner rcwa_tuner;
int rcwa_tuner_create(rcwa_tuner** out);
void rcwa_tuner_destroy(rcwa_tuner* t);
int rcwa_tuner_set_sms(rcwa_tuner* t, int sms);
int rcwa_tuner_candidates(int op, int n, int* choices);
int rcwa_tuner_default(const rcwa_tuner* t, int op, int n, int batch);
int rcwa_tuner_set(rcwa_tuner* t, int op, int n, int batch, int choice);
int rcwa_tuner_get(const rcwa_tuner* t, int op, int n, int batch, int* choice);
int rcwa_tuner_count(const rcwa_tuner* t);
int rcwa_tuner_entry(const rcwa_tuner* t, int index, int* op, int* n, int* batch_class, int* choice,
                     int* ncand, int* cand, double* ms);
int rcwa_tuner_save(const rcwa_tuner* t, const char* path);
int rcwa_tuner_load(rcwa_tuner* t, const char* path);
int rcwa_engine_set_tuner(rcwa_engine* e, rcwa_tuner* t, int mode);
/* Time every candidate of (op, n, batch) now, record the entry, and return
 * the fastest choice and the candidates' milliseconds (ms[4]). */
int rcwa_tuner_measure(rcwa_engine* e, rcwa_tuner* t, int op, int n, int batch, int* choice, double* ms);

/* ---- learned surrogate ------------------------------------------------------
 * No counterpart in the reference.  A fully connected network with n_layers
 * hidden layers of n_hidden units (GELU) mapping n_in grating parameters to
 * n_out efficiencies, trained on efficiencies this engine computed; the
 * engine's FP64 solve is its fallback (openrcwa_b200/surrogate.py).
 * Parameters, in order for every layer: W (out x in, row-major) then b (out).
 * Training: FP32 weights, minibatch Adam on the mean squared error.
 * rcwa_mlp_predict: BF16 weights and activations with FP32 accumulation on the
 * tensor cores (n_hidden, n_out <= 256); rcwa_mlp_predict_fp32: the FP32
 * training forward.  Rows are host float arrays [n][n_in] / [n][n_out]. */
typedef struct rcwa_mlp rcwa_mlp;
int rcwa_mlp_create(rcwa_engine* e, int n_in, int n_hidden, int n_layers, int n_out, unsigned long long seed,
                    rcwa_mlp** out);
void rcwa_mlp_destroy(rcwa_mlp* m);
long long rcwa_mlp_param_count(const rcwa_mlp* m);
int rcwa_mlp_get_params(rcwa_mlp* m, float* params);
int rcwa_mlp_set_params(rcwa_mlp* m, const float* params);
int rcwa_mlp_set_data(rcwa_mlp* m, const float* X, const float* Y, int n);
int rcwa_mlp_train(rcwa_mlp* m, int epochs, int batch, float lr, unsigned long long seed, float* loss_per_epoch);
int rcwa_mlp_loss_grad(rcwa_mlp* m, const float* X, const float* Y, int n, double* loss, float* grad);
int rcwa_mlp_predict_fp32(rcwa_mlp* m, const float* X, int n, float* Y);
int rcwa_mlp_predict(rcwa_mlp* m, const float* X, int n, float* Y);
/* Squared Euclidean distance from each query row Q [n][n_in] (host floats,
 * the features the network was trained on) to its nearest row of the
 * training set given to rcwa_mlp_set_data, into d2[n] (host).  skip_self
 * ignores distances of exactly 0, so training rows passed as queries get
 * their leave-one-out distance.  n_in <= 32.  The surrogate's test of whether
 * a query lies where the network has seen data. */
int rcwa_mlp_nn_distance(rcwa_mlp* m, const float* Q, int n, int skip_self, float* d2);

/* ---- slab S-matrices and the Redheffer star product -------------------------
 * Batched, FP64, host buffers; every matrix row-major [batch][n*n].
 *
 * rcwa_slab_smatrix_batched: dtmm::RCWAScatterMatrix::compute_v2
 * (rcwa/RCWAScatterMatrix.cpp:90-146) -- the S-matrix of one z-uniform slab
 * with modes W, V, gamma[batch][n] seen from a reference medium W0, V0, over a
 * thickness wz at wavelength lambda (X = exp(i gamma wz lambda/2pi)).  The
 * slab S-matrix is symmetric: Rdu = Rud and Tdd = Tuu
 * (rcwa/RCWAScatterMatrix.h:40-47), so only Rud and Tuu are returned.
 *
 * rcwa_star_product_batched: the cascade update of the z-integrators
 * (core/RCWAIntegrator.cpp:57-67, core/RedhefferIntegrator.cpp:136-146):
 * the running S-matrix (Rud, Rdu, Tdd, Tuu), updated in place, absorbs the
 * slab (rud, rdu, tdd, tuu) below it.  Start from Tdd = Tuu = I,
 * Rud = Rdu = 0 (core/RCWAIntegrator.cpp:36-39).
 *
 * status[batch] (optional): 0 or RCWA_ERR_SINGULAR per item; the return value
 * is the first nonzero status. */
int rcwa_slab_smatrix_batched(rcwa_engine* e, int n, int batch,
                              const rcwa_cplx* W, const rcwa_cplx* V, const rcwa_cplx* gamma,
                              const rcwa_cplx* W0, const rcwa_cplx* V0,
                              const double* lambda, const double* wz,
                              rcwa_cplx* Rud, rcwa_cplx* Tuu, int* status);
int rcwa_star_product_batched(rcwa_engine* e, int n, int batch,
                              rcwa_cplx* Rud, rcwa_cplx* Rdu, rcwa_cplx* Tdd, rcwa_cplx* Tuu,
                              const rcwa_cplx* rud, const rcwa_cplx* rdu,
                              const rcwa_cplx* tdd, const rcwa_cplx* tuu, int* status);

/* RCWAIntegrator::compute(N) (core/RCWAIntegrator.cpp:21-86) over the
 * sampler's matrices: P, Q [nslab + 2][n*n] row-major as LayerSampler::sample
 * (core/LayerSampler.h:51-53) gives them at depth z0 (sample 0), at the
 * midpoints z0 + (i + 1/2)(z1 - z0)/nslab of the nslab slabs (samples
 * 1 .. nslab) and at z1 (sample nslab + 1).  Every sample's modes come from
 * WaveEquationSolver::solve (eigenvectors W of P Q, keff = GammaSqrtOp of the
 * eigenvalues, V = Q W keff^-1); the slabs' S-matrices are taken against the
 * modes at z1 and cascaded with the star product, pairwise in ceil(log2
 * nslab) batched levels (the product is associative; the reference folds
 * them from the top down), and the last step brings the top side into the
 * modes at z0.  Outputs (any may be NULL) as the integrator's accessors:
 * Rud, Rdu, Tdd, Tuu [n*n]; W0, V0 [n*n], gam0 [n] (z0); W1, V1, gam1 (z1).
 * nslab = 0 is the region without slabs (the identity S-matrix brought into
 * the modes at z0).  Returns RCWA_ERR_NOCONV / RCWA_ERR_NONFINITE from an
 * eigensolve, RCWA_ERR_SINGULAR from an LU, else RCWA_OK. */
int rcwa_rcwa_integrate(rcwa_engine* e, int n, int nslab, double lambda, double z0, double z1,
                        const rcwa_cplx* P, const rcwa_cplx* Q,
                        rcwa_cplx* Rud, rcwa_cplx* Rdu, rcwa_cplx* Tdd, rcwa_cplx* Tuu,
                        rcwa_cplx* W0, rcwa_cplx* V0, rcwa_cplx* gam0,
                        rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1);

/* DifferentialIntegrator::compute(N) (core/DifferentialIntegrator.cpp:21-133):
 * P, Q [2 nslab + 1][n*n] at z0 + k dz/2 (dz = (z1 - z0)/nslab), so slab i
 * takes samples 2i, 2i + 1, 2i + 2 (its ends and midpoint); the modes at z0
 * and z1 are those of samples 0 and 2 nslab.  Per slab the fourth-order
 * transfer blocks L11, L12, L21, L22 (:55-66) are taken into the modes at z1
 * and turned into an S-matrix (:73-97), all slabs in one batch; the cascade
 * and the last step are those of rcwa_rcwa_integrate.  nslab >= 1; outputs
 * and return codes as rcwa_rcwa_integrate. */
int rcwa_differential_integrate(rcwa_engine* e, int n, int nslab, double lambda, double z0, double z1,
                                const rcwa_cplx* P, const rcwa_cplx* Q,
                                rcwa_cplx* Rud, rcwa_cplx* Rdu, rcwa_cplx* Tdd, rcwa_cplx* Tuu,
                                rcwa_cplx* W0, rcwa_cplx* V0, rcwa_cplx* gam0,
                                rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1);

/* LayerSampler::sample (core/LayerSampler.h:51-53) as a callback: P and Q
 * (n*n row-major, host) at depth z; returns 0, or nonzero to abort. */
typedef int (*rcwa_sampler)(void* user, double z, rcwa_cplx* P, rcwa_cplx* Q);

/* RedhefferIntegrator::compute(p, maxN, pe) (core/RedhefferIntegrator.cpp:
 * 190-328, its triple-division branch): an interval's first-order
 * perturbation S-matrix about the modes at its midpoint
 * (evaluatePerturbationAndDifference, :330-398) is accepted when no entry of
 * its perturbation exceeds pe in modulus, else the interval is split in
 * thirds (the middle third keeps the parent's modes).  The intervals of one
 * subdivision level are evaluated in one batch (new samples through the
 * callback, their modes in one batched eigensolve); the accepted intervals,
 * in depth order, are projected from the modes above them, cascaded with the
 * star product and the bottom brought into the modes at z1.  max_intervals
 * bounds the accepted intervals (RCWA_ERR_NOCONV beyond it; the reference
 * ignores maxN).  n_intervals = N(), n_eig = the eigen-solves performed (the
 * reference's nEigVal() stays 2 in this branch).  Outputs as
 * rcwa_rcwa_integrate; a failing callback gives RCWA_ERR_INVALID. */
int rcwa_redheffer_integrate(rcwa_engine* e, int n, double lambda, double z0, double z1, double pe,
                             int max_intervals, rcwa_sampler sample, void* user,
                             rcwa_cplx* Rud, rcwa_cplx* Rdu, rcwa_cplx* Tdd, rcwa_cplx* Tuu,
                             rcwa_cplx* W0, rcwa_cplx* V0, rcwa_cplx* gam0,
                             rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1, int* n_intervals, int* n_eig);

/* ---- eigensolver without device allocation ---------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (code running inside another framework's memory pool, real-time loops where
 * an allocation may stall, hosts that fix their device footprint up front):
 * the same batched eigensolver as rcwa_zgeev_batched, on caller-owned DEVICE
 * buffers, with its scratch in a static device array of the library that every
 * GPU loading it holds until exit (about 38 MB).  Allocates nothing.
 *   A     device [batch][n*n] row-major, overwritten (Schur form on return)
 *   w     device [batch][n] eigenvalues
 *   VR    device [batch][n*n] row-major unit-norm right eigenvectors
 *   info  device [batch] per-matrix status (0 or RCWA_ERR_NOCONV/NONFINITE)
 *   stream  cudaStream_t (NULL = legacy default stream); the call is
 *           asynchronous on it.
 * Limits: n <= RCWA_NOALLOC_MAX_N and batch <= RCWA_NOALLOC_MAX_BATCH, else
 * RCWA_ERR_UNSUPPORTED.  The first call on a device looks up the scratch
 * array's device address (cudaGetSymbolAddress) with that device current;
 * under CUDA's lazy module loading (the default since CUDA 12.2) that lookup
 * is also when the driver reserves the array, so make the first call at
 * set-up time, before any stream capture; later calls reserve nothing.  A
 * CUDA error already pending on the calling thread is reported as
 * RCWA_ERR_CUDA and left pending.  All calls share the one scratch array, so
 * calls whose work overlaps on the GPU (other streams, other threads) race:
 * serialise them. */
#define RCWA_NOALLOC_MAX_N 64
#define RCWA_NOALLOC_MAX_BATCH 64
int rcwa_zgeev_batched_noalloc(int n, int batch, rcwa_cplx* A, rcwa_cplx* w,
                               rcwa_cplx* VR, int* info, void* stream);

/* ---- the .ofd RCWA mode (sol/rcwa_bridge.cpp) --------------------------- */

/* rcwalayer_t, same fields and order (include/orcwa_rcwa.h:33-41). */
typedef struct {
  double eps1, eps2, eps1i, eps2i, fill, fill_y, thickness;
} rcwa_layer_spec;

/* rcwapole_t, same fields and order (include/orcwa_rcwa.h:51-58); layer 0-based. */
typedef struct {
  int layer, side;
  double einf, ae, be, ce;
} rcwa_pole_spec;

/* The globals rcwa_run() reads (include/orcwa_rcwa.h:60-76, sol/rcwa_bridge.cpp:35-40). */
typedef struct {
  int nHx;                       /* NRcwaHarmonics   */
  double period_x;               /* RcwaPeriod       */
  int nHy;                       /* NRcwaHarmonicsY  */
  double period_y;               /* RcwaPeriodY (used when nHy > 0, else period_x) */
  int n_layers;                  /* NRcwaLayer       */
  const rcwa_layer_spec* layers; /* RcwaLayer        */
  int n_poles;                   /* NRcwaPole        */
  const rcwa_pole_spec* poles;   /* RcwaPole         */
  double theta_deg, phi_deg;     /* RcwaTheta, RcwaPhi */
  int n_freq;                    /* NFreq1           */
  const double* freq;            /* Freq1 [Hz]       */
} rcwa_ofd_setup;

/* The computation of rcwa_run (sol/rcwa_bridge.cpp:145-366) with every
 * frequency solved in one batch, without the file output:
 *   R, T        [n_freq][2]  (TE, TM) totals, REF.sum() / TRN.sum() (:311-312)
 *   ordR, ordT  NULL or [2][n_freq][nOrdX*nOrdY] propagating-order efficiencies,
 *               evanescent orders set to 0 (the bridge's ordR/ordT, :289-319)
 *   status      NULL or [n_freq]
 * Returns 1-style errors as RCWA_ERR_INVALID for an invalid setup (:149-152,
 * :246-249). */
int rcwa_ofd_solve(rcwa_engine* e, const rcwa_ofd_setup* s, double* R, double* T,
                   double* ordR, double* ordT, int* status);

#ifdef __cplusplus
}
#endif

#endif /* RCWA_B200_H */

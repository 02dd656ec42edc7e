/*
 * qesb.h — C ABI of the B200-native QES-Winds lambda solver (libqesb200.so).
 *
 * The library replaces the solve step that the reference reaches through
 *     Solver *SolverFactory::create(const int &type, const qes::Domain &, const float &tol)
 *     solver->resetLambda();
 *     solver->solve(WINDSGeneralData *WGD, const int &itermax);
 * (reference src/winds/SolverFactory.cpp:35-60, src/winds/Solver.h:61-120,
 * called from qesWinds/qesWindsMain.cpp:154-169). A C++ adaptor with exactly
 * that interface lives in qes-public_b200/host/Solver_B200.h.
 *
 * Arrays use the reference's own layouts (src/qes/Domain.h:143-167), passed
 * as plain pointers:
 *   cell arrays  (e f g h m n, icellflag, lambda): (nx-1)(ny-1)(nz-1) values,
 *                index i + j*(nx-1) + k*(nx-1)*(ny-1);
 *   face arrays  (u0 v0 w0 u v w):                 nx*ny*nz values,
 *                index i + j*nx + k*nx*ny;
 *   dz_array:                                       nz-1 values (ghost at 0);
 * with nx = Nx+1, ny = Ny+1, nz = Nz+2 (src/qes/Domain.cpp:11-13).
 *
 * Every entry point returns a qesb_status; none calls exit(). Handles are
 * owned by the caller; one handle serves one host thread at a time.
 */
#ifndef QESB_H
#define QESB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qesb_status {
  QESB_OK = 0,
  QESB_ERR_ARG = 1,      /* bad size, null pointer, unknown option */
  QESB_ERR_CUDA = 2,     /* a CUDA runtime call failed (message: qesb_last_error) */
  QESB_ERR_NOMEM = 3,    /* device allocation failed */
  QESB_ERR_STATE = 4,    /* call out of order (e.g. solve before set_inputs) */
  QESB_ERR_NUMERIC = 5,  /* NaN or Inf met in lambda during the solve */
  QESB_ERR_NODEV = 6     /* no CUDA device, or not an sm_100 device */
} qesb_status;

typedef struct qesb_handle qesb_handle;

/* Grid: base cell counts and spacings, as qes::Domain(Nx, Ny, Nz, dx, dy, dz)
 * takes them (src/qes/Domain.cpp:7-31), plus the vertical spacing array
 * (Domain::dz_array, src/qes/Domain.h:191), nz-1 = Nz+1 entries. */
typedef struct qesb_grid {
  int Nx, Ny, Nz;
  float dx, dy;
  const float *dz_array;
} qesb_grid;

/* Per-solve report. */
typedef struct qesb_stats {
  int iterations;        /* SOR iterations performed (the reference's `iter`) */
  int converged;         /* 1 if the stop came from max|dlambda| <= tol, 2 if from the window
                            rule (qesb_set_window_rule), 0 if from itermax */
  double residual;       /* FP64 max|lambda - lambda_old| of the last iteration */
  double ms_total;       /* device time of the whole solve (CUDA events) */
  double ms_sor;         /* device time of the SOR iterations alone */
  int path;              /* 0 = full-coefficient sweep, 1 = packed wall-mask sweep */
  int sweeps_per_launch; /* iterations fused per sweep launch */
  int launches;          /* kernels this solve launched (including polls and early exits) */
  int pre_iterations;    /* iterations of the over-relaxed pre-phase (qesb_set_prephase), its start
                            stage (qesb_set_prephase_start) included; 0 if none */
  double max_divergence; /* final check, in FP64: max |du/dx + dv/dy + dw/dz| over fluid cells
                            (icellflag 1), i in [1,nx-3], j in [1,ny-3], k in [1,nz-4], of the
                            corrected winds; -1 when the solve wrote no winds */
  double window_drift;   /* window rule: FP64 max|lambda - lambda(window iterations earlier)| at the
                            last window check; -1 when the rule is off or no window completed */
  double ms_sweeps;      /* device time of the sweep-kernel loops alone (pre-phase and reference loop,
                            CUDA events on the launching stream around them; a batch's loops for
                            every domain of the batch); -1 on the fused tile and full-coefficient paths */
} qesb_stats;

/* Library and device. */
const char *qesb_version(void);
const char *qesb_last_error(void);          /* thread-local message of the last failure */

/* Solver(qes::Domain, const float &tol) — src/winds/Solver.cpp:77-91 and
 * SolverFactory::create — src/winds/SolverFactory.cpp:35-60. Allocates the
 * device buffers for this grid on `device` (the reference always uses
 * device 0, Solver_GPU_GlobalMemory.cu:226). lambda starts at zero. */
qesb_status qesb_create(const qesb_grid *grid, float tol, int device, qesb_handle **out);
qesb_status qesb_destroy(qesb_handle *h);

/* Solver::resetLambda — src/winds/Solver.h:115-120: lambda, lambda_old, R <- 0. */
qesb_status qesb_reset_lambda(qesb_handle *h);

/* The WINDSGeneralData fields the solve reads (src/winds/Solver_CPU.cpp:56-231):
 * e f g h m n, icellflag, u0 v0 w0. Host pointers, copied to the device.
 * The coefficient arrays are inspected: when every updated cell's
 * coefficients are 0 or one per-layer value (stair-step walls, as
 * Wall::solverCoefficients leaves them) the sweep runs on a 1-byte wall mask
 * instead of six floats; otherwise on the full coefficients. */
qesb_status qesb_set_inputs(qesb_handle *h, const float *e, const float *f, const float *g,
                            const float *hc, const float *m, const float *n, const int *icellflag,
                            const float *u0, const float *v0, const float *w0);
/* The same inputs when the coefficients are the stair-step walls of the flag
 * field (the reference's default mesh: Wall::defineWalls then
 * Wall::solverCoefficients, src/winds/Wall.cpp:44-350): icellflag, u0, v0, w0
 * from the host (16 bytes per cell instead of 40), e..n computed from
 * icellflag on the device by the reference's rules, bit for bit what
 * Wall::solverCoefficients gives. Not for cut-cell coefficients (meshTypeFlag
 * 1) or coefficients read from a file: pass those to qesb_set_inputs. */
qesb_status qesb_set_inputs_flags(qesb_handle *h, const int *icellflag, const float *u0, const float *v0,
                                  const float *w0);
/* Same, from device pointers (reference layouts) already on the handle's device. */
qesb_status qesb_set_inputs_device(qesb_handle *h, const float *e, const float *f, const float *g,
                                   const float *hc, const float *m, const float *n,
                                   const int *icellflag, const float *u0, const float *v0,
                                   const float *w0);

/* Solver::solve(WGD, itermax) — src/winds/Solver_CPU.cpp:42-238:
 * R from u0 v0 w0; SOR red-black sweeps while (iter < itermax && max|dlambda| > tol)
 * with the ground mirror lambda(k=0) <- lambda(k=1) after each iteration;
 * then u v w = u0 v0 w0 + correction, zeroed on the faces of solid cells.
 * Host output pointers (nullable: skip that component). lambda persists on
 * the handle between calls, as in the reference CPU solvers, until
 * qesb_reset_lambda. */
qesb_status qesb_solve(qesb_handle *h, int itermax, float *u, float *v, float *w, qesb_stats *st);
/* Same, writing device pointers (reference face layout). */
qesb_status qesb_solve_device(qesb_handle *h, int itermax, float *u, float *v, float *w,
                              qesb_stats *st);

/* lambda in the reference cell layout (host pointers). set = warm start. */
qesb_status qesb_set_lambda(qesb_handle *h, const float *lambda);
qesb_status qesb_get_lambda(qesb_handle *h, float *lambda);
qesb_status qesb_get_divergence(qesb_handle *h, float *R);  /* R of the last solve */
/* FP64 max|dlambda| of each iteration of the last solve, iterations 0..n-1. */
qesb_status qesb_get_residual_history(qesb_handle *h, double *out, int n);

/* Runs n launches of the fused sweep kernel back to back on the current
 * inputs (no polls, no stop) and returns their total device time in *ms and
 * the iterations each launch fuses in *k. Advances lambda by n*k iterations;
 * meant for measuring the kernel alone. Requires stair-step inputs. */
qesb_status qesb_time_sweeps(qesb_handle *h, int n, float *ms, int *k);

/* Autotuner: times every sweep variant (fused tile shapes and split launch
 * shapes) for a few launches on this handle's inputs and keeps the fastest
 * for the handle's grid; the choice is cached for the process per grid shape
 * and used by later solves whose "variant" option is -1. lambda is restored
 * afterwards. us_per_iter (nullable, n_variants entries) receives each
 * variant's time per iteration; *best the chosen index. Needs stair-step
 * inputs (the full-coefficient path has a single variant). */
qesb_status qesb_autotune(qesb_handle *h, int *best, float *us_per_iter, int n_variants);
int qesb_num_variants(void);

/* Over-relaxed pre-phase (no reference counterpart; a warm start for the
 * reference loop). When omega is in (1, 2) and max_iterations > 0, each solve
 * on the packed sweep path first runs red-black SOR with this omega (same
 * kernels and FP64 rule, omega/sum and 1 - omega in place of the reference's
 * 1.78f, Solver_CPU_RB.cpp:118-125) from the current lambda until
 * max|dlambda| <= tol or max_iterations; then the reference loop runs as
 * always, with omega = 1.78 and the handle's tolerance, from that lambda. The
 * result therefore meets exactly the reference's stopping rule; only the
 * starting point differs. omega = 0 turns it off (the default). On the
 * packed path a set pre-phase runs on the sweep kernels (the fused tile
 * shapes have none); the full-coefficient path ignores it. */
qesb_status qesb_set_prephase(qesb_handle *h, float omega, float tol, int max_iterations);

/* Start stage of the pre-phase (no reference counterpart). With
 * iterations > 0 and a pre-phase set, each solve's pre-phase begins with
 * `iterations` red-black sweeps at this omega (in (0, 2); its own omega/sum
 * table and 1 - omega, no stop on the tolerance), then continues at the
 * pre-phase's omega until its tolerance. Over-relaxation near 2 from a rough
 * start first amplifies the start's rough error; a short stage at a smaller
 * omega damps it. qesb_stats.pre_iterations counts both parts; the reference
 * loop is unchanged. iterations = 0 turns it off (the default). */
qesb_status qesb_set_prephase_start(qesb_handle *h, float omega, int iterations);

/* Window stopping rule (no reference counterpart; a reachable stop for the
 * reference loop). The reference stops when one iteration changes lambda by at
 * most tol (Solver_CPU.cpp:93,129-143). In FP32 that change never falls below
 * the rounding flutter of lambda's largest values (10-15 ulp on the benchmark
 * cities), where the winds are still 1-5e-3 m/s from their converged values, so
 * a small tol is never met and a large one stops early. With window > 0 the
 * reference loop also stops, after every window-th iteration n, when
 *     max over all cells |lambda_n - lambda_(n - window)| <= tol   (FP64, exact)
 * a drift that keeps falling below the flutter. Iterations, the per-iteration
 * rule and itermax are unchanged; st->converged = 2 marks a window stop and
 * st->window_drift holds the last window's value. The pre-phase
 * (qesb_set_prephase) is not affected; the first window starts when the
 * reference loop does. Applies to qesb_solve/qesb_solve_device and
 * qesb_solve_batch (every handle of a batch must use the same window length);
 * the packed path then runs on the sweep kernels, not the fused tile shapes.
 * The first call with window > 0 allocates one lambda-sized buffer on the
 * handle. window = 0 turns the rule off (the default). */
qesb_status qesb_set_window_rule(qesb_handle *h, int window, double tol);

/* FP64 run of the same SOR (no reference counterpart; the precision check of
 * an FP32 result). On the handle's inputs, in double on the device: R, then
 * from lambda0 (host, cell layout, widened to double; NULL: zero)
 * pre_iterations red-black iterations of the pre-phase (0 for none): the
 * first min(pre_iterations, its start-stage count) at the handle's start-stage
 * omega when qesb_set_prephase_start set one, the rest at pre_omega; then
 * `iterations` at the reference's omega (1.78f as a double), the
 * ground mirror after each, with the reference's loop bounds and operation
 * order, no stopping rule; then the correction. Pass the counts a solve
 * reported (qesb_stats.pre_iterations, .iterations) to measure that solve's
 * FP32 rounding error: rep receives max|lambda - lambda64| over all cells
 * (lambda: the handle's current lambda), max|lambda64|, and, when u, v, w
 * (device face arrays, the FP32 winds of the solve) are given, the max over
 * all faces of |x - x64| for x = u, v, w (else -1), and the device ms of the
 * FP64 run. lambda64 (host, nullable, cell layout) receives the FP64 lambda.
 * Allocates two cell arrays of doubles for the call. */
typedef struct qesb_fp64_report {
  double lambda_max_abs_err;
  double lambda_max_abs;
  double wind_max_err;
  double ms;
} qesb_fp64_report;
qesb_status qesb_fp64_same_sor(qesb_handle *h, const float *lambda0, float pre_omega, int pre_iterations,
                               int iterations, const float *u, const float *v, const float *w, double *lambda64,
                               qesb_fp64_report *rep);

/* Batched solve (no reference counterpart: the reference solves one domain
 * per Solver::solve call, src/winds/Solver.h:108). Each of the n handles
 * holds one domain's inputs (qesb_set_inputs / qesb_set_inputs_device, on
 * the packed stair-step path) and its starting lambda; all are solved
 * together by persistent bulk-staged red/black launches in CUDA-graph
 * chunks, each domain stopping on its own loop condition
 * (Solver_CPU_RB.cpp:106) and leaving the launches' work list as soon as it
 * does. Results are those of n qesb_solve_device calls, bit for bit: lambda
 * stays in each handle; u[i], v[i], w[i] (device pointers, each array
 * nullable) receive domain i's corrected winds. st[i] (nullable array): as
 * for qesb_solve, with ms_sor = device time from the start of the batch's
 * iterations (pre-phase included) to the poll that ended domain i, ms_total =
 * the whole batch. All handles on one
 * device; the work runs on handles[0]'s stream, whose "variant" option picks
 * the bulk launch shape when it names one. */
qesb_status qesb_solve_batch(qesb_handle *const *handles, int n, int itermax, float *const *u,
                             float *const *v, float *const *w, qesb_stats *st);

/* Log-law wall treatment after a solve, replacing the call
 * WGD->wall->wallLogBC(WGD, true) that qesWindsMain.cpp:157-166 makes when
 * logLawFlag = 1 (src/winds/Wall.cpp:352-803), for stair-step walls: u, v, w
 * (device face arrays, nx*ny*nz each, typically the winds qesb_solve_device
 * just wrote) are changed in place on the faces of fluid cells next to solid
 * ones, side by side in the reference's order (below, above, back, front,
 * right, left). z0 is WINDSGeneralData::z0 (roughness length, m); dz is the
 * Domain's nominal dz (Domain::getDomainSize, Domain.h:104), whose first value
 * (dx) the reference uses for the x and the y walls alike, as here. Runs on the
 * handle's stream and returns when done; its first call on a handle allocates
 * a byte per cell for the wall sides. Cells flagged 7 or 8 (cut cells, whose
 * walls the first part of wallLogBC treats) make it return QESB_ERR_STATE
 * without changing u, v, w. Results agree with the reference to float
 * rounding of atan2, cos and sin (the rest is the reference's arithmetic). */
qesb_status qesb_wall_log_law(qesb_handle *h, float z0, float dz, float *u, float *v, float *w);

/* Workspace files (NetCDF classic, 64-bit offsets): the fields of the solve's
 * path with the dimension and variable names, layouts and attributes of the
 * reference's workspace output (src/winds/WINDSOutputWorkspace.cpp:40-154):
 * t(t); x_face, y_face, z_face, x, y, z; u, v, w, u0, v0, w0 (t, z_face, y_face,
 * x_face); dz_array(z); icellflag, e, f, g, h, m, n (t, z, y, x), one record.
 * netCDF-C reads the file like any NetCDF file. Host arrays in the reference
 * layouts. */
qesb_status qesb_workspace_write(const char *path, const qesb_grid *grid, double t, const float *u, const float *v,
                                 const float *w, const float *u0, const float *v0, const float *w0,
                                 const int *icellflag, const float *e, const float *f, const float *g,
                                 const float *h, const float *m, const float *n);
/* Grid of a workspace file (classic CDF-1 or CDF-2; NetCDF-4 files are
 * refused with the conversion to use): base counts from the x, y, z
 * dimensions, dx and dy (nullable) from the cell-centre coordinates. */
qesb_status qesb_workspace_dims(const char *path, int *Nx, int *Ny, int *Nz, float *dx, float *dy);
/* Reads a workspace's fields (record 0) into host arrays, any of which may be
 * NULL; numeric types are converted. The role of the reference's coefficient
 * re-read (src/winds/WINDSGeneralData.cpp:880-910), whole arrays. */
qesb_status qesb_workspace_read(const char *path, int Nx, int Ny, int Nz, float *dz_array, int *icellflag,
                                float *e, float *f, float *g, float *h, float *m, float *n, float *u0, float *v0,
                                float *w0, float *u, float *v, float *w);

/* Batch autotuner: times every sweep launch shape on the domain list that
 * qesb_solve_batch would run for these handles (same checks), a few launches
 * each from the handles' current lambda, and stores the fastest as
 * handles[0]'s "batch_variant" option, which qesb_solve_batch then uses.
 * lambda is left unchanged (the sweeps advance the split-layout copy only).
 * us_per_iter (nullable, n_variants entries) receives each shape's time per
 * iteration over the whole list, at its variant index (entries below the
 * first sweep shape are left untouched); *best the chosen index. */
qesb_status qesb_autotune_batch(qesb_handle *const *handles, int n, int *best, float *us_per_iter, int n_variants);

/* Tolerance (Solver::tol) and tuning knobs. Keys:
 *   "sweeps_per_launch"  iterations fused per sweep launch (0 = autotuned)
 *   "path"               0 = force full coefficients, 1 = allow the packed mask (default)
 *   "graph"              1 = run the iteration loop as a CUDA graph (default), 0 = plain launches
 *   "pdl"                1 = z-march list sweeps and window checks as programmatic dependent launches,
 *                        each grid's CTAs scheduled while the previous grid finishes; 0 = off (default:
 *                        inside the CUDA-graph chunks it measured 0.6 % slower on the headline batch)
 *   "variant"            sweep variant index (-1 = autotuned / default), see qesb_num_variants
 *   "batch_variant"      sweep shape for qesb_solve_batch led by this handle (-1 = from "variant");
 *                        set by qesb_autotune_batch
 *   "autotune"           1 = run qesb_autotune at the first solve of an untuned grid shape (default 0)
 *   "wait_limit"         polls of a staged sweep's shared-memory stage barrier before the kernel gives
 *                        up, lets its copies in flight land, and the solve returns QESB_ERR_CUDA
 *                        ("sweep stage wait gave up"); 0 = the default (2^22 polls). Applies to the
 *                        bulk-copy sweep shapes and to batches led by this handle */
qesb_status qesb_set_tolerance(qesb_handle *h, float tol);
qesb_status qesb_set_option(qesb_handle *h, const char *key, int value);
/* cudaStream_t to run on (NULL = the handle's own stream). */
qesb_status qesb_set_stream(qesb_handle *h, void *stream);
/* The stream the handle's work runs on (its own, or the one set): callers
 * that add work on the same data (the warm-start glue below) order it there. */
qesb_status qesb_get_stream(qesb_handle *h, void **stream);

/* ---------------------------------------------------------------------
 * Warm-start network (tensor-core kernels).
 * --------------------------------------------------------------------- */
/* Handle-side glue of the warm start (device pointers, the handle's stream).
 * The network grid is planes 0..Nz-1 of the X x Y cell grid (all but the top
 * boundary plane), channels-last [Nz][Ny][Nx][C] BF16.
 *   qesb_compute_divergence: R from the current inputs (as a solve does first).
 *   qesb_warm_input:  network input from R, icellflag and dz (C a multiple of
 *                     8, >= 8; channels R/s, solid, dz/mean dz, boundary,
 *                     height fraction, then zeros);
 *                     *scale (device) receives s = max|R| over updated cells.
 *   qesb_warm_target: lambda/s and a 1/0 weight (updated cells) per voxel, FP32.
 *   qesb_warm_apply:  lambda <- s * yhead[v][0] on updated cells (yhead FP32
 *                     [V][N]), 0 elsewhere, ground plane mirrored: the next
 *                     qesb_solve starts from it. */
qesb_status qesb_compute_divergence(qesb_handle *h);
qesb_status qesb_warm_input(qesb_handle *h, void *x, int C, unsigned *scale);
/* qesb_warm_input followed by a 2x2x2 average (qesb_net_pool2), bit for bit,
 * in one pass: the input of a network run at half resolution, on the
 * (Nz/2) x (Ny/2) x (Nx/2) grid (even sizes). */
qesb_status qesb_warm_input_half(qesb_handle *h, void *x, int C, unsigned *scale);
qesb_status qesb_warm_target(qesb_handle *h, float *tgt, float *w, const unsigned *scale);
qesb_status qesb_warm_apply(qesb_handle *h, const float *yhead, int N, const unsigned *scale);
/* qesb_warm_apply for a network run at half resolution: yhead on the
 * (Nz/2) x (Ny/2) x (Nx/2) grid (even sizes), interpolated trilinearly to
 * the cell centres. */
qesb_status qesb_warm_apply_up2(qesb_handle *h, const float *yhead, int N, const unsigned *scale);

/* The learned warm start as one call (no reference counterpart; the reference
 * starts every solve from lambda = 0 after resetLambda, qesWindsMain.cpp:154).
 * qesb_warmnet_load reads a trained network (the "QESBWNT1" weights file that
 * qes-public_b200/qesb/warmstart.py writes: levels, resolution, channels, then
 * each layer's FP32 weights and bias) onto `device`, converting the weights to
 * the convolution kernels' BF16 layout. qesb_warm_start runs it for handle
 * h's current inputs on h's stream: R, the network input (R / max|R|, solid
 * flag, dz, boundary flag, height), the forward pass (BF16 tcgen05
 * convolutions, FP32 accumulation), and lambda <- max|R| * prediction on the
 * updated cells (trilinear from the half-resolution grid when the network
 * runs at res 2), ground plane mirrored; the next solve on h starts from it.
 * The grid's Nx, Ny and Nz must be multiples of res * 2^(levels-1). The first
 * call for a grid shape allocates that shape's activations on the network
 * (kept until qesb_warmnet_destroy); calls on one network are serialised. It
 * returns when the start is in place (QESB_ERR_CUDA if a tensor-core wait gave
 * up). */
typedef struct qesb_warmnet qesb_warmnet;
qesb_status qesb_warmnet_load(const char *path, int device, qesb_warmnet **out);
qesb_status qesb_warmnet_destroy(qesb_warmnet *net);
qesb_status qesb_warm_start(qesb_handle *h, qesb_warmnet *net);
/* qesb_warm_start for n handles of one grid shape at once: their network
 * inputs stacked along z (qesb_conv3d_items), one launch per layer for all of
 * them, each start the one qesb_warm_start would give. Each handle's input
 * and apply run on its own stream, ordered with the forward pass on handle
 * 0's stream by an event; returns when every start is in place. */
qesb_status qesb_warm_start_batch(qesb_handle *const *hs, int n, qesb_warmnet *net);

/* Self-test of the tcgen05 GEMM core: C[128 x N] = A[128 x K] * B[N x K]^T
 * in BF16 with FP32 accumulation. A is [128][K] (a_mn = 0) or [K][128]
 * (a_mn = 1); B is [N][K] (b_mn = 0) or [K][N] (b_mn = 1); BF16 bit patterns,
 * host pointers. N a multiple of 16 in [16, 256], K a multiple of 64. */
qesb_status qesb_umma_selftest(const uint16_t *A, const uint16_t *B, float *C, int N, int K, int a_mn,
                               int b_mn);

/* 3x3x3 convolution (zero padding, stride 1) as an implicit GEMM on the
 * tensor cores; all pointers are device pointers, activations channels-last
 * BF16 [D][H][W][C]. Input = channel concatenation of x1 (c1 channels; at
 * (D/2, H/2, W/2) read through x2 nearest upsampling when up1) and x2 (c2
 * channels, nullable when c2 = 0); c1, c2 multiples of 16. sign = +1 reads
 * taps at v + offset (forward), -1 at v - offset (input gradient). Bm is the
 * weight matrix [N][Kp] BF16, k = tap*(c1+c2) + c, Kp = roundup(27*(c1+c2), 64)
 * zero-padded; tap = (dz+1)*9 + (dy+1)*3 + (dx+1). Output [D][H][W][N] to y
 * (BF16) or yf (FP32); optional bias[N] (FP32), ReLU, and mask (BF16 [V][N]:
 * output zeroed where mask <= 0). N in {16, 32, 64, 128}. *err is set if a
 * kernel's tensor-core completion wait gives up. Grids with W a multiple of
 * 128 and N in {16, 32} run direct kernels (the 27 taps as shifted
 * descriptors into staged input rows): forward convolutions of one 16-channel
 * input without mask march along z, each input plane staged once by
 * tensor-map copies; the others stage each 16-channel slice once per tile.
 * The remaining grids run the implicit GEMM (per-tap gather). Small grids (fewer than about two
 * 128-voxel tiles per SM) split the K chunks over more CTAs and add FP32
 * partial sums in a scratch buffer kept per (device, stream), one slice per
 * split, allocated on the first such call on a stream and grown as needed (a
 * few MB for the network's deep levels); the slices are added in a fixed
 * order, so every call gives the same bits. */
qesb_status qesb_conv3d(const void *x1, int c1, int up1, const void *x2, int c2, int D, int H, int W,
                        int sign, const void *Bm, int Kp, int N, void *y, void *yf, const float *bias,
                        int relu, const void *mask, int *err, void *stream);
/* The same over `items` grids of D x H x W stacked along z (activations
 * [items * D][H][W][C]; x1 under up1 [items * D/2][H/2][W/2][c1]): one launch
 * for all of them, taps never reaching from one item into the next, so each
 * item's output is qesb_conv3d's on that item alone. D even when items > 1. */
qesb_status qesb_conv3d_items(const void *x1, int c1, int up1, const void *x2, int c2, int items, int D,
                              int H, int W, int sign, const void *Bm, int Kp, int N, void *y, void *yf,
                              const float *bias, int relu, const void *mask, int *err, void *stream);
/* Process-wide choice of the qesb_conv3d kernel: 0 = the default: forward
 * convolutions without mask on rows of 128 (or a multiple), 64 or 32 voxels
 * run the z-marching kernel (input planes staged once by tensor-map copies,
 * copies, MMAs and read-out of different planes overlapping on their own
 * warps; concatenated inputs; an upsampled input first written on the output
 * grid; split over input channels when the weights and planes do not fit one
 * CTA), with three output planes per MMA up to 32 output channels; else the
 * direct kernel where it applies; else the implicit GEMM. 1 = implicit GEMM
 * everywhere, 2 = the direct kernel, else the implicit GEMM, 3 / 4 = the
 * z-marching kernel for one 16-channel input only, 2 / 4 output rows per CTA,
 * 5 = as 3 with a four-stage implicit GEMM, 6 = as 0 with one output plane per
 * MMA - for comparison. */
qesb_status qesb_net_set_conv_path(int path);
/* Weight gradient dW[tap*(c1+c2) + c][n] += sum_v X[v + offset(tap)][c] * dY[v][n]
 * (FP32, accumulated with atomics: zero it first); X as in qesb_conv3d,
 * dY BF16 [V][N]; vchunk = voxels per CTA (>= 64). */
qesb_status qesb_conv3d_wgrad(const void *x1, int c1, int up1, const void *x2, int c2, int D, int H,
                              int W, const void *dY, int N, long vchunk, float *dW, int *err,
                              void *stream);

/* Elementwise kernels of the network (device pointers; BF16 activations
 * channels-last; FP32 gradients where named float). */
qesb_status qesb_net_pool2(const void *x, void *y, int D, int H, int W, int C, void *stream);
/* 2x2x2 average of an FP32 scalar field [D][H][W] (even sizes). */
qesb_status qesb_net_pool2_f32(const float *x, float *y, int D, int H, int W, void *stream);
qesb_status qesb_net_skip_grad(const float *gcat, int ccat, int coff, const float *gpool, const void *e,
                               void *ge, int D, int H, int W, int C, void *stream);
qesb_status qesb_net_up_grad(const float *gcat, int ccat, const void *x, void *gx, int D, int H, int W,
                             int C, void *stream);
qesb_status qesb_net_to_bf16(const float *g, const void *mask, void *out, long n, void *stream);
qesb_status qesb_net_colsum(const void *g, long V, int C, float *db, void *stream);
qesb_status qesb_net_mse(const float *yhead, int N, const float *tgt, const float *w, long V,
                         float inv_count, void *g, double *loss, void *stream);
/* Adds a low-frequency term: the weighted error averaged over F^3 blocks,
 * beta * mean(block error^2), to *loss and its gradient to g (channel 0). */
qesb_status qesb_net_mse_coarse(const float *yhead, int N, const float *tgt, const float *w, int D,
                                int H, int W, int F, float beta, void *g, double *loss, void *stream);
qesb_status qesb_net_adam_conv(float *Wt, float *m, float *v, const float *dW, int cin, int cout,
                               int cout_real, void *Bm, int Kp, void *Bd, int Kd, float lr, float b1,
                               float b2, float eps, int step, float grad_scale, void *stream);
qesb_status qesb_net_adam_vec(float *p, float *m, float *v, const float *g, int n, float lr, float b1,
                              float b2, float eps, int step, float grad_scale, void *stream);

/* ---------------------------------------------------------------------
 * Solve without allocating. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code whose device memory is all
 * owned by another allocator (a framework's caching allocator holding the
 * GPU, a host with a fixed device-memory budget) and long-running coupling
 * loops that must not allocate or free once started (an allocation costs a
 * device synchronisation and can fragment memory). This entry point neither
 * creates a handle nor allocates: its scratch (solve state, per-iteration
 * residuals, dz, R) lives in one file-scope device array of
 * QESB_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * the process exits. That caps the grid at QESB_NOALLOC_MAX_CELLS cells
 * (Nx*Ny*(Nz+1)), QESB_NOALLOC_MAX_Z layers and QESB_NOALLOC_MAX_ITERS
 * iterations; larger requests return QESB_ERR_ARG with the limits in
 * qesb_last_error().
 *
 * Same semantics and bits as qesb_solve_device on the full-coefficient
 * red-black sweep: inputs e..n, icellflag, u0 v0 w0, lambda and the outputs
 * u v w are DEVICE pointers in the reference layouts; lambda is read as the
 * starting point and left holding the result (the caller keeps it between
 * calls, as Solver keeps its lambda); dz_array in `grid` is a host pointer.
 * Runs on `stream` (NULL: the legacy default stream) and returns when done.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. Every call shares the one array and resets the
 * parts that must start at zero, so calls that overlap on the GPU (other
 * streams, other host threads) race and must not be issued. st (nullable)
 * gets iterations, convergence and residual; its times are 0.
 * --------------------------------------------------------------------- */
#define QESB_NOALLOC_SCRATCH_BYTES (32u << 20)
#define QESB_NOALLOC_MAX_ITERS 16384
#define QESB_NOALLOC_MAX_Z 1024
#define QESB_NOALLOC_MAX_CELLS \
  ((QESB_NOALLOC_SCRATCH_BYTES - 256u - 8u * QESB_NOALLOC_MAX_ITERS - 4u * QESB_NOALLOC_MAX_Z) / 4u)

qesb_status qesb_solve_noalloc(const qesb_grid *grid, float tol, int itermax, const float *e,
                               const float *f, const float *g, const float *hc, const float *m,
                               const float *n, const int *icellflag, const float *u0,
                               const float *v0, const float *w0, float *lambda, float *u, float *v,
                               float *w, void *stream, qesb_stats *st);

/* ---------------------------------------------------------------------
 * Seeded synthetic-city generator (host). Restates the reference's set-up of
 * the solver inputs for flat terrain and stair-step cuboid buildings:
 *   ground flags      src/winds/WINDSGeneralData.cpp:438-444
 *   building cells    src/winds/PolyBuilding.cpp:130-237 (RectangularBuilding.h:70-108)
 *   wall coefficients src/winds/Wall.cpp:44-350, 827-846
 *   power-law inflow  src/winds/WindProfilerSensorType.cpp:220,328-333,571-621
 *   solid faces       src/winds/Wall.cpp:805-825
 * --------------------------------------------------------------------- */
typedef struct qesb_building {
  float x_start, y_start;   /* south-west corner, m */
  float length, width;      /* extent along x and y, m */
  float height, base_height;
} qesb_building;

typedef struct qesb_inflow {
  float u_ref;    /* speed at z_ref, m/s */
  float z_ref;    /* m */
  float p;        /* power-law exponent (the reference carries it in siteZ0) */
  float dir_deg;  /* meteorological direction; 270 blows toward +x */
} qesb_inflow;

/* dz_array for a uniform (ratio == 1) or geometrically stretched grid:
 * dz[k] = dz0 * ratio^(k-1) for k >= 1, dz[0] = dz[1]. */
qesb_status qesb_city_dz(int Nz, float dz0, float ratio, float *dz_array);

/* Fill icellflag, e..n and u0 v0 w0 for the given buildings and inflow. */
qesb_status qesb_city_build(const qesb_grid *grid, int n_buildings, const qesb_building *b,
                            const qesb_inflow *inflow, int *icellflag, float *e, float *f,
                            float *g, float *hc, float *m, float *n, float *u0, float *v0,
                            float *w0);

/* qesb_city_build on the device: the same icellflag, e..n, u0, v0, w0, bit for
 * bit, written by kernels into device arrays (reference layouts) on `stream`
 * (NULL: the default stream). The building list and inflow are host inputs;
 * the vertical grid, each building's cell box and layer range, and the
 * power-law profile are evaluated on the host as qesb_city_build does, the
 * per-cell and per-face work on the device. Returns once the arrays are
 * written. Restates the same reference steps as qesb_city_build. */
qesb_status qesb_city_build_device(const qesb_grid *grid, int n_buildings, const qesb_building *b,
                                   const qesb_inflow *inflow, int *icellflag, float *e, float *f, float *g,
                                   float *hc, float *m, float *n, float *u0, float *v0, float *w0,
                                   void *stream);

/* Only the initial winds of qesb_city_build for another inflow over the same
 * icellflag (power-law profile, then the solid faces zeroed): a wind-direction
 * ensemble rebuilds no walls. */
qesb_status qesb_city_inflow(const qesb_grid *grid, const int *icellflag, const qesb_inflow *inflow, float *u0,
                             float *v0, float *w0);

/* Seed-indexed random city: up to max_buildings non-overlapping cuboids with
 * footprints U[fp_min, fp_max] m, heights U[h_min, h_max] m, and a random
 * inflow (u_ref U[3,10] m/s at 10 m, p U[0.1,0.3], direction U[0,360)).
 * Writes the buildings and inflow chosen; returns the count in *n_out. */
qesb_status qesb_city_random(const qesb_grid *grid, uint64_t seed, int max_buildings,
                             float fp_min, float fp_max, float h_min, float h_max,
                             qesb_building *b_out, int *n_out, qesb_inflow *inflow_out);

#ifdef __cplusplus
}
#endif
#endif /* QESB_H */

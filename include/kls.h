/*
 * kls.h - C ABI of libkls.so, the B200 (sm_100a) implementation of the
 * Kalnajs log-spiral matrix-method eigenvalue path:
 *
 *   orbit integration -> W_l(alpha) table + N_m(alpha) -> M(omega) contraction
 *   -> det(I - M(omega)) -> omega-plane scan / Newton root (Omega_p, gamma).
 *
 * Every entry point returns an int status (KLS_OK = 0).  The library owns all
 * device memory; the caller owns host buffers.  Host arrays exported in
 * "reference layout" use the reference's Julia column-major order.
 *
 * Threading: one context per device per host thread.  A context is not
 * re-entrant; distinct contexts are independent.
 *
 * Reference interfaces replaced (paths inside epolyach/Kalnajs_log_spirals):
 *   KalnajsConfig / load_config     src/KalnajsLogSpiral/Configuration.jl:139-261
 *   create_toomre_zang_model        src/KalnajsLogSpiral/Models.jl:40-57
 *   precompute_all + to_device      src/KalnajsLogSpiral/BasisFunctions.jl:73-165, 397-437
 *   compute_determinant(_batched)   src/KalnajsLogSpiral/MatrixBuilder.jl:197-239
 *   build_M_matrix                  src/KalnajsLogSpiral/MatrixBuilder.jl:242-244
 *   grid_scan / find_minimum        src/KalnajsLogSpiral/GridScan.jl:25-88, 234-246
 *   newton_search / NewtonResult    src/KalnajsLogSpiral/NewtonSolver.jl:19-172
 */
#ifndef KLS_H
#define KLS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define KLS_OK               0
#define KLS_ERR_CONFIG       1  /* invalid configuration / argument          */
#define KLS_ERR_CUDA         2  /* a CUDA runtime call failed                 */
#define KLS_ERR_OOM          3  /* device allocation failed                   */
#define KLS_ERR_STATE        4  /* call order (e.g. det before precompute)    */
#define KLS_ERR_NONFINITE    5  /* non-finite value in an input or result     */
#define KLS_ERR_SINGULAR     6  /* singular 2x2 Newton Jacobian               */
#define KLS_ERR_UNSUPPORTED  7  /* mode not available on this device          */
#define KLS_ERR_TIMEOUT      8  /* a bounded device-side wait ran out: the
                                   contraction pipeline stalled; the call's
                                   results are invalid, the context stays usable */

/* ---- precision modes of the contraction -------------------------------- */
#define KLS_MODE_FP64        0  /* plain FP64 (the oracle form)               */
#define KLS_MODE_MIXED       1  /* split-BF16 tensor-core contraction, FP32
                                   accumulation; FP64 weights/LU              */
#define KLS_MODE_ANCHORED    2  /* M(omega) = M(omega_a) + dM: the FP64 M at
                                   the anchor set by kls_set_anchor plus the
                                   split-BF16 contraction of the weight
                                   differences w_k(omega) - w_k(omega_a).
                                   dM is ~|omega - omega_a| / gamma of M, so
                                   near the anchor its split-BF16 error is that
                                   fraction of the split form's (1e-6 of omega
                                   away: ~1e-11 of max|M|) at the cost of a
                                   KLS_MODE_MIXED evaluation                  */

/* ---- forms of the FP64 contraction (kls_set_f64_form) -------------------- */
#define KLS_F64_4M           0  /* four real DMMA products per complex one     */
#define KLS_F64_3M           1  /* three (Gauss): Re = P1 - P2,
                                   Im = (P3 - P1) - P2 with P3 = (ar+ai)(br+bi) */

/* ---- configuration: the [physics] [model] [grid] TOML sections ---------- *
 * Mirrors PhysicsConfig / ModelConfig / GridConfig
 * (Configuration.jl:31-67).  q1 is real-valued here (the reference types it
 * Int, Configuration.jl:42); integer values reproduce the reference.        */
typedef struct kls_config {
    int32_t m;          /* azimuthal number                                 */
    double  G;          /* gravitational constant                           */
    double  L0;         /* taper angular-momentum scale                     */
    int32_t n_zang;     /* taper exponent                                   */
    double  q1;         /* dispersion parameter, q = q1 - 1                 */
    int32_t NR;         /* guiding-centre radii                             */
    int32_t Ne;         /* circulation (v) points                           */
    double  Rc_min, Rc_max, v_min;
    int32_t N_alpha;    /* log-spiral alpha points on [-alpha_max, alpha_max]*/
    double  alpha_max;
    int32_t l_min, l_max;  /* radial harmonics                              */
    int32_t nw;         /* orbit integration points                          */
    int32_t nwa;        /* stored (subsampled) orbit points                  */
    /* Quadrature rules of the alpha, ln Rc and v grids (KLS_QUAD_*), the
     * --quad=alpha-Rc-v option of NL_julia_boole.jl:14-16, 221-249.  0 keeps
     * the package's rules (trapezoid, trapezoid, Simpson).                  */
    int32_t quad_alpha, quad_rc, quad_v;
} kls_config;

#define KLS_QUAD_DEFAULT     0
#define KLS_QUAD_TRAPEZOID   1
#define KLS_QUAD_SIMPSON     2  /* falls back to the trapezoid rule for even n */
#define KLS_QUAD_BOOLE       3  /* n = 4k + 1 points, else the Simpson rule   */

/* Dimensions derived from a config (and device padding). */
typedef struct kls_dims {
    int32_t NPh;        /* NR * Ne                                          */
    int32_t n_l;        /* l_max - l_min + 1                                */
    int32_t N_alpha;
    int32_t N_alpha_pad;/* row length of the device W table                 */
    int64_t K;          /* NPh * n_l contraction length                     */
    int64_t K_pad;      /* padded rows of the device W table                */
    int32_t nwa;
    int64_t device_bytes; /* device memory held by the context             */
} kls_dims;

/* Newton parameters: NewtonConfig (Configuration.jl:84-100). */
typedef struct kls_newton_cfg {
    int32_t max_iter;
    double  tol;
    double  delta;
    int32_t use_line_search;
    int32_t max_line_search;
    int32_t mode;          /* KLS_MODE_* used for every det evaluation        */
} kls_newton_cfg;

/* NewtonResult (NewtonSolver.jl:19-27). */
typedef struct kls_newton_result {
    double  Omega_p;
    double  gamma;
    double  omega_re, omega_im;
    double  det_re, det_im;
    int32_t iterations;
    int32_t converged;
    int32_t det_evals;     /* determinant evaluations performed               */
} kls_newton_result;

/* Grid-scan parameters: ScanConfig (Configuration.jl:72-79). */
typedef struct kls_scan_cfg {
    int32_t n_Op, n_gamma;
    double  Omega_p_min, Omega_p_max;
    double  gamma_min, gamma_max;
    int32_t mode;
    int32_t batch;         /* omegas per device launch (<=0: library choice)  */
} kls_scan_cfg;

typedef struct kls_ctx kls_ctx;

/* ---- lifecycle ---------------------------------------------------------- */
/* Replaces create_toomre_zang_model + the device selection of to_device.
 * The configuration is checked before the device is touched
 * (KLS_ERR_CONFIG): the reference's own (nw, nwa) DimensionMismatch, and the
 * sizes this library supports: NR * Ne < 2^31, NPh * n_l <= 4e9 and
 * N_alpha <= 7168 (the LU keeps two rows of N_alpha complex values in one
 * CTA's shared memory). */
int kls_create(const kls_config* cfg, int device, kls_ctx** out);
int kls_destroy(kls_ctx* ctx);
/* Message of the last failing call on this context (never NULL). */
const char* kls_last_error(const kls_ctx* ctx);
/* Message for failures of calls without a context (kls_create,
 * kls_det_lu_static). */
const char* kls_create_error(void);
/* Sizes of the context's data: the NPh, n_l and N_alpha fields of
 * PrecomputedData (BasisFunctions.jl:30-60), the padded device sizes and the
 * device memory the context holds. */
int kls_get_dims(const kls_ctx* ctx, kls_dims* out);
/* Launch subsequent work on this cudaStream_t (NULL = the context's own). */
int kls_set_stream(kls_ctx* ctx, void* cuda_stream);

/* ---- omega-independent stage: precompute_all + to_device ---------------- *
 * Grids, orbit integration, Jacobian + DF, W_l table, N_m(alpha), DJ, F0l,
 * Omega_res; all on the device, table device-resident (BasisFunctions.jl:73). */
int kls_precompute(kls_ctx* ctx);
/* Build the split-BF16 copy of the W table used by KLS_MODE_MIXED.         */
int kls_prepare_mixed(kls_ctx* ctx);
/* Free the FP64 W table after building the split-BF16 copy (no reference
 * counterpart): a mixed-only context, 13 GB instead of 40 GB at NR=501,
 * Ne=51, N_alpha=301, l in [-100, 100], so that many default-size models fit
 * one GPU.  Afterwards KLS_MODE_FP64 calls, kls_export_W and FP64 batches
 * return KLS_ERR_STATE.                                                     */
int kls_release_fp64(kls_ctx* ctx);

/* ---- exports in reference layout (host, column-major) ------------------- *
 * Omega_1/Omega_2/jacobian/F0/FE/FL/DJ: [NR, Ne]; w1/ra/pha: [nwa, NR, Ne]
 * (OrbitIntegration.jl:43-54); any pointer may be NULL to skip it.         */
int kls_export_orbits(kls_ctx* ctx, double* Omega_1, double* Omega_2,
                      double* jacobian, double* F0, double* FE, double* FL,
                      double* DJ, double* w1, double* ra, double* pha);
/* Grids (OrbitIntegration.jl:26-38): each [NR, Ne] except S_RC [NR].      */
int kls_export_grids(kls_ctx* ctx, double* Rc, double* e, double* E,
                     double* L_m, double* S_RC, double* S_e);
/* alpha, d_alpha, N_kernel: [N_alpha] (BasisFunctions.jl:106-121).         */
int kls_export_alpha(kls_ctx* ctx, double* alpha, double* d_alpha, double* N_kernel);
/* F0l, Omega_res: [NPh, n_l] (BasisFunctions.jl:139-153).                  */
int kls_export_resonant(kls_ctx* ctx, double* F0l, double* Omega_res);
/* W_l_mat [NPh, N_alpha, n_l] complex (interleaved re,im), restricted to the
 * harmonics [il0, il0+nl) to bound host memory (BasisFunctions.jl:55-56).  */
int kls_export_W(kls_ctx* ctx, int il0, int nl, double* W_ri);

/* ---- hot path ----------------------------------------------------------- */
/* compute_determinant for n omegas (interleaved re,im), one batched launch
 * sequence; det_ri interleaved re,im; log_abs = log|det| (may be NULL).
 * Host buffers in, host buffers out (MatrixBuilder.jl:197-239).  A NaN
 * determinant (a non-finite table row or weight) returns KLS_ERR_NONFINITE. */
int kls_det_batch(kls_ctx* ctx, const double* omega_ri, int n, int mode,
                  double* det_ri, double* log_abs);
/* compute_determinant for one omega (MatrixBuilder.jl:197): det_re, det_im
 * and log_abs (may be NULL); the same launch sequence as a batch of one.   */
int kls_det(kls_ctx* ctx, double omega_re, double omega_im, int mode, double* det_re,
            double* det_im, double* log_abs);
/* Same with device buffers on the context's stream; no host synchronisation.*/
int kls_det_batch_device(kls_ctx* ctx, const double* d_omega_ri, int n, int mode,
                         double* d_det_ri, double* d_log_abs);
/* M(omega) [N_alpha, N_alpha] complex column-major (MatrixBuilder.jl:242).  */
int kls_build_M(kls_ctx* ctx, double omega_re, double omega_im, int mode, double* M_ri);
/* Anchor of KLS_MODE_ANCHORED (no reference counterpart): one FP64
 * evaluation at omega_a that keeps M(omega_a) on the device (N_alpha^2
 * complex) and returns det(I - M(omega_a)) in det_ri (may be NULL).  Needs
 * the FP64 table (KLS_ERR_STATE after kls_release_fp64) and builds the
 * split-BF16 table if it is missing.  A later call moves the anchor.       */
int kls_set_anchor(kls_ctx* ctx, double omega_re, double omega_im, double* det_ri);

/* grid_scan (GridScan.jl:25-88): det_grid [n_gamma, n_Op] column-major
 * complex; argmin of |det| in column-major order (GridScan.jl:234-246).   */
int kls_scan(kls_ctx* ctx, const kls_scan_cfg* sc, double* det_grid_ri,
             double* log_abs_grid, double* Omega_p0, double* gamma0);

/* newton_search (NewtonSolver.jl:36-172).  history: (max_iter) x 3 row-major
 * (Omega_p, gamma, |det|) per iteration, may be NULL.                      */
int kls_newton(kls_ctx* ctx, double Omega_p0, double gamma0, const kls_newton_cfg* nc,
               kls_newton_result* res, double* history);

/* Mixed-precision Newton with an FP64-anchored finish (no reference
 * counterpart; it returns a point at which the reference's stopping rule
 * |det| < nc->tol holds on a determinant of FP64 accuracy).  det(I - M(omega))
 * is holomorphic in omega = m Omega_p + i gamma, so one complex slope S gives
 * the reference's whole 2x2 finite-difference Jacobian (dF/dOmega_p = m S,
 * dF/dgamma = i S) and the step is delta omega = -det / S.  Steps are
 * accepted as the reference accepts them (every step, no line search),
 * except that a step shorter than 1e-4 that does not lower |det| ends a
 * phase (the determinant's rounding decides such steps):
 *   phase 1: secant iteration on split-BF16 determinants.  The first slope
 *            is the forward difference of the pair (omega, omega + h),
 *            h = m*mixed_delta, evaluated as one batch; each later step's
 *            determinant gives the next secant slope.  While the Newton step
 *            is longer than far_step, steps of FP64 accuracy follow the
 *            reference's own path instead: det at an FP64 anchor and the
 *            slope by an anchored forward difference of step m * nc->delta.
 *            The phase ends when the next step is shorter than
 *            mixed_step_tol (taken without an evaluation), at the noise
 *            floor, or after mixed_max_iter + fp64_max_iter steps.
 *   phase 2: kls_set_anchor at the last point (one FP64 determinant), then
 *            KLS_MODE_ANCHORED determinants (FP64 accuracy near the anchor),
 *            secant steps starting with the phase-1 slope; a step beyond
 *            anchor_radius of the anchor moves the anchor (another FP64
 *            determinant) and is followed by a forward-difference slope.  A
 *            short step that does not lower |det| is retried once with a
 *            forward-difference slope.  The phase ends when |det| < tol and
 *            the next step is below 1e-11 (|det| < tol alone fixes the root
 *            only to tol / |det'|), when |det| < tol and stops falling, or
 *            after fp64_max_iter steps.  final_fp64 != 0 adds one plain FP64
 *            determinant at the result, which then decides `converged` and
 *            is the returned det.                                          */
typedef struct kls_hybrid_cfg {
    double  mixed_delta;
    double  mixed_step_tol;
    int32_t mixed_max_iter;
    int32_t fp64_max_iter;
    double  anchor_radius;
    int32_t final_fp64;
    double  far_step;
} kls_hybrid_cfg;
/* evals[0..2] (may be NULL): split-BF16, plain FP64 (anchors included) and
 * anchored determinant evaluations.                                        */
int kls_newton_hybrid(kls_ctx* ctx, double Omega_p0, double gamma0, const kls_newton_cfg* nc,
                      const kls_hybrid_cfg* hc, kls_newton_result* res, int32_t* evals,
                      double* history);

/* Determinants of n_matrices caller-supplied complex N x N matrices (device
 * memory, row-major, interleaved re,im; the input is not modified) into
 * d_det_ri (n complex) and d_log_abs (n doubles, may be NULL), launched on
 * `stream` (NULL = legacy default stream); no host synchronisation.  No
 * counterpart in the reference.  It allocates nothing: it is for callers that
 * must not allocate device memory themselves, e.g. a host whose pool allocator
 * owns the whole GPU, or a loop that cannot take cudaMalloc's implicit device
 * synchronisation.  Scratch is a fixed 16 MiB array inside libkls.so (held on
 * every GPU that loads the library until exit), so n_matrices * N * N must not
 * exceed 1,048,576; larger requests return KLS_ERR_CONFIG.  The first call on
 * a device looks up the array's device address (make it before any stream
 * capture).  Calls whose kernels overlap on one GPU race on the shared
 * scratch.  Errors are described by kls_create_error().                    */
int kls_det_lu_static(const double* d_A_ri, int n_matrices, int N, double* d_det_ri,
                      double* d_log_abs, void* stream);

/* ---- learned root proposer (no reference counterpart) -------------------- *
 * MLP features (5) -> width (GELU) x (depth - 1) -> outputs (3), FP32 master
 * weights, BF16 tensor-core GEMMs with FP32 accumulation, Adam; trained and
 * run on the device by the library's own kernels.  Parameter order (flat
 * fp32): for each layer, W [out][in] row-major then b [out].               */
typedef struct kls_mlp kls_mlp;
int kls_mlp_create(int device, int width, int depth, uint64_t seed, kls_mlp** out);
int kls_mlp_destroy(kls_mlp* mlp);
int kls_mlp_num_params(const kls_mlp* mlp, int64_t* n);
int kls_mlp_get_params(kls_mlp* mlp, float* params);
int kls_mlp_set_params(kls_mlp* mlp, const float* params);
/* X [n][5] -> Y [n][3], host buffers. */
int kls_mlp_forward(kls_mlp* mlp, const float* X, int n, float* Y);
/* Mean-squared-error loss and its gradient (flat, params order) on one batch. */
int kls_mlp_grad(kls_mlp* mlp, const float* X, const float* T, int n, float* grads, float* loss);
/* Adam over shuffled minibatches; loss_hist[e] = mean minibatch loss of epoch e. */
int kls_mlp_train(kls_mlp* mlp, const float* X, const float* T, int n, int epochs, int batch,
                  float lr, uint64_t seed, float* loss_hist);

/* ---- uneven batch over models --------------------------------------------- *
 * The reference scans one model at a time (grid_scan, GridScan.jl:25-88; its
 * multi-GPU form GridScan.jl:125-197 splits one model's omega columns over
 * devices).  A kls_multi evaluates `batch` omegas for each of n_models
 * precomputed contexts (any mix of NR, Ne, N_alpha and l range, one device)
 * per pass: the contraction of every model is one persistent launch, and the
 * whole pass (omega upload, weights, contraction, split reduction, LU,
 * result download) is one CUDA graph replay.  Each model keeps its
 * context's K split count (tune with kls_autotune before creating the
 * batch), so every determinant is bitwise what kls_det_batch returns for
 * that context: the batch runs the KLS_MIXED_TMEM kernel body (one CTA pair
 * per model, tile pair and K split, from per-model descriptors) when that is
 * every model's split-BF16 form, else the KLS_MIXED_ONE_CTA body.  The contexts must outlive the batch and are not modified;
 * a batch is not re-entrant.  Errors: kls_multi_last_error (NULL handle:
 * errors of kls_multi_create).                                              */
typedef struct kls_multi kls_multi;
typedef struct kls_multi_info {
    int32_t n_models, batch, mode;
    int32_t n_items;              /* work items of the persistent contraction */
    int32_t grid;                 /* CTAs of the persistent contraction       */
    int32_t graph;                /* 1: passes replay a captured CUDA graph    */
    int32_t launches_per_replay;  /* kernels in one pass                      */
    int64_t replays;              /* passes so far                            */
    double  last_ms;              /* device time of the last pass (ms)        */
    int32_t schedule;             /* mixed form, the faster of two passes timed
                                     at creation: one-CTA / pair kernels: 0
                                     persistent round robin or 1 one CTA per
                                     item; TMEM-operand form: 1 one launch with
                                     a CTA pair per item or 2 one launch per
                                     model                                    */
    double  schedule_ms[2];       /* those two passes (ms)                    */
} kls_multi_info;
int kls_multi_create(kls_ctx* const* models, int n_models, int mode, int batch, kls_multi** out);
int kls_multi_destroy(kls_multi* mm);
const char* kls_multi_last_error(const kls_multi* mm);
/* omega_ri [n_models][n] interleaved; det_ri [n_models][n] interleaved;
 * log_abs [n_models][n] (may be NULL).                                      */
int kls_multi_det(kls_multi* mm, const double* omega_ri, int n, double* det_ri, double* log_abs);
/* grid_scan of every model over one (Omega_p, gamma) grid, omega =
 * m_model * Omega_p + i gamma; per model a [n_gamma, n_Op] column-major
 * block of det_grid_ri / log_abs_grid and the column-major argmin
 * (Omega_p0[i], gamma0[i]) as in GridScan.jl:234-246.  sc->mode and
 * sc->batch are ignored (the batch's own).                                  */
int kls_scan_multi(kls_multi* mm, const kls_scan_cfg* sc, double* det_grid_ri,
                   double* log_abs_grid, double* Omega_p0, double* gamma0);
int kls_multi_get_info(const kls_multi* mm, kls_multi_info* out);

/* ---- autotuner (no reference counterpart) ---------------------------------- *
 * Times the contraction of `mode` for the context at `batch` omegas per call
 * with each candidate K split count (the occupancy-derived default, half,
 * twice and three times it) and, for the split-BF16 form, each kernel (one
 * CTA or a CTA pair per tile), and keeps the fastest for the context.  Results
 * are cached per (device name, mode, N_alpha_pad, K_pad, batch) for the
 * process, and in the text file named by the environment variable
 * KLS_TUNE_CACHE when it is set.                                            */
typedef struct kls_tune_result {
    int32_t mode;
    int32_t splits;               /* chosen K splits                          */
    int32_t default_splits;       /* the untuned choice                       */
    int32_t candidates;           /* candidates timed (0: from the cache)     */
    double  ms_per_omega;         /* contraction time of the choice           */
    double  default_ms_per_omega; /* and of the untuned choice (0: cached)    */
    int32_t form;                 /* kernel chosen: KLS_MIXED_* for the split
                                     form, KLS_F64_* for FP64                 */
} kls_tune_result;
int kls_autotune(kls_ctx* ctx, int mode, int batch, kls_tune_result* out);
/* Set the K split count of `mode` by hand (clamped to what the table
 * allows); determinants stay batch-independent for a fixed count.         */
int kls_set_splits(kls_ctx* ctx, int mode, int splits);
/* FP64 contraction form (no reference counterpart): KLS_F64_4M (default) or
 * KLS_F64_3M; the K split count is reset to the form's default.  Both stay
 * within the FP64 parity tolerances; they differ in the last bits.  An
 * uneven batch (kls_multi_create) needs every FP64 model in the same form. */
int kls_set_f64_form(kls_ctx* ctx, int form);

/* ---- determinant stage form (no reference counterpart) -------------------- *
 * KLS_LU_CLUSTER factors each I - M(omega) on one thread-block cluster of 8
 * (or 16) CTAs with the matrix held in their shared memory (latency: one
 * matrix per cluster); KLS_LU_CTA uses one CTA per matrix through L2
 * (throughput for many matrices).  KLS_LU_AUTO (default) takes the cluster
 * form when N_alpha >= 128 and the batch fits one wave of clusters.  Both
 * forms return bitwise the same determinants.  KLS_LU_CLUSTER fails with
 * KLS_ERR_UNSUPPORTED when N_alpha is too large for it.                      */
#define KLS_LU_AUTO          0
#define KLS_LU_CTA           1
#define KLS_LU_CLUSTER       2
int kls_set_lu_mode(kls_ctx* ctx, int mode);

/* ---- split-BF16 contraction kernel (no reference counterpart) ------------- *
 * KLS_MIXED_TMEM (the default when N_alpha_pad <= 384): a CTA pair
 * (tcgen05 cta_group::2, M = 256) per two 64-alpha x 1-omega tiles; the
 * omega-dependent operand w conj(W) is formed once per omega, written from
 * registers straight into tensor memory and read by the MMA from there, the
 * table rows (all N_alpha_pad of them, half per CTA) come from shared memory
 * by TMA.  The older forms re-form that operand once per 128-row tile:
 * KLS_MIXED_ONE_CTA: one CTA per 128-row x 64-alpha x 2-omega tile.
 * KLS_MIXED_PAIR: a cluster of two CTAs per 256-row tile (tcgen05
 * cta_group::2, M = 256): each SM forms half as much of the per-omega
 * operand; it pays off when 2 N_alpha_pad is a multiple of 256 (otherwise
 * the last pair's odd CTA has no rows).  ONE_CTA and PAIR return the same
 * bits (and the bits of the uneven multi-model batch); TMEM sums in another
 * order (same accuracy).  KLS_MIXED_AUTO picks TMEM where it applies, else
 * ONE_CTA; kls_autotune times all of them.
 * Calls kls_prepare_mixed first if needed.                                    */
#define KLS_MIXED_AUTO       0
#define KLS_MIXED_ONE_CTA    1
#define KLS_MIXED_PAIR       2
#define KLS_MIXED_TMEM       3
int kls_set_mixed_form(kls_ctx* ctx, int form);

/* Accumulation chunk of the KLS_MIXED_TMEM form (no reference counterpart):
 * the FP32 tensor-memory accumulator is flushed into FP64 every k_blocks
 * blocks of 32 complex k (default 128, i.e. 4096 terms per FP32 chain).
 * Shorter chunks bound the FP32 accumulation error more tightly; each flush
 * pauses the MMA while the accumulator is drained.                          */
int kls_set_mixed_chunk(kls_ctx* ctx, int k_blocks);

/* ---- failure handling of the device pipeline (no reference counterpart) --- *
 * Every wait of the KLS_MIXED_TMEM contraction (on a copy, an MMA or another
 * warp) is bounded by this limit (default 2 s; the older mixed forms keep a
 * fixed 2 s).  A wait that runs out makes the call return KLS_ERR_TIMEOUT
 * instead of hanging the GPU; the context stays usable.                     */
int kls_set_wait_limit(kls_ctx* ctx, double seconds);
/* Test hooks for the failure paths (no trap, no fault, no unbounded wait):
 * KLS_FAULT_SKIP_ARRIVAL makes the next KLS_MIXED_TMEM contraction skip one
 * producer warp's "operand ready" arrival in its first CTA pair, so the MMA
 * warp's bounded wait runs out and the call returns KLS_ERR_TIMEOUT; it
 * clears itself after that launch.  KLS_FAULT_NAN_ROW writes NaN into the
 * device weight numerator G_k = DJ F0l of the first table row, so every
 * determinant is NaN and host-buffer calls (kls_det_batch, kls_scan,
 * kls_newton, ...) return KLS_ERR_NONFINITE.  KLS_FAULT_NONE clears both and
 * restores the row.                                                        */
#define KLS_FAULT_NONE          0
#define KLS_FAULT_SKIP_ARRIVAL  1
#define KLS_FAULT_NAN_ROW       2
int kls_set_fault_injection(kls_ctx* ctx, int mode);

/* ---- instrumentation ----------------------------------------------------- */
/* Per-stage device time (ms) of the last det batch when timing is enabled:
 * [0] weights, [1] contraction, [2] reduce/epilogue, [3] LU.               */
int kls_enable_timing(kls_ctx* ctx, int on);
int kls_get_stage_ms(kls_ctx* ctx, float* ms4);
/* Device time (ms) of the last kls_precompute's orbit_kernel [0] and
 * wl_kernel [1] when timing was enabled before it.                         */
int kls_get_precompute_ms(kls_ctx* ctx, float* ms2);
/* Kernels launched by this context since creation (monotone counter).      */
int64_t kls_launch_count(const kls_ctx* ctx);

/* ---- bounds-checked build (no reference counterpart) ---------------------- *
 * libkls_checked.so, built from the same sources with KLS_CHECKED, guards
 * the global accesses of the FP64 determinant path (orbits, W_l, rows,
 * weights, contraction, reduction, LU, the allocation-free LU): an index
 * outside its buffer's extent is skipped and logged instead of read or
 * written.  kls_bounds_report returns, for the current device, the number
 * of skipped accesses since the last reset and the site code (KlsSite in
 * csrc/kls_internal.cuh), element index and extent of the first one;
 * reset != 0 clears the logs.  Outputs may be NULL.  The reference has no
 * sanitizer; this is the stand-in for one.  In the default libkls.so it
 * returns KLS_ERR_UNSUPPORTED (message in kls_create_error()).             */
int kls_bounds_report(int64_t* violations, int32_t* first_site, int64_t* first_index,
                      int64_t* first_extent, int reset);

#ifdef __cplusplus
}
#endif
#endif /* KLS_H */

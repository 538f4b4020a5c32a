// Internal declarations shared by the libkls.so translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <climits>
#include <cstdint>
#include <string>
#include "kls.h"

#define KLS_PI 3.14159265358979323846

// Contraction tile geometry (FP64 path): the W table rows are padded to a
// multiple of KLS_TILE so that alpha tiles never need masking.
constexpr int KLS_TILE = 64;
constexpr int KLS_KROW_ALIGN = 64;   // K rows padded to a multiple of this
// TMEM-operand split-BF16 form: FP32 weight variants per k pair (float4 each)
constexpr int KLS_TM_WVAR = 2;

// Per-orbit scalar fields written by the orbit kernel (struct of arrays,
// each NPh doubles, orbit index p = iR + NR*ie as in the reference).
enum OrbitField {
  OF_RC = 0, OF_E_ECC, OF_V, OF_R1, OF_R2, OF_ENERGY, OF_LM, OF_L2M, OF_SGNL, OF_SE,
  OF_OM1, OF_OM2, OF_JAC, OF_F0, OF_FE, OF_FL, OF_DJ,
  OF_COUNT
};

struct kls_mixed;   // split-BF16 tables (kls_mixed.cu)

// One model of an uneven batch (device-resident descriptor, kls_multi.cu).
// The tables are the model context's own; the per-omega buffers belong to
// the batch.
struct kls_mdesc {
  const double* Wre;          // [K_pad][Na_pad]
  const double* Wim;
  const double* Gk;           // [K_pad]
  const double* Ok;           // [K_pad]
  const double* Nk;           // [Na]
  const double* omega;        // [batch][2]
  double2* wt;                // [batch][K_pad]
  double2* part;              // FP64 form: [batch][splits][Na_pad][Na_pad]
  double2* A;                 // [batch][Na][Na]
  double2* det;               // [batch]
  double* logabs;             // [batch]
  double G;
  int64_t K_pad, k_per_split;
  int Na, Na_pad, splits, model;
  // mixed form
  const void* Xh;             // BF16 hi / lo, 2 Na_pad rows in 64-k blocks
  const void* Xl;
  const void* tmap_h;         // device copies of the TMA descriptors (64-byte aligned)
  const void* tmap_l;
  void* wt32;                 // [batch][K_pad] float2, permuted per 64-block
  double* mpart;              // [batch][msplits][2 Na_pad][2 Na_pad] column-major planes
  int msplits, kb_per_split, nkb_total, om_per_item;
};

// One model of an uneven batch in the TMEM-operand split-BF16 form (device
// descriptor): the model context's tensor maps and split parameters and the
// batch's buffers.
struct alignas(64) kls_tm_model {
  CUtensorMap tb_h, tb_l, ty_h, ty_l;
  const float2* wt32;          // [batch][K_pad / 2][KLS_TM_WVAR] float4 weight variants
  double* part;                // [batch * tiles_a][splits][Npad][128] FP64 partials
  int64_t K_pad;
  unsigned long long wait_ns;
  int Npad, tiles_a, n_tiles, splits, kb_per_split, nkb_total, chunk, pad;
};

// One work item of the persistent contraction: FP64 form (model, omega z,
// 64 x 64 tile, K split); mixed form (model, first omega z, 128-row x
// 64-alpha tile, K split, n_om omegas from z, k-blocks [kb0, kb0 + nkb)).
struct kls_item {
  int model, z, tile, split;
  int n_om, kb0, nkb, pad;
};

struct kls_ctx {
  kls_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is launched on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  std::string err;

  // dimensions
  int NR = 0, Ne = 0, NPh = 0, n_l = 0, Na = 0, Na_pad = 0, nwa = 0, nw = 0, nwai = 0;
  int64_t K = 0, K_pad = 0;
  bool precomputed = false;
  int64_t device_bytes = 0;

  // omega-independent device data
  double* d_cosw = nullptr;   // [nw]
  double* d_sinw = nullptr;   // [nw]
  double* d_of = nullptr;     // [OF_COUNT][NPh]
  double* d_SRC = nullptr;    // [NR]
  double* d_rc = nullptr;     // [NR] guiding-centre radii (host C-library pow)
  int* d_valid = nullptr;     // [NPh]  orbit usable for W (all samples finite)
  double* d_w1 = nullptr;     // [NPh][nwa]
  double* d_ra = nullptr;
  double* d_pha = nullptr;
  double* d_alpha = nullptr;  // [Na]
  double* d_dalpha = nullptr; // [Na]
  double* d_N = nullptr;      // [Na]
  double* d_Gk = nullptr;     // [K_pad]  DJ * F0l per row k = il*NPh + p
  double* d_Ok = nullptr;     // [K_pad]  Omega_res per row
  double* d_F0l = nullptr;    // [K_pad]  F0l per row (export only)
  double* d_Wre = nullptr;    // [K_pad][Na_pad]
  double* d_Wim = nullptr;

  // per-batch workspace (grown on demand)
  int ws_omega = 0;           // omegas the workspace holds
  int splits = 1;             // K splits of the contraction (fixed per context)
  int f64_form = KLS_F64_4M;  // FP64 contraction: 4 or 3 (Gauss) real products
  double* d_omega = nullptr;  // [ws_omega][2]
  double2* d_wt = nullptr;    // [ws_omega][K_pad]
  double2* d_part = nullptr;  // [ws_omega][splits][Na_pad][Na_pad]
  double2* d_A = nullptr;     // [ws_omega][Na][Na]  I - M (row-major), overwritten by LU
  double2* d_M = nullptr;     // [Na][Na] optional M export (row-major beta, alpha)
  // KLS_MODE_ANCHORED: FP64 M at the anchor omega (row-major beta, alpha)
  double2* d_anchorM = nullptr;
  bool anchor_set = false;
  double anchor_w[2] = {0.0, 0.0};
  double2* d_det = nullptr;   // [ws_omega]
  double* d_logabs = nullptr; // [ws_omega]
  double* h_pinned = nullptr; // pinned staging for omegas/dets
  int h_pinned_cap = 0;

  kls_mixed* mixed = nullptr;

  // test hook of the non-finite path: G_k[0] overwritten with NaN, original kept
  bool gk0_poisoned = false;
  double gk0_saved = 0.0;

  // determinant stage: KLS_LU_* form and the cluster size it uses (-1: not
  // chosen yet, 0: the cluster form does not fit)
  int lu_mode = 0;
  int lu_cluster = -1;

  // instrumentation
  int64_t launches = 0;
  bool timing = false;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float stage_ms[4] = {0, 0, 0, 0};
  // precompute kernels when timing is on: orbit_kernel, wl_kernel
  cudaEvent_t pev[4] = {nullptr, nullptr, nullptr, nullptr};
  float pre_ms[2] = {0, 0};
};

// event pair around one precompute kernel (no-op unless c->timing)
inline void kls_pre_mark(kls_ctx* c, int i) {
  if (!c->timing) return;
  if (!c->pev[i]) cudaEventCreate(&c->pev[i]);
  cudaEventRecord(c->pev[i], c->stream);
}

// ---- helpers -------------------------------------------------------------
int kls_fail(kls_ctx* c, int code, const std::string& msg);
int kls_cuda_fail(kls_ctx* c, cudaError_t e, const char* what);
#define KLS_CK(ctx, call)                                                   \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) return kls_cuda_fail((ctx), e_, #call);          \
  } while (0)
#define KLS_LAUNCHED(ctx)                                                   \
  do {                                                                      \
    (ctx)->launches++;                                                      \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess) return kls_cuda_fail((ctx), e_, "kernel launch"); \
  } while (0)

// numpy-style linspace point: a + i*(b-a)/(n-1), the last point exactly b
__host__ __device__ inline double kls_lin(double a, double b, int n, int i) {
  if (n <= 1) return a;
  if (i == n - 1) return b;
  double step = (b - a) / (double)(n - 1);
  return a + (double)i * step;
}

// ---- stage entry points (host side, launch on ctx->stream) ---------------
int kls_run_orbits(kls_ctx* c);
int kls_upload_alpha(kls_ctx* c);
int kls_run_basis(kls_ctx* c);
int kls_run_weights(kls_ctx* c, int n, const double* anchor = nullptr);
int kls_run_contract_f64(kls_ctx* c, int n, int splits);
int kls_run_reduce(kls_ctx* c, int n, int splits, bool export_M);
int kls_run_lu(kls_ctx* c, int n);
int kls_choose_splits(const kls_ctx* c);
// mixed-precision path (kls_mixed.cu)
int kls_mixed_prepare(kls_ctx* c);
int kls_mixed_contract(kls_ctx* c, int n, int splits);
int kls_mixed_reduce(kls_ctx* c, int n, bool export_M, const double2* Ma = nullptr);
int kls_mixed_check(kls_ctx* c);     // pipeline timeout flag of the last launches
void kls_mixed_free(kls_ctx* c);
// uneven batch over models (kls_multi.cu drives these)
int kls_multi_launch_f64(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs, int n_pairs,
                         const kls_item* d_items, int n_items, int* d_counter, int grid,
                         int64_t max_K_pad, int form);
int kls_multi_launch_lu(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs, int n_pairs,
                        int max_Na);
int kls_multi_launch_f64_weights(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs,
                                 int n_pairs, int64_t max_K_pad);
int kls_multi_contract_slots(int device, int form);
int64_t kls_f64_k_per_split(int64_t K_pad, int splits);
int kls_multi_launch_mixed(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs,
                           int n_pairs, const kls_item* d_items, const int* d_starts, int grid,
                           int64_t max_K_pad, int* d_err);
int kls_mixed_slots(int device);
int kls_mixed_splits_of(const kls_ctx* c);
// K splits of the one-CTA form (the uneven batch runs that kernel body)
int kls_mixed_legacy_splits(const kls_ctx* c);
int kls_mixed_default_splits(const kls_ctx* c);
int kls_mixed_set_form(kls_ctx* c, int form);
int kls_mixed_form_of(const kls_ctx* c);
int kls_mixed_set_splits(kls_ctx* c, int splits);
const void* kls_mixed_tables(const kls_ctx* c, const void** Xl, const void** tmap_h,
                             const void** tmap_l);
int kls_mixed_set_wait(kls_ctx* c, unsigned long long ns, int fault_mode);
// TMEM-operand form of the split-BF16 contraction (kls_mixed_tm.cu)
struct kls_mixed_tm;
bool kls_tm_supported(const kls_ctx* c);
int kls_tm_default_splits(const kls_ctx* c);
int kls_tm_create(kls_ctx* c, const void* Xh, const void* Xl, kls_mixed_tm** out);
void kls_tm_destroy(kls_mixed_tm* t);
int kls_tm_splits(const kls_mixed_tm* t);
void kls_tm_set_splits(const kls_ctx* c, kls_mixed_tm* t, int s);
void kls_tm_set_chunk(kls_mixed_tm* t, int stages);
int kls_mixed_set_chunk(kls_ctx* c, int stages);
int kls_tm_contract(kls_ctx* c, kls_mixed_tm* t, int n, int* d_err, unsigned long long wait_ns,
                    int fault_skip);
int kls_tm_reduce(kls_ctx* c, kls_mixed_tm* t, int n, bool export_M, const double2* Ma);
// the context's TMEM-operand state when that is its split-BF16 form (else null)
kls_mixed_tm* kls_mixed_tm_state(const kls_ctx* c, unsigned long long* wait_ns);
void kls_tm_describe(const kls_ctx* c, const kls_mixed_tm* t, unsigned long long wait_ns,
                     int batch, kls_tm_model* out);
// per_model: one launch of the single-model kernel per model (h_tm: host
// copies of the descriptors) instead of one launch over every item
int kls_tm_multi_launch(cudaStream_t st, const kls_mdesc* d_md, const kls_tm_model* d_tm,
                        const int2* d_pairs, int n_pairs, const int4* d_items, int n_items,
                        int64_t max_K_pad, int max_Npad, int* d_err, const kls_tm_model* h_tm,
                        int n_models, bool per_model);

// NVTX range for the lifetime of a scope (profilers show the library's
// stages by name; without a tool attached a push/pop is a no-op call)
struct KlsRange {
  explicit KlsRange(const char* name) { nvtxRangePushA(name); }
  ~KlsRange() { nvtxRangePop(); }
  KlsRange(const KlsRange&) = delete;
  KlsRange& operator=(const KlsRange&) = delete;
};

// ---- bounds-checked build (KLS_CHECKED) ------------------------------------
// libkls_checked.so is the same sources compiled with -DKLS_CHECKED: every
// guarded global access of the FP64 determinant path (orbit, W_l, row,
// weight, contraction, reduction and LU kernels) first tests its element
// index against the extent of the buffer it touches, as the launch's own
// parameters size it.  An access outside is skipped (a load reads 0) and
// counted in this translation unit's device log, with the site code, index
// and extent of the first one; kls_bounds_report collects the logs of every
// unit.  The guards are written with the statement macros below, which
// expand to nothing (KLS_IF, KLS_UNLESS) or to the unguarded expression
// (KLS_LD) in the default build, so its preprocessed source is the
// unguarded one token for token.
enum KlsSite {
  KS_ORBIT_TABLE = 1,   // cos / sin of the w grid, Rc and S_RC tables
  KS_ORBIT_SAMPLES,     // w1 / r / theta samples written per orbit
  KS_ORBIT_FIELDS,      // per-orbit scalar fields and the validity flag
  KS_WL_SAMPLES,        // orbit samples and fields read by the W_l kernel
  KS_WL_OUT,            // W table rows written
  KS_ROWS,              // G_k / Omega_res / F0l rows and the fields they read
  KS_NKERNEL,           // alpha grid and N_m(alpha)
  KS_WEIGHTS,           // omega and the weight rows
  KS_CONTRACT_SRC,      // table tiles and weights staged by the contraction
  KS_CONTRACT_OUT,      // contraction partials written
  KS_REDUCE,            // partials summed, I - M and M written
  KS_LU,                // LU matrices, determinants
  KS_LU_STATIC,         // allocation-free LU: input, scratch, determinants
};
#ifdef KLS_CHECKED
struct KlsBoundsLog {
  unsigned long long count;
  long long index, extent;
  int site, pad;
};
namespace {
__device__ KlsBoundsLog g_kls_bounds;   // one per translation unit
}
__device__ __forceinline__ bool kls_in_bounds(long long i, long long n, int site) {
  if (i >= 0 && i < n) return true;
  if (atomicAdd(&g_kls_bounds.count, 1ull) == 0ull) {
    g_kls_bounds.index = i;
    g_kls_bounds.extent = n;
    g_kls_bounds.site = site;
  }
  return false;
}
#define KLS_IB(i, n, site) kls_in_bounds((long long)(i), (long long)(n), (site))
#define KLS_IF(cond) if (cond)
#define KLS_UNLESS(cond, action) if (!(cond)) action;
#define KLS_LD(cond, expr, fallback) ((cond) ? (expr) : (fallback))
// host: every unit registers the reader of its log at load time
int kls_bounds_register(int (*reader)(KlsBoundsLog* out, bool reset));
namespace {
int kls_bounds_read(KlsBoundsLog* out, bool reset) {
  if (cudaMemcpyFromSymbol(out, g_kls_bounds, sizeof(KlsBoundsLog)) != cudaSuccess) return -1;
  if (reset) {
    KlsBoundsLog z{};
    if (cudaMemcpyToSymbol(g_kls_bounds, &z, sizeof z) != cudaSuccess) return -1;
  }
  return 0;
}
const int kls_bounds_registered = kls_bounds_register(&kls_bounds_read);
}
#else
#define KLS_IF(cond)
#define KLS_UNLESS(cond, action)
#define KLS_LD(cond, expr, fallback) expr
#endif

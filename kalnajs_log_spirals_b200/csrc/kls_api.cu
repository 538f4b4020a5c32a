// C ABI of libkls.so (declared in include/kls.h).
//
// Host-side control of the path: configuration checks, device memory,
// the omega-independent precompute (BasisFunctions.precompute_all +
// to_device), batched determinants (MatrixBuilder.compute_determinant /
// _batched), the omega-plane scan (GridScan.grid_scan / find_minimum) and the
// Newton search (NewtonSolver.newton_search) with the reference's exact
// step, line-search, clamp and stopping rules.
#include "kls_internal.cuh"
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

static thread_local std::string g_create_err;

#ifdef KLS_CHECKED
// readers of the translation units' bounds logs (registered at load time)
static std::vector<int (*)(KlsBoundsLog*, bool)>& bounds_readers() {
  static std::vector<int (*)(KlsBoundsLog*, bool)> r;
  return r;
}
int kls_bounds_register(int (*reader)(KlsBoundsLog* out, bool reset)) {
  bounds_readers().push_back(reader);
  return (int)bounds_readers().size();
}
#endif

int kls_fail(kls_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  else g_create_err = msg;
  return code;
}

int kls_cuda_fail(kls_ctx* c, cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  int code = (e == cudaErrorMemoryAllocation) ? KLS_ERR_OOM : KLS_ERR_CUDA;
  return kls_fail(c, code, m);
}

namespace {

constexpr int WS_CHUNK = 16;   // omegas per device launch sequence

int validate(const kls_config* k, std::string& msg) {
  char buf[256];
  auto bad = [&](const char* m) { msg = m; return KLS_ERR_CONFIG; };
  if (!k) return bad("config is NULL");
  if (k->NR < 1 || k->Ne < 1) return bad("NR and Ne must be >= 1");
  if (k->N_alpha < 1) return bad("N_alpha must be >= 1");
  if (k->l_max < k->l_min) return bad("l_max must be >= l_min");
  if (!(k->Rc_min > 0.0) || !(k->Rc_max >= k->Rc_min)) return bad("need 0 < Rc_min <= Rc_max");
  if (!(k->q1 > 0.0)) return bad("q1 must be > 0");
  if (!(k->alpha_max >= 0.0)) return bad("alpha_max must be >= 0");
  if (k->n_zang < 0) return bad("n_zang must be >= 0");
  if (k->nw < 3 || k->nwa < 2 || k->nwa > k->nw) return bad("need nw >= 3 and 2 <= nwa <= nw");
  int nwai = (k->nw - 1) / (k->nwa - 1);
  int len = (k->nw - 1) / nwai + 1;   // length(1:nwai:nw)
  if (len != k->nwa) {
    snprintf(buf, sizeof buf,
             "length(1:nwai:nw) = %d differs from nwa = %d (the reference fails with a "
             "DimensionMismatch for this (nw, nwa))", len, k->nwa);
    msg = buf;
    return KLS_ERR_CONFIG;
  }
  double np = (double)k->NR * k->Ne;
  if (np > (double)INT_MAX) return bad("NR * Ne must be below 2^31 (orbit index range)");
  if (np * (k->l_max - k->l_min + 1) > 4.0e9) return bad("NPh * n_l too large");
  // the determinant's LU keeps two rows of N_alpha complex values in the
  // shared memory of one CTA (227 KB on sm_100)
  if (k->N_alpha > 7168) return bad("N_alpha must be <= 7168 (LU rows in shared memory)");
  if (!std::isfinite(k->G) || !std::isfinite(k->L0) || !std::isfinite(k->v_min))
    return bad("non-finite G, L0 or v_min");
  for (int q : {k->quad_alpha, k->quad_rc, k->quad_v})
    if (q < KLS_QUAD_DEFAULT || q > KLS_QUAD_BOOLE) return bad("unknown quadrature rule");
  return KLS_OK;
}

template <typename T>
int dalloc(kls_ctx* c, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T) + 16);
  if (e != cudaSuccess) {
    *p = nullptr;
    char buf[160];
    snprintf(buf, sizeof buf, "cudaMalloc of %.3f GB failed: %s", count * sizeof(T) / 1e9,
             cudaGetErrorString(e));
    return kls_fail(c, KLS_ERR_OOM, buf);
  }
  c->device_bytes += (int64_t)(count * sizeof(T));
  return KLS_OK;
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

int ensure_ws(kls_ctx* c, int n) {
  if (n <= c->ws_omega && c->d_part) return KLS_OK;
  int cap = std::max(n, c->ws_omega);
  dfree(c->d_omega); dfree(c->d_wt); dfree(c->d_part); dfree(c->d_A); dfree(c->d_det);
  dfree(c->d_logabs);
  c->d_omega = nullptr; c->d_wt = nullptr; c->d_part = nullptr; c->d_A = nullptr;
  c->d_det = nullptr; c->d_logabs = nullptr;
  c->ws_omega = 0;
  int r;
  if ((r = dalloc(c, &c->d_omega, (size_t)2 * cap))) return r;
  if ((r = dalloc(c, &c->d_wt, (size_t)cap * c->K_pad))) return r;
  if ((r = dalloc(c, &c->d_part, (size_t)cap * c->splits * c->Na_pad * c->Na_pad))) return r;
  if ((r = dalloc(c, &c->d_A, (size_t)cap * c->Na * c->Na))) return r;
  if ((r = dalloc(c, &c->d_det, (size_t)cap))) return r;
  if ((r = dalloc(c, &c->d_logabs, (size_t)cap))) return r;
  c->ws_omega = cap;
  return KLS_OK;
}

// One launch sequence for n (<= ws) omegas already in c->d_omega.
int run_batch(kls_ctx* c, int n, int mode, bool export_M) {
  KlsRange range(mode == KLS_MODE_FP64 ? "kls det batch (FP64)"
                 : mode == KLS_MODE_MIXED ? "kls det batch (split-BF16)"
                                          : "kls det batch (anchored)");
  int r;
  const int splits = c->splits;
  if (mode != KLS_MODE_FP64 && mode != KLS_MODE_MIXED && mode != KLS_MODE_ANCHORED)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown precision mode");
  const bool anchored = mode == KLS_MODE_ANCHORED;
  if (anchored && !c->anchor_set)
    return kls_fail(c, KLS_ERR_STATE, "KLS_MODE_ANCHORED needs kls_set_anchor first");
  if (c->timing) KLS_CK(c, cudaEventRecord(c->ev[0], c->stream));
  if ((r = kls_run_weights(c, n, anchored ? c->anchor_w : nullptr))) return r;
  if (c->timing) KLS_CK(c, cudaEventRecord(c->ev[1], c->stream));
  if (mode == KLS_MODE_FP64) {
    if (!c->d_Wre) return kls_fail(c, KLS_ERR_STATE, "the FP64 table was released (kls_release_fp64)");
    if ((r = kls_run_contract_f64(c, n, splits))) return r;
  } else {
    if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
    if ((r = kls_mixed_contract(c, n, splits))) return r;
  }
  if (c->timing) KLS_CK(c, cudaEventRecord(c->ev[2], c->stream));
  if (mode != KLS_MODE_FP64) {
    if ((r = kls_mixed_reduce(c, n, export_M, anchored ? c->d_anchorM : nullptr))) return r;
  } else if ((r = kls_run_reduce(c, n, splits, export_M))) {
    return r;
  }
  if (c->timing) KLS_CK(c, cudaEventRecord(c->ev[3], c->stream));
  if ((r = kls_run_lu(c, n))) return r;
  if (c->timing) KLS_CK(c, cudaEventRecord(c->ev[4], c->stream));
  return KLS_OK;
}

int collect_timing(kls_ctx* c) {
  if (!c->timing) return KLS_OK;
  KLS_CK(c, cudaEventSynchronize(c->ev[4]));
  for (int i = 0; i < 4; ++i) {
    float ms = 0.f;
    KLS_CK(c, cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]));
    c->stage_ms[i] += ms;
  }
  return KLS_OK;
}

int check_ready(kls_ctx* c) {
  if (!c) return KLS_ERR_CONFIG;
  if (!c->precomputed) return kls_fail(c, KLS_ERR_STATE, "kls_precompute has not run");
  KLS_CK(c, cudaSetDevice(c->device));
  return KLS_OK;
}

// Host-buffer batch: omegas in, dets out, chunked by the workspace size.
int det_batch_host(kls_ctx* c, const double* omega_ri, int n, int mode, double* det_ri,
                   double* log_abs) {
  int r;
  if (c->timing) std::fill(c->stage_ms, c->stage_ms + 4, 0.f);
  for (int b = 0; b < n; b += WS_CHUNK) {
    int nb = std::min(WS_CHUNK, n - b);
    for (int i = 0; i < 2 * nb; ++i)
      if (!std::isfinite(omega_ri[2 * b + i]))
        return kls_fail(c, KLS_ERR_NONFINITE, "non-finite omega");
    if ((r = ensure_ws(c, nb))) return r;
    KLS_CK(c, cudaMemcpyAsync(c->d_omega, omega_ri + 2 * b, 2 * nb * sizeof(double),
                              cudaMemcpyHostToDevice, c->stream));
    if ((r = run_batch(c, nb, mode, false))) return r;
    KLS_CK(c, cudaMemcpyAsync(det_ri + 2 * b, c->d_det, nb * sizeof(double2),
                              cudaMemcpyDeviceToHost, c->stream));
    if (log_abs)
      KLS_CK(c, cudaMemcpyAsync(log_abs + b, c->d_logabs, nb * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    KLS_CK(c, cudaStreamSynchronize(c->stream));
    if (mode != KLS_MODE_FP64 && (r = kls_mixed_check(c))) return r;
    if ((r = collect_timing(c))) return r;
    for (int i = 0; i < nb; ++i)
      if (std::isnan(det_ri[2 * (b + i)]) || std::isnan(det_ri[2 * (b + i) + 1])) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "NaN determinant at omega = %.17g%+.17gi (a non-finite table row, weight "
                 "or model value)", omega_ri[2 * (b + i)], omega_ri[2 * (b + i) + 1]);
        return kls_fail(c, KLS_ERR_NONFINITE, buf);
      }
  }
  return KLS_OK;
}

// 2x2 solve J x = F by LU with partial pivoting (the order LAPACK dgesv uses
// for Julia's J \ F).  Returns false on an exactly singular factor.
bool solve2(const double J[2][2], const double F[2], double x[2]) {
  double a00 = J[0][0], a01 = J[0][1], a10 = J[1][0], a11 = J[1][1];
  double f0 = F[0], f1 = F[1];
  if (std::fabs(a10) > std::fabs(a00)) {
    std::swap(a00, a10); std::swap(a01, a11); std::swap(f0, f1);
  }
  if (a00 == 0.0) return false;
  double l = a10 * (1.0 / a00);
  double u11 = a11 - l * a01;
  if (u11 == 0.0) return false;
  double y1 = f1 - l * f0;
  x[1] = y1 / u11;
  x[0] = (f0 - a01 * x[1]) / a00;
  return true;
}

}  // namespace

// ======================================================================
extern "C" {

const char* kls_create_error(void) { return g_create_err.c_str(); }

const char* kls_last_error(const kls_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

int kls_create(const kls_config* cfg, int device, kls_ctx** out) {
  if (!out) return kls_fail(nullptr, KLS_ERR_CONFIG, "out is NULL");
  *out = nullptr;
  std::string msg;
  int r = validate(cfg, msg);
  if (r) return kls_fail(nullptr, r, msg);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return kls_fail(nullptr, KLS_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return kls_fail(nullptr, KLS_ERR_CONFIG, "bad device index");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
    return kls_fail(nullptr, KLS_ERR_UNSUPPORTED, "libkls.so is built for sm_100a (B200)");
  kls_ctx* c = new kls_ctx();
  c->cfg = *cfg;
  c->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaStreamCreateWithFlags(
      &c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete c;
    return kls_fail(nullptr, KLS_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
  }
  c->own_stream = c->stream;
  for (auto& ev : c->ev) cudaEventCreate(&ev);
  c->NR = cfg->NR; c->Ne = cfg->Ne; c->NPh = cfg->NR * cfg->Ne;
  c->n_l = cfg->l_max - cfg->l_min + 1;
  c->Na = cfg->N_alpha;
  c->Na_pad = ((cfg->N_alpha + KLS_TILE - 1) / KLS_TILE) * KLS_TILE;
  c->nw = cfg->nw; c->nwa = cfg->nwa; c->nwai = (cfg->nw - 1) / (cfg->nwa - 1);
  c->K = (int64_t)c->NPh * c->n_l;
  c->K_pad = ((c->K + KLS_KROW_ALIGN - 1) / KLS_KROW_ALIGN) * KLS_KROW_ALIGN;
  c->splits = kls_choose_splits(c);

  size_t need = (size_t)2 * c->K_pad * c->Na_pad * sizeof(double);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  if (need > fr) {
    char buf[200];
    snprintf(buf, sizeof buf, "W table needs %.2f GB, device has %.2f GB free", need / 1e9,
             fr / 1e9);
    kls_destroy(c);
    return kls_fail(nullptr, KLS_ERR_OOM, buf);
  }
  if ((r = dalloc(c, &c->d_cosw, c->nw)) || (r = dalloc(c, &c->d_sinw, c->nw)) ||
      (r = dalloc(c, &c->d_of, (size_t)OF_COUNT * c->NPh)) ||
      (r = dalloc(c, &c->d_SRC, c->NR)) || (r = dalloc(c, &c->d_rc, c->NR)) ||
      (r = dalloc(c, &c->d_valid, c->NPh)) ||
      (r = dalloc(c, &c->d_w1, (size_t)c->NPh * c->nwa)) ||
      (r = dalloc(c, &c->d_ra, (size_t)c->NPh * c->nwa)) ||
      (r = dalloc(c, &c->d_pha, (size_t)c->NPh * c->nwa)) ||
      (r = dalloc(c, &c->d_alpha, c->Na)) || (r = dalloc(c, &c->d_dalpha, c->Na)) ||
      (r = dalloc(c, &c->d_N, c->Na)) || (r = dalloc(c, &c->d_Gk, c->K_pad)) ||
      (r = dalloc(c, &c->d_Ok, c->K_pad)) || (r = dalloc(c, &c->d_F0l, c->K_pad)) ||
      (r = dalloc(c, &c->d_Wre, (size_t)c->K_pad * c->Na_pad)) ||
      (r = dalloc(c, &c->d_Wim, (size_t)c->K_pad * c->Na_pad)) ||
      (r = dalloc(c, &c->d_M, (size_t)c->Na * c->Na))) {
    std::string m = c->err;
    kls_destroy(c);
    return kls_fail(nullptr, r, m);
  }
  *out = c;
  return KLS_OK;
}

int kls_destroy(kls_ctx* c) {
  if (!c) return KLS_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  kls_mixed_free(c);
  void* ptrs[] = {c->d_cosw, c->d_sinw, c->d_of, c->d_SRC, c->d_rc, c->d_valid, c->d_w1, c->d_ra,
                  c->d_pha, c->d_alpha, c->d_dalpha, c->d_N, c->d_Gk, c->d_Ok, c->d_F0l,
                  c->d_Wre, c->d_Wim, c->d_omega, c->d_wt, c->d_part, c->d_A, c->d_M,
                  c->d_anchorM, c->d_det, c->d_logabs};
  for (void* p : ptrs) dfree(p);
  for (auto& ev : c->ev) if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->pev) if (ev) cudaEventDestroy(ev);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return KLS_OK;
}

int kls_get_dims(const kls_ctx* c, kls_dims* d) {
  if (!c || !d) return KLS_ERR_CONFIG;
  d->NPh = c->NPh; d->n_l = c->n_l; d->N_alpha = c->Na; d->N_alpha_pad = c->Na_pad;
  d->K = c->K; d->K_pad = c->K_pad; d->nwa = c->nwa; d->device_bytes = c->device_bytes;
  return KLS_OK;
}

int kls_set_stream(kls_ctx* c, void* s) {
  if (!c) return KLS_ERR_CONFIG;
  c->stream = s ? (cudaStream_t)s : c->own_stream;
  return KLS_OK;
}

int kls_precompute(kls_ctx* c) {
  KlsRange range("kls_precompute");
  if (!c) return KLS_ERR_CONFIG;
  KLS_CK(c, cudaSetDevice(c->device));
  int r;
  if ((r = kls_run_orbits(c))) return r;
  if ((r = kls_run_basis(c))) return r;
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  if (c->timing && c->pev[3]) {
    KLS_CK(c, cudaEventElapsedTime(&c->pre_ms[0], c->pev[0], c->pev[1]));
    KLS_CK(c, cudaEventElapsedTime(&c->pre_ms[1], c->pev[2], c->pev[3]));
  }
  c->precomputed = true;
  return KLS_OK;
}

int kls_prepare_mixed(kls_ctx* c) {
  int r = check_ready(c);
  if (r) return r;
  return kls_mixed_prepare(c);
}

int kls_release_fp64(kls_ctx* c) {
  int r = check_ready(c);
  if (r) return r;
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  if (c->d_Wre) {
    cudaFree(c->d_Wre);
    cudaFree(c->d_Wim);
    c->d_Wre = c->d_Wim = nullptr;
    c->device_bytes -= (int64_t)(2 * (size_t)c->K_pad * c->Na_pad * sizeof(double));
  }
  return KLS_OK;
}

int kls_export_orbits(kls_ctx* c, double* Om1, double* Om2, double* jac, double* F0,
                      double* FE, double* FL, double* DJ, double* w1, double* ra, double* pha) {
  int r = check_ready(c);
  if (r) return r;
  const size_t n = c->NPh;
  struct { double* h; int f; } fl[] = {{Om1, OF_OM1}, {Om2, OF_OM2}, {jac, OF_JAC}, {F0, OF_F0},
                                       {FE, OF_FE},   {FL, OF_FL},   {DJ, OF_DJ}};
  for (auto& x : fl)
    if (x.h) KLS_CK(c, cudaMemcpy(x.h, c->d_of + (size_t)x.f * n, n * sizeof(double),
                                  cudaMemcpyDeviceToHost));
  // [p][j] on the device is the reference's column-major [nwa, NR, Ne]
  if (w1) KLS_CK(c, cudaMemcpy(w1, c->d_w1, n * c->nwa * sizeof(double), cudaMemcpyDeviceToHost));
  if (ra) KLS_CK(c, cudaMemcpy(ra, c->d_ra, n * c->nwa * sizeof(double), cudaMemcpyDeviceToHost));
  if (pha) KLS_CK(c, cudaMemcpy(pha, c->d_pha, n * c->nwa * sizeof(double), cudaMemcpyDeviceToHost));
  return KLS_OK;
}

int kls_export_grids(kls_ctx* c, double* Rc, double* e, double* E, double* L_m, double* S_RC,
                     double* S_e) {
  int r = check_ready(c);
  if (r) return r;
  const size_t n = c->NPh;
  struct { double* h; int f; } fl[] = {{Rc, OF_RC}, {e, OF_E_ECC}, {E, OF_ENERGY}, {L_m, OF_LM},
                                       {S_e, OF_SE}};
  for (auto& x : fl)
    if (x.h) KLS_CK(c, cudaMemcpy(x.h, c->d_of + (size_t)x.f * n, n * sizeof(double),
                                  cudaMemcpyDeviceToHost));
  if (S_RC) KLS_CK(c, cudaMemcpy(S_RC, c->d_SRC, c->NR * sizeof(double), cudaMemcpyDeviceToHost));
  return KLS_OK;
}

int kls_export_alpha(kls_ctx* c, double* alpha, double* dalpha, double* Nk) {
  int r = check_ready(c);
  if (r) return r;
  if (alpha) KLS_CK(c, cudaMemcpy(alpha, c->d_alpha, c->Na * sizeof(double), cudaMemcpyDeviceToHost));
  if (dalpha) KLS_CK(c, cudaMemcpy(dalpha, c->d_dalpha, c->Na * sizeof(double), cudaMemcpyDeviceToHost));
  if (Nk) KLS_CK(c, cudaMemcpy(Nk, c->d_N, c->Na * sizeof(double), cudaMemcpyDeviceToHost));
  return KLS_OK;
}

int kls_export_resonant(kls_ctx* c, double* F0l, double* Ores) {
  int r = check_ready(c);
  if (r) return r;
  if (F0l) KLS_CK(c, cudaMemcpy(F0l, c->d_F0l, c->K * sizeof(double), cudaMemcpyDeviceToHost));
  if (Ores) KLS_CK(c, cudaMemcpy(Ores, c->d_Ok, c->K * sizeof(double), cudaMemcpyDeviceToHost));
  return KLS_OK;
}

int kls_export_W(kls_ctx* c, int il0, int nl, double* W) {
  if (c->precomputed && !c->d_Wre)
    return kls_fail(c, KLS_ERR_STATE, "the FP64 table was released (kls_release_fp64)");
  int r = check_ready(c);
  if (r) return r;
  if (il0 < 0 || nl < 0 || il0 + nl > c->n_l || !W)
    return kls_fail(c, KLS_ERR_CONFIG, "bad harmonic range for kls_export_W");
  const size_t rows = c->NPh, ld = c->Na_pad;
  std::vector<double> re(rows * ld), im(rows * ld);
  for (int q = 0; q < nl; ++q) {
    size_t r0 = (size_t)(il0 + q) * rows;
    KLS_CK(c, cudaMemcpy(re.data(), c->d_Wre + r0 * ld, rows * ld * sizeof(double),
                         cudaMemcpyDeviceToHost));
    KLS_CK(c, cudaMemcpy(im.data(), c->d_Wim + r0 * ld, rows * ld * sizeof(double),
                         cudaMemcpyDeviceToHost));
    // reference layout [NPh, N_alpha, n_l], column-major, interleaved complex
    double* blk = W + (size_t)2 * q * rows * c->Na;
    for (int a = 0; a < c->Na; ++a)
      for (size_t p = 0; p < rows; ++p) {
        blk[2 * (p + rows * a)] = re[p * ld + a];
        blk[2 * (p + rows * a) + 1] = im[p * ld + a];
      }
  }
  return KLS_OK;
}

int kls_det_batch(kls_ctx* c, const double* omega_ri, int n, int mode, double* det_ri,
                  double* log_abs) {
  int r = check_ready(c);
  if (r) return r;
  if (n < 0 || (n > 0 && (!omega_ri || !det_ri)))
    return kls_fail(c, KLS_ERR_CONFIG, "bad arguments to kls_det_batch");
  return det_batch_host(c, omega_ri, n, mode, det_ri, log_abs);
}

int kls_det(kls_ctx* c, double wr, double wi, int mode, double* det_re, double* det_im,
            double* log_abs) {
  int r = check_ready(c);
  if (r) return r;
  if (!det_re || !det_im) return kls_fail(c, KLS_ERR_CONFIG, "bad arguments to kls_det");
  const double om[2] = {wr, wi};
  double d[2];
  if ((r = det_batch_host(c, om, 1, mode, d, log_abs))) return r;
  *det_re = d[0];
  *det_im = d[1];
  return KLS_OK;
}

int kls_det_batch_device(kls_ctx* c, const double* d_omega, int n, int mode, double* d_det,
                         double* d_log_abs) {
  int r = check_ready(c);
  if (r) return r;
  if (n < 0 || (n > 0 && (!d_omega || !d_det)))
    return kls_fail(c, KLS_ERR_CONFIG, "bad arguments to kls_det_batch_device");
  if (c->timing) std::fill(c->stage_ms, c->stage_ms + 4, 0.f);
  for (int b = 0; b < n; b += WS_CHUNK) {
    int nb = std::min(WS_CHUNK, n - b);
    if ((r = ensure_ws(c, nb))) return r;
    KLS_CK(c, cudaMemcpyAsync(c->d_omega, d_omega + 2 * b, 2 * nb * sizeof(double),
                              cudaMemcpyDeviceToDevice, c->stream));
    if ((r = run_batch(c, nb, mode, false))) return r;
    KLS_CK(c, cudaMemcpyAsync(d_det + 2 * b, c->d_det, nb * sizeof(double2),
                              cudaMemcpyDeviceToDevice, c->stream));
    if (d_log_abs)
      KLS_CK(c, cudaMemcpyAsync(d_log_abs + b, c->d_logabs, nb * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
    if (c->timing) {
      // stage times need the events of every chunk; keep the device busy otherwise
      if ((r = collect_timing(c))) return r;
    }
  }
  return KLS_OK;
}

int kls_build_M(kls_ctx* c, double wr, double wi, int mode, double* M) {
  int r = check_ready(c);
  if (r) return r;
  if (!M) return kls_fail(c, KLS_ERR_CONFIG, "M is NULL");
  if ((r = ensure_ws(c, 1))) return r;
  double om[2] = {wr, wi};
  KLS_CK(c, cudaMemcpyAsync(c->d_omega, om, sizeof om, cudaMemcpyHostToDevice, c->stream));
  if ((r = run_batch(c, 1, mode, true))) return r;
  std::vector<double2> h((size_t)c->Na * c->Na);
  KLS_CK(c, cudaMemcpyAsync(h.data(), c->d_M, h.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                            c->stream));
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  if (mode != KLS_MODE_FP64 && (r = kls_mixed_check(c))) return r;
  const int N = c->Na;
  for (int b = 0; b < N; ++b)
    for (int a = 0; a < N; ++a) {   // device [b][a] -> host column-major (b + N a)
      M[2 * (b + (size_t)N * a)] = h[(size_t)b * N + a].x;
      M[2 * (b + (size_t)N * a) + 1] = h[(size_t)b * N + a].y;
    }
  return KLS_OK;
}

int kls_set_anchor(kls_ctx* c, double wr, double wi, double* det_ri) {
  KlsRange range("kls_set_anchor");
  int r = check_ready(c);
  if (r) return r;
  if (!std::isfinite(wr) || !std::isfinite(wi))
    return kls_fail(c, KLS_ERR_NONFINITE, "non-finite anchor omega");
  if (!c->d_Wre) return kls_fail(c, KLS_ERR_STATE, "the FP64 table was released (kls_release_fp64)");
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  if (!c->d_anchorM && (r = dalloc(c, &c->d_anchorM, (size_t)c->Na * c->Na))) return r;
  if ((r = ensure_ws(c, 1))) return r;
  c->anchor_set = false;
  const double om[2] = {wr, wi};
  KLS_CK(c, cudaMemcpyAsync(c->d_omega, om, sizeof om, cudaMemcpyHostToDevice, c->stream));
  if ((r = run_batch(c, 1, KLS_MODE_FP64, true))) return r;
  KLS_CK(c, cudaMemcpyAsync(c->d_anchorM, c->d_M, (size_t)c->Na * c->Na * sizeof(double2),
                            cudaMemcpyDeviceToDevice, c->stream));
  double2 d;
  KLS_CK(c, cudaMemcpyAsync(&d, c->d_det, sizeof d, cudaMemcpyDeviceToHost, c->stream));
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  if ((r = collect_timing(c))) return r;
  if (std::isnan(d.x) || std::isnan(d.y))
    return kls_fail(c, KLS_ERR_NONFINITE, "NaN determinant at the anchor");
  c->anchor_w[0] = wr;
  c->anchor_w[1] = wi;
  c->anchor_set = true;
  if (det_ri) { det_ri[0] = d.x; det_ri[1] = d.y; }
  return KLS_OK;
}

int kls_scan(kls_ctx* c, const kls_scan_cfg* sc, double* det_grid, double* log_abs_grid,
             double* Op0, double* g0) {
  KlsRange range("kls_scan");
  int r = check_ready(c);
  if (r) return r;
  if (!sc || sc->n_Op < 1 || sc->n_gamma < 1 || !det_grid)
    return kls_fail(c, KLS_ERR_CONFIG, "bad scan configuration");
  if ((long long)sc->n_Op * sc->n_gamma > INT_MAX)
    return kls_fail(c, KLS_ERR_CONFIG, "scan grid larger than 2^31 - 1 points");
  const int nO = sc->n_Op, nG = sc->n_gamma, n = nO * nG;
  std::vector<double> om(2 * (size_t)n), la((size_t)n);
  // column-major det_grid[i_gamma, j_Op] (GridScan.jl:47, :101-104)
  for (int j = 0; j < nO; ++j) {
    double Op = kls_lin(sc->Omega_p_min, sc->Omega_p_max, nO, j);
    for (int i = 0; i < nG; ++i) {
      double g = kls_lin(sc->gamma_min, sc->gamma_max, nG, i);
      om[2 * ((size_t)i + (size_t)nG * j)] = c->cfg.m * Op;
      om[2 * ((size_t)i + (size_t)nG * j) + 1] = g;
    }
  }
  if ((r = det_batch_host(c, om.data(), n, sc->mode, det_grid, la.data()))) return r;
  if (log_abs_grid) std::copy(la.begin(), la.end(), log_abs_grid);
  // argmin |det| in column-major order, first occurrence; NaN wins as in Julia
  int best = 0;
  double bv = INFINITY;
  for (int q = 0; q < n; ++q) {
    double v = std::hypot(det_grid[2 * q], det_grid[2 * q + 1]);
    if (std::isnan(v)) { best = q; break; }
    if (v < bv) { bv = v; best = q; }
  }
  int i = best % nG, j = best / nG;
  if (Op0) *Op0 = kls_lin(sc->Omega_p_min, sc->Omega_p_max, nO, j);
  if (g0) *g0 = kls_lin(sc->gamma_min, sc->gamma_max, nG, i);
  return KLS_OK;
}

int kls_newton(kls_ctx* c, double Op_init, double g_init, const kls_newton_cfg* nc,
               kls_newton_result* res, double* history) {
  KlsRange range("kls_newton");
  int r = check_ready(c);
  if (r) return r;
  if (!nc || !res || nc->max_iter < 1) return kls_fail(c, KLS_ERR_CONFIG, "bad Newton arguments");
  const double m = (double)c->cfg.m, tol = nc->tol, delta = nc->delta;
  double Op = Op_init, g = g_init;
  bool converged = false;
  int iteration = 0, evals = 0;
  double last_w[2] = {NAN, NAN}, last_det[2] = {NAN, NAN};
  auto det1 = [&](double wr, double wi, double* d) -> int {
    double w[2] = {wr, wi};
    int q = det_batch_host(c, w, 1, nc->mode, d, nullptr);
    if (q) return q;
    ++evals;
    last_w[0] = wr; last_w[1] = wi; last_det[0] = d[0]; last_det[1] = d[1];
    return KLS_OK;
  };
  std::memset(res, 0, sizeof *res);
  for (int it = 1; it <= nc->max_iter; ++it) {
    iteration = it;
    double d[2];
    if ((r = det1(m * Op, g, d))) return r;
    double F[2] = {d[0], d[1]};
    double rn = std::hypot(F[0], F[1]);
    if (history) {
      history[3 * (it - 1)] = Op;
      history[3 * (it - 1) + 1] = g;
      history[3 * (it - 1) + 2] = std::hypot(d[0], d[1]);
    }
    if (rn < tol) { converged = true; break; }
    // finite-difference Jacobian (NewtonSolver.jl:98-109): one batched launch
    double w2[4] = {m * (Op + delta), g, m * Op, g + delta}, d2[4];
    if ((r = det_batch_host(c, w2, 2, nc->mode, d2, nullptr))) return r;
    evals += 2;
    double J[2][2] = {{(d2[0] - d[0]) / delta, (d2[2] - d[0]) / delta},
                      {(d2[1] - d[1]) / delta, (d2[3] - d[1]) / delta}};
    double x[2];
    if (!solve2(J, F, x)) {
      res->Omega_p = Op; res->gamma = g; res->iterations = iteration; res->converged = 0;
      res->det_evals = evals;
      return kls_fail(c, KLS_ERR_SINGULAR, "singular finite-difference Jacobian");
    }
    double dx0 = -x[0], dx1 = -x[1];
    if (nc->use_line_search) {
      double a = 1.0;
      for (int ls = 1; ls <= nc->max_line_search; ++ls) {
        double Opn = Op + a * dx0, gn = g + a * dx1;
        if (gn < 1e-4 || Opn < 0.0 || Opn > 1.0) { a *= 0.5; continue; }
        double dn[2];
        if ((r = det1(m * Opn, gn, dn))) return r;
        if (std::hypot(dn[0], dn[1]) < rn) { Op = Opn; g = gn; break; }
        a *= 0.5;
        if (ls == nc->max_line_search) { Op += dx0; g += dx1; }
      }
    } else {
      Op += dx0;
      g += dx1;
    }
    g = std::max(g, 1e-4);
    Op = std::min(std::max(Op, 0.0), 1.0);
  }
  // final evaluation (NewtonSolver.jl:160-161); the kernels are deterministic,
  // so an omega that was just evaluated is not recomputed
  double dfin[2];
  if (last_w[0] == m * Op && last_w[1] == g) {
    dfin[0] = last_det[0]; dfin[1] = last_det[1];
  } else if ((r = det1(m * Op, g, dfin))) {
    return r;
  }
  res->Omega_p = Op; res->gamma = g; res->omega_re = m * Op; res->omega_im = g;
  res->det_re = dfin[0]; res->det_im = dfin[1];
  res->iterations = iteration; res->converged = converged ? 1 : 0; res->det_evals = evals;
  return KLS_OK;
}

int kls_newton_hybrid(kls_ctx* c, double Op_init, double g_init, const kls_newton_cfg* nc,
                      const kls_hybrid_cfg* hc, kls_newton_result* res, int32_t* evals,
                      double* history) {
  KlsRange range("kls_newton_hybrid");
  int r = check_ready(c);
  if (r) return r;
  if (!nc || !hc || !res || hc->mixed_max_iter < 0 || hc->fp64_max_iter < 1 ||
      !(hc->mixed_delta > 0.0) || !(hc->anchor_radius > 0.0) || !(hc->far_step > 0.0))
    return kls_fail(c, KLS_ERR_CONFIG, "bad hybrid Newton arguments");
  using cplx = std::complex<double>;
  const double m = (double)c->cfg.m, tol = nc->tol;
  // omega = m Omega_p + i gamma, with the reference's clamps on (Omega_p, gamma)
  auto clamp = [&](cplx w) {
    const double Op = std::min(std::max(w.real() / m, 0.0), 1.0);
    return cplx(m * Op, std::max(w.imag(), 1e-4));
  };
  auto usable = [](cplx s) { return std::isfinite(std::abs(s)) && std::abs(s) > 0.0; };
  cplx w = clamp(cplx(m * Op_init, g_init));
  int n_mixed = 0, n_fp64 = 0, n_anch = 0, it_total = 0;
  std::memset(res, 0, sizeof *res);
  auto hist = [&](cplx at, double a) {
    if (history && it_total < nc->max_iter) {
      history[3 * it_total] = at.real() / m;
      history[3 * it_total + 1] = at.imag();
      history[3 * it_total + 2] = a;
    }
    ++it_total;
  };
  auto det = [&](const cplx* ws, int n, int mode, cplx* out) -> int {
    double in[4], o[4];
    for (int i = 0; i < n; ++i) { in[2 * i] = ws[i].real(); in[2 * i + 1] = ws[i].imag(); }
    int q = det_batch_host(c, in, n, mode, o, nullptr);
    if (q) return q;
    for (int i = 0; i < n; ++i) out[i] = cplx(o[2 * i], o[2 * i + 1]);
    (mode == KLS_MODE_MIXED ? n_mixed : mode == KLS_MODE_FP64 ? n_fp64 : n_anch) += n;
    return KLS_OK;
  };
  auto finish = [&](cplx at, cplx d, bool conv) {
    res->Omega_p = at.real() / m; res->gamma = at.imag();
    res->omega_re = at.real(); res->omega_im = at.imag();
    res->det_re = d.real(); res->det_im = d.imag();
    res->iterations = it_total;
    res->converged = conv ? 1 : 0;
    res->det_evals = n_mixed + n_fp64 + n_anch;
    if (evals) { evals[0] = n_mixed; evals[1] = n_fp64; evals[2] = n_anch; }
  };
  // det(I - M(omega)) is holomorphic in omega, so one complex slope S =
  // d det / d omega gives the whole 2x2 finite-difference Jacobian of the
  // reference (dF/dOmega_p = m S, dF/dgamma = i S) and the Newton step is
  // delta omega = -det / S.
  // Steps are taken as the reference takes them (NewtonSolver.jl:66-161:
  // every step accepted, no line search), except that a step of the noise
  // scale that does not lower |det| ends a phase: there the determinant's
  // rounding, not the root, decides the direction.
  const double noise_step = 1e-4;
  // ---- phase 1: split-BF16 secant iteration, with far steps of FP64
  //      accuracy while the Newton step is longer than far_step
  const double h = m * hc->mixed_delta;
  cplx S, f;
  {
    const cplx ws[2] = {w, w + h};
    cplx d[2];
    if ((r = det(ws, 2, KLS_MODE_MIXED, d))) return r;
    hist(w, std::abs(d[0]));
    f = d[0];
    S = (d[1] - d[0]) / h;
  }
  bool haveS = usable(S);
  // far step at w: det at an FP64 anchor, slope by an anchored forward
  // difference (step m * nc->delta, the reference's Jacobian step); leaves
  // f = FP64 det at w, S = that slope
  auto far_slope = [&]() -> int {
    double d2[2];
    int q = kls_set_anchor(c, w.real(), w.imag(), d2);
    if (q) return q;
    ++n_fp64;
    f = cplx(d2[0], d2[1]);
    hist(w, std::abs(f));
    const cplx wd = w + m * nc->delta;
    cplx fd;
    if ((q = det(&wd, 1, KLS_MODE_ANCHORED, &fd))) return q;
    S = (fd - f) / (m * nc->delta);
    haveS = usable(S);
    return KLS_OK;
  };
  bool fp64_f = false;                           // f is of FP64 accuracy (a far step's)
  for (int it = 0; haveS && it < hc->mixed_max_iter + hc->fp64_max_iter; ++it) {
    if (std::abs(f / S) > hc->far_step) {
      if (!fp64_f && (r = far_slope())) return r;
      if (!haveS) break;
      fp64_f = true;
      if (std::abs(f) < tol) break;
      const cplx wn = clamp(w - f / S);
      if (wn == w) break;
      w = wn;
      if ((r = far_slope())) return r;         // det and slope at the new point
      continue;
    }
    if (fp64_f) {                                // back to the split form at w
      if ((r = det(&w, 1, KLS_MODE_MIXED, &f))) return r;
      hist(w, std::abs(f));
      fp64_f = false;
    }
    const cplx wn = clamp(w - f / S);
    const double step = std::abs(wn - w);
    if (step < hc->mixed_step_tol) {             // below the split form's resolution
      w = wn;
      break;
    }
    cplx fn;
    if ((r = det(&wn, 1, KLS_MODE_MIXED, &fn))) return r;
    hist(wn, std::abs(fn));
    if (!(std::abs(fn) < std::abs(f)) && step < noise_step) break;   // noise floor: stay at w
    const cplx Sn = (fn - f) / (wn - w);
    w = wn;
    f = fn;
    if (usable(Sn)) S = Sn;
  }
  // ---- phase 2: FP64 anchor, then anchored determinants
  cplx wa = w;
  if (!fp64_f) {                                 // (a far step left its anchor at w)
    double d2[2];
    if ((r = kls_set_anchor(c, w.real(), w.imag(), d2))) return r;
    ++n_fp64;
    f = cplx(d2[0], d2[1]);
    hist(w, std::abs(f));
  }
  // a determinant of FP64 accuracy at wn: anchored near the anchor, else a
  // new anchor there
  auto eval2 = [&](cplx wn, cplx* out) -> int {
    if (std::abs(wn - wa) > hc->anchor_radius) {
      double d2[2];
      int q = kls_set_anchor(c, wn.real(), wn.imag(), d2);
      if (q) return q;
      ++n_fp64;
      wa = wn;
      *out = cplx(d2[0], d2[1]);
      return KLS_OK;
    }
    return det(&wn, 1, KLS_MODE_ANCHORED, out);
  };
  bool converged = false, fresh = false;
  for (int it = 0; it < hc->fp64_max_iter; ++it) {
    if (!haveS) {                                  // forward-difference slope at w
      const cplx wd = w + m * nc->delta;
      cplx fd;
      if ((r = eval2(wd, &fd))) return r;
      S = (fd - f) / (m * nc->delta);
      haveS = fresh = true;
    }
    if (!usable(S)) {
      finish(w, f, false);
      return kls_fail(c, KLS_ERR_SINGULAR, "singular Jacobian in the FP64-anchored phase");
    }
    const cplx wn = clamp(w - f / S);
    const double step = std::abs(wn - w);
    if (std::abs(f) < tol && step <= 1e-11) { converged = true; break; }
    if (wn == w) break;                            // clamped in place
    cplx fn;
    if ((r = eval2(wn, &fn))) return r;
    hist(wn, std::abs(fn));
    if (std::abs(fn) < std::abs(f) || step >= noise_step) {
      // accepted (a long step is accepted even if |det| grows, as the
      // reference accepts every step); secant slope after a short step, a
      // fresh forward difference at the new point after a long one
      const cplx Sn = (fn - f) / (wn - w);
      w = wn;
      f = fn;
      if (step < noise_step && usable(Sn)) {
        S = Sn;
        fresh = false;
      } else {
        haveS = false;
      }
      continue;
    }
    if (std::abs(f) < tol) { converged = true; break; }   // |det| stopped falling below tol
    if (fresh) break;                              // a fresh slope did not help either
    haveS = false;
  }
  if (hc->final_fp64) {
    if ((r = det(&w, 1, KLS_MODE_FP64, &f))) return r;
    converged = std::abs(f) < tol;
  }
  finish(w, f, converged);
  return KLS_OK;
}

// ---- autotuner ------------------------------------------------------------------
namespace {

std::mutex g_tune_mu;
std::map<std::string, std::pair<int, int>> g_tune;   // key -> (splits, mixed form)
bool g_tune_loaded = false;

std::string tune_key(const kls_ctx* c, int mode, int batch) {
  cudaDeviceProp p;
  std::string dev = "gpu";
  if (cudaGetDeviceProperties(&p, c->device) == cudaSuccess) dev = p.name;
  for (char& ch : dev)
    if (ch == ' ') ch = '_';
  std::ostringstream o;
  o << dev << "|" << mode << "|" << c->Na_pad << "|" << c->K_pad << "|" << batch;
  return o.str();
}

// cache file lines: "<key> <splits> <form>"
void tune_load_file() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("KLS_TUNE_CACHE");
  if (!path || !*path) return;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream in(line);
    std::string key;
    int s = 0, form = 0;
    if (in >> key >> s && s > 0) {
      if (!(in >> form)) form = 0;
      g_tune[key] = std::make_pair(s, form);
    }
  }
}

void tune_store(const std::string& key, int s, int form) {
  g_tune[key] = std::make_pair(s, form);
  const char* path = std::getenv("KLS_TUNE_CACHE");
  if (!path || !*path) return;
  std::ofstream f(path, std::ios::app);
  f << key << " " << s << " " << form << "\n";
}

int apply_splits(kls_ctx* c, int mode, int s) {
  if (mode == KLS_MODE_FP64) {
    if (c->splits != s) {
      c->splits = s;
      c->ws_omega = 0;            // the next batch reallocates the partials
    }
    return KLS_OK;
  }
  return kls_mixed_set_splits(c, s);
}

// contraction time per omega (ms) at the context's current split count
int time_contraction(kls_ctx* c, int mode, int n, double* ms) {
  int r;
  if ((r = ensure_ws(c, n))) return r;
  std::vector<double> om(2 * (size_t)n);
  for (int z = 0; z < n; ++z) {
    om[2 * z] = c->cfg.m * (0.3 + 0.3 * z / std::max(1, n));
    om[2 * z + 1] = 0.02 + 0.2 * z / std::max(1, n);
  }
  KLS_CK(c, cudaMemcpyAsync(c->d_omega, om.data(), om.size() * sizeof(double),
                            cudaMemcpyHostToDevice, c->stream));
  if ((r = kls_run_weights(c, n))) return r;
  auto once = [&]() -> int {
    return mode == KLS_MODE_FP64 ? kls_run_contract_f64(c, n, c->splits)
                                 : kls_mixed_contract(c, n, 0);
  };
  if ((r = once())) return r;               // warm-up (and workspace growth)
  cudaEvent_t e0, e1;
  KLS_CK(c, cudaEventCreate(&e0));
  KLS_CK(c, cudaEventCreate(&e1));
  const int reps = 3;
  cudaEventRecord(e0, c->stream);
  for (int i = 0; i < reps && !r; ++i) r = once();
  cudaEventRecord(e1, c->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  if (e != cudaSuccess) return kls_cuda_fail(c, e, "autotune timing");
  if (mode == KLS_MODE_MIXED && (r = kls_mixed_check(c))) return r;
  *ms = t / reps / n;
  return KLS_OK;
}

}  // namespace

int kls_autotune(kls_ctx* c, int mode, int batch, kls_tune_result* out) {
  KlsRange range("kls_autotune");
  int r = check_ready(c);
  if (r) return r;
  if (mode != KLS_MODE_FP64 && mode != KLS_MODE_MIXED)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown precision mode");
  if (batch < 1 || batch > WS_CHUNK) return kls_fail(c, KLS_ERR_CONFIG, "bad autotune batch");
  if (mode == KLS_MODE_FP64 && !c->d_Wre)
    return kls_fail(c, KLS_ERR_STATE, "the FP64 table was released (kls_release_fp64)");
  if (mode == KLS_MODE_MIXED && !c->mixed && (r = kls_mixed_prepare(c))) return r;
  const bool mixed = mode == KLS_MODE_MIXED;
  const int def = mixed ? kls_mixed_default_splits(c) : kls_choose_splits(c);
  const int def_form = mixed ? kls_mixed_form_of(c) : c->f64_form;
  const int max_s = mixed ? (int)std::max<int64_t>(1, c->K_pad / 64)
                          : (int)std::max<int64_t>(1, c->K_pad / (16 * 8));
  auto apply = [&](int s, int form) -> int {
    if (mixed && (r = kls_mixed_set_form(c, form))) return r;
    if (!mixed) c->f64_form = form;
    return apply_splits(c, mode, s);
  };
  kls_tune_result res{};
  res.mode = mode;
  res.default_splits = def;
  const std::string key = tune_key(c, mode, batch);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load_file();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      res.splits = std::min(it->second.first, max_s);
      res.form = mixed ? (it->second.second ? it->second.second : def_form) : it->second.second;
      if ((r = apply(res.splits, res.form))) return r;
      if (out) *out = res;
      return KLS_OK;
    }
  }
  // each mode also chooses its kernel: one CTA, a CTA pair or the
  // TMEM-operand pair (split-BF16), 4 or 3 real products (FP64); split
  // candidates around each form's own default
  std::vector<int> forms = mixed ? std::vector<int>{KLS_MIXED_ONE_CTA, KLS_MIXED_PAIR}
                                 : std::vector<int>{KLS_F64_4M, KLS_F64_3M};
  if (mixed && kls_mixed_set_form(c, KLS_MIXED_TMEM) == KLS_OK) forms.push_back(KLS_MIXED_TMEM);
  if (mixed) kls_mixed_set_form(c, def_form);
  double best_ms = INFINITY;
  int best = def, best_form = def_form;
  for (int form : forms) {
    int fdef = def;
    if (mixed) {
      if ((r = kls_mixed_set_form(c, form))) return r;
      fdef = kls_mixed_default_splits(c);
    } else {
      c->f64_form = form;
      fdef = kls_choose_splits(c);
    }
    std::vector<int> cand = {std::max(1, fdef / 2), fdef, 2 * fdef, 3 * fdef};
    // the TMEM-operand form's default is the number of resident CTA pairs:
    // fewer splits leave a single omega (Newton's evaluations) on part of a
    // wave, so only whole multiples of it are candidates
    if (mixed && form == KLS_MIXED_TMEM) {
      cand = {fdef};
      // more splits only while the FP64 partials of `batch` omegas stay within
      // 2 GiB (batch x N_pad/64 tiles x splits x N_pad x 128 doubles): an
      // uneven batch of many default-size models holds one such buffer each
      const double per_split = (double)batch * (c->Na_pad / 64) * c->Na_pad * 128 * 8;
      for (int k = 2; k <= 3; ++k)
        if (per_split * k * fdef <= 2.0 * 1024 * 1024 * 1024) cand.push_back(k * fdef);
    }
    for (int& s : cand) s = std::max(1, std::min(s, max_s));
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    for (int s : cand) {
      if ((r = apply(s, form))) return r;
      double ms = 0.0;
      if ((r = time_contraction(c, mode, batch, &ms))) return r;
      if (s == def && form == def_form) res.default_ms_per_omega = ms;
      if (ms < best_ms) {
        best_ms = ms;
        best = s;
        best_form = form;
      }
      res.candidates++;
    }
  }
  if ((r = apply(best, best_form))) return r;
  res.splits = best;
  res.form = best_form;
  res.ms_per_omega = best_ms;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_store(key, best, best_form);
  }
  if (out) *out = res;
  return KLS_OK;
}

int kls_set_splits(kls_ctx* c, int mode, int splits) {
  int r = check_ready(c);
  if (r) return r;
  if (splits < 1) return kls_fail(c, KLS_ERR_CONFIG, "splits must be >= 1");
  if (mode == KLS_MODE_FP64) {
    const int max_s = (int)std::max<int64_t>(1, c->K_pad / (16 * 8));
    return apply_splits(c, mode, std::min(splits, max_s));
  }
  if (mode != KLS_MODE_MIXED) return kls_fail(c, KLS_ERR_CONFIG, "unknown precision mode");
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  return apply_splits(c, mode, splits);
}

int kls_set_mixed_form(kls_ctx* c, int form) {
  int r = check_ready(c);
  if (r) return r;
  if (form != KLS_MIXED_AUTO && form != KLS_MIXED_ONE_CTA && form != KLS_MIXED_PAIR &&
      form != KLS_MIXED_TMEM)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown mixed contraction form");
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  if (form == KLS_MIXED_AUTO)
    form = kls_mixed_set_form(c, KLS_MIXED_TMEM) == KLS_OK ? KLS_MIXED_TMEM : KLS_MIXED_ONE_CTA;
  return kls_mixed_set_form(c, form);
}

int kls_set_mixed_chunk(kls_ctx* c, int k_blocks) {
  int r = check_ready(c);
  if (r) return r;
  if (k_blocks < 1 || k_blocks > 1 << 20)
    return kls_fail(c, KLS_ERR_CONFIG, "chunk must be in [1, 2^20] k-blocks");
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  return kls_mixed_set_chunk(c, k_blocks);
}

int kls_set_wait_limit(kls_ctx* c, double seconds) {
  int r = check_ready(c);
  if (r) return r;
  if (!(seconds > 0.0) || seconds > 60.0)
    return kls_fail(c, KLS_ERR_CONFIG, "wait limit must be in (0, 60] seconds");
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  return kls_mixed_set_wait(c, (unsigned long long)(seconds * 1e9), -1);
}

int kls_set_fault_injection(kls_ctx* c, int mode) {
  int r = check_ready(c);
  if (r) return r;
  if (mode < KLS_FAULT_NONE || mode > KLS_FAULT_NAN_ROW)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown fault injection mode");
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  if (mode == KLS_FAULT_NAN_ROW) {
    if (!c->gk0_poisoned) {
      KLS_CK(c, cudaMemcpy(&c->gk0_saved, c->d_Gk, sizeof(double), cudaMemcpyDeviceToHost));
      const double nan = NAN;
      KLS_CK(c, cudaMemcpy(c->d_Gk, &nan, sizeof(double), cudaMemcpyHostToDevice));
      c->gk0_poisoned = true;
    }
    return KLS_OK;
  }
  if (mode == KLS_FAULT_NONE) {
    if (c->gk0_poisoned) {
      KLS_CK(c, cudaMemcpy(c->d_Gk, &c->gk0_saved, sizeof(double), cudaMemcpyHostToDevice));
      c->gk0_poisoned = false;
    }
    return c->mixed ? kls_mixed_set_wait(c, 0, KLS_FAULT_NONE) : KLS_OK;
  }
  if (!c->mixed && (r = kls_mixed_prepare(c))) return r;
  return kls_mixed_set_wait(c, 0, mode);
}

int kls_set_f64_form(kls_ctx* c, int form) {
  int r = check_ready(c);
  if (r) return r;
  if (form != KLS_F64_4M && form != KLS_F64_3M)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown FP64 contraction form");
  if (c->f64_form != form) {
    c->f64_form = form;
    return apply_splits(c, KLS_MODE_FP64, kls_choose_splits(c));
  }
  return KLS_OK;
}

int kls_set_lu_mode(kls_ctx* c, int mode) {
  if (!c) return KLS_ERR_CONFIG;
  if (mode != KLS_LU_AUTO && mode != KLS_LU_CTA && mode != KLS_LU_CLUSTER)
    return kls_fail(c, KLS_ERR_CONFIG, "unknown LU mode");
  c->lu_mode = mode;
  return KLS_OK;
}

int kls_enable_timing(kls_ctx* c, int on) {
  if (!c) return KLS_ERR_CONFIG;
  c->timing = on != 0;
  return KLS_OK;
}

int kls_get_precompute_ms(kls_ctx* c, float* ms2) {
  if (!c || !ms2) return KLS_ERR_CONFIG;
  ms2[0] = c->pre_ms[0];
  ms2[1] = c->pre_ms[1];
  return KLS_OK;
}

int kls_get_stage_ms(kls_ctx* c, float* ms4) {
  if (!c || !ms4) return KLS_ERR_CONFIG;
  for (int i = 0; i < 4; ++i) ms4[i] = c->stage_ms[i];
  return KLS_OK;
}

int64_t kls_launch_count(const kls_ctx* c) { return c ? c->launches : 0; }

int kls_bounds_report(int64_t* violations, int32_t* first_site, int64_t* first_index,
                      int64_t* first_extent, int reset) {
#ifdef KLS_CHECKED
  int64_t n = 0, idx = 0, ext = 0;
  int32_t site = 0;
  for (auto rd : bounds_readers()) {
    KlsBoundsLog l{};
    if (rd(&l, reset != 0))
      return kls_fail(nullptr, KLS_ERR_CUDA, "kls_bounds_report: a device log could not be read");
    if (l.count && !n) {
      site = l.site;
      idx = l.index;
      ext = l.extent;
    }
    n += (int64_t)l.count;
  }
  if (violations) *violations = n;
  if (first_site) *first_site = site;
  if (first_index) *first_index = idx;
  if (first_extent) *first_extent = ext;
  return KLS_OK;
#else
  (void)violations; (void)first_site; (void)first_index; (void)first_extent; (void)reset;
  return kls_fail(nullptr, KLS_ERR_UNSUPPORTED,
                  "kls_bounds_report: this library is the default build; the bounds-checked "
                  "build is libkls_checked.so");
#endif
}

}  // extern "C"

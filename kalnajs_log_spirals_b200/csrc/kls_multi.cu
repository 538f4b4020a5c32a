// Uneven batch: det(I - M(omega)) for many disk models of different sizes in
// shared launches (no reference counterpart as one launch: the reference runs
// grid_scan once per model, and its multi-GPU scan, GridScan.jl:125-197,
// splits one model's omega columns over devices).
//
// Every model keeps its own context (tables on the device); a kls_multi adds
// per-omega buffers for a fixed batch of omegas per model and device-resident
// descriptors (kls_mdesc), and lists the contraction's work items over all
// models.  One batch is
//
//   H2D omegas -> weights (all models) -> persistent contraction (all models)
//   -> split reduction (all models) -> LU (all models) -> D2H dets
//
// captured once into a CUDA graph and replayed for every chunk of omegas.
// The FP64 contraction takes items from an atomic counter in list order; for
// the mixed one the batch times one pass with each of two schedules of the
// same list (a persistent round robin, one CTA per item) and keeps the faster.  Each model's K split count is its context's own
// (kls_autotune chooses it), so a determinant from the batch is bitwise the
// one kls_det_batch returns for the same context.  When every model's
// split-BF16 form is the TMEM-operand one, the contraction is that form's
// kernel body driven by per-model descriptors, one CTA pair per (model, tile
// pair, K split); otherwise the one-CTA form's body.
#include "kls_internal.cuh"
#include <cuda.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <vector>

struct kls_multi {
  int device = 0, mode = 0, batch = 0, n_models = 0;
  int f64_form = KLS_F64_4M;        // FP64: every model's contraction form
  std::vector<kls_ctx*> ctx;
  cudaStream_t stream = nullptr;
  std::string err;

  std::vector<kls_mdesc> md;
  std::vector<kls_item> items;
  std::vector<kls_item> list;       // mixed: items in locality order
  std::vector<int> starts;          // mixed: per-CTA item ranges
  int schedule = 0;                 // mixed: 0 persistent round robin, 1 one CTA (pair) per
                                    // item, 2 (TMEM form) one launch per model
  bool tm = false;                  // mixed: some model in the TMEM-operand form
  bool old = false;                 // mixed: some model in the one-CTA / pair forms
  std::vector<char> use_tm;         // per model: TMEM-operand form
  std::vector<int2> pairs_tm, pairs_old;   // (model, omega) pairs of each form
  int2 *d_pairs_tm = nullptr, *d_pairs_old = nullptr;
  int tm_schedule = 1;              // TMEM form: 1 one launch over items, 2 one per model
  double tm_schedule_ms[2] = {0, 0};
  std::vector<kls_tm_model> tmd;    // its per-model descriptors
  std::vector<int4> tm_items;       // (model, tile pair, split): one CTA pair each
  kls_tm_model* d_tm = nullptr;
  int4* d_tm_items = nullptr;
  int max_Npad = 0;
  double schedule_ms[2] = {0, 0};   // mixed: eager-pass time of each schedule
  std::vector<int2> pairs;          // (model, omega) pairs
  int grid = 0, max_Na = 0;
  int64_t max_K_pad = 0;

  kls_mdesc* d_md = nullptr;
  kls_item* d_items = nullptr;
  int* d_starts = nullptr;
  int2* d_pairs = nullptr;
  int* d_counter = nullptr;
  int* d_err = nullptr;
  uint8_t* d_tmaps = nullptr;       // 2 CUtensorMap per model
  double* d_omega = nullptr;        // [n_models][batch][2]
  double2* d_det = nullptr;         // [n_models][batch]
  double* d_logabs = nullptr;
  std::vector<void*> bufs;          // per-model buffers to free

  double* h_omega = nullptr;        // pinned [n_models][batch][2]
  double* h_det = nullptr;          // pinned [n_models][batch][2]
  double* h_logabs = nullptr;       // pinned [n_models][batch]
  int* h_err = nullptr;             // pinned

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t replays = 0;
  float last_ms = 0.f;
};

namespace {

thread_local std::string g_multi_create_err;

int mfail(kls_multi* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  else g_multi_create_err = msg;
  return code;
}
int mcuda(kls_multi* m, cudaError_t e, const char* what) {
  return mfail(m, e == cudaErrorMemoryAllocation ? KLS_ERR_OOM : KLS_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}
#define KM_CK(m, call)                                          \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return mcuda((m), e_, #call);        \
  } while (0)

template <typename T>
int malloc_buf(kls_multi* m, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return mcuda(m, e, "cudaMalloc (uneven batch buffers)");
  }
  m->bufs.push_back(*p);
  return KLS_OK;
}

// mixed items: effective K splits so that every split owns >= 1 k-block
constexpr int MIX_BK = 64, MIX_BM = 128, MIX_AB = 64;

// Item order follows the one-model grids (tile fastest, then split, then
// omega), model after model with the largest models first: CTAs that run at
// the same time then work on the same k-range of one table, so its X and Y
// rows are read from DRAM once and reused from L2, as in the one-model launch.
int build_items(kls_multi* m) {
  m->items.clear();
  m->pairs.clear();
  m->pairs_tm.clear();
  m->pairs_old.clear();
  for (int i = 0; i < m->n_models; ++i)
    for (int z = 0; z < m->batch; ++z) {
      m->pairs.push_back(make_int2(i, z));
      (m->use_tm[i] ? m->pairs_tm : m->pairs_old).push_back(make_int2(i, z));
    }
  if (m->mode != KLS_MODE_FP64 && !m->old) return KLS_OK;   // TMEM items: build_tm_items
  std::vector<int> order(m->n_models);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const kls_mdesc &x = m->md[a], &y = m->md[b];
    return (double)x.K_pad * x.Na_pad * x.Na_pad > (double)y.K_pad * y.Na_pad * y.Na_pad;
  });
  if (m->mode == KLS_MODE_FP64) {
    for (int i : order) {
      const kls_mdesc& d = m->md[i];
      const int tiles = (d.Na_pad / KLS_TILE) * (d.Na_pad / KLS_TILE);
      for (int z = 0; z < m->batch; ++z)
        for (int s = 0; s < d.splits; ++s)
          for (int t = 0; t < tiles; ++t) {
            int64_t kb = (int64_t)s * d.k_per_split;
            int64_t ke = std::min(d.K_pad, kb + d.k_per_split);
            m->items.push_back(kls_item{i, z, t, s, 1, 0, (int)std::max<int64_t>(0, ke - kb), 0});
          }
    }
    m->grid = std::max(1, std::min((int)m->items.size(), kls_multi_contract_slots(m->device, m->f64_form)));
    return KLS_OK;
  }
  m->list.clear();
  for (int i : order) {
    if (m->use_tm[i]) continue;           // in the TMEM-operand launch
    const kls_mdesc& d = m->md[i];
    const int tiles = (2 * d.Na_pad / MIX_BM) * (d.Na_pad / MIX_AB);
    for (int z = 0; z < m->batch; z += d.om_per_item) {
      const int n_om = std::min(d.om_per_item, m->batch - z);
      for (int s = 0; s < d.msplits; ++s)
        for (int t = 0; t < tiles; ++t) {
          const int kb0 = s * d.kb_per_split;
          const int nkb = std::min(d.nkb_total, kb0 + d.kb_per_split) - kb0;
          if (nkb <= 0) continue;
          m->list.push_back(kls_item{i, z, t, s, n_om, kb0, nkb, 0});
        }
    }
  }
  return KLS_OK;
}

// TMEM-operand form: one CTA pair per (model, tile pair, K split), model by
// model with the largest first, split-major so that pairs running together
// read the same k-range of one table.
void build_tm_items(kls_multi* m) {
  m->tm_items.clear();
  std::vector<int> order(m->tmd.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const kls_tm_model &x = m->tmd[a], &y = m->tmd[b];
    return (double)x.K_pad * x.Npad * x.Npad > (double)y.K_pad * y.Npad * y.Npad;
  });
  for (int i : order) {
    const kls_tm_model& d = m->tmd[i];
    const int pairs = (d.n_tiles + 1) / 2;
    for (int s = 0; s < d.splits; ++s)
      for (int p = 0; p < pairs; ++p) m->tm_items.push_back(make_int4(i, p, s, 0));
  }
  m->tm_schedule = 1;
}

// Mixed form: per-CTA item ranges of the ordered list.  Schedule 0: a
// persistent grid of one CTA per SM, CTA b taking items b, b + grid, ...;
// schedule 1: one CTA per item (the hardware block scheduler hands items to
// SMs as they free up, in list order).
int schedule_items(kls_multi* m, int policy) {
  const int n = (int)m->list.size();
  m->items.clear();
  if (policy == 0) {
    const int grid = std::max(1, std::min(n, kls_mixed_slots(m->device)));
    m->starts.assign(grid + 1, 0);
    for (int b = 0; b < grid; ++b) {
      m->starts[b] = (int)m->items.size();
      for (int k = b; k < n; k += grid) m->items.push_back(m->list[k]);
    }
    m->starts[grid] = (int)m->items.size();
    m->grid = grid;
  } else {
    m->items = m->list;
    m->starts.resize(n + 1);
    std::iota(m->starts.begin(), m->starts.end(), 0);
    m->grid = std::max(1, n);
  }
  m->schedule = policy;
  if (cudaMemcpy(m->d_items, m->items.data(), m->items.size() * sizeof(kls_item),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->d_starts, m->starts.data(), m->starts.size() * sizeof(int),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return mcuda(m, cudaGetLastError(), "cudaMemcpy (schedule)");
  return KLS_OK;
}

int launch_batch(kls_multi* m) {
  int r;
  const int np = (int)m->pairs.size();
  if (m->mode == KLS_MODE_FP64) {
    r = kls_multi_launch_f64(m->stream, m->d_md, m->d_pairs, np, m->d_items, (int)m->items.size(),
                             m->d_counter, m->grid, m->max_K_pad, m->f64_form);
  } else {
    // the mixed weights are converted from the FP64 weights of the same pass
    r = kls_multi_launch_f64_weights(m->stream, m->d_md, m->d_pairs, np, m->max_K_pad);
    if (!r && m->tm)
      r = kls_tm_multi_launch(m->stream, m->d_md, m->d_tm, m->d_pairs_tm, (int)m->pairs_tm.size(),
                              m->d_tm_items, (int)m->tm_items.size(), m->max_K_pad, m->max_Npad,
                              m->d_err, m->tmd.data(), (int)m->tmd.size(), m->tm_schedule == 2);
    if (!r && m->old)
      r = kls_multi_launch_mixed(m->stream, m->d_md, m->d_pairs_old, (int)m->pairs_old.size(),
                                 m->d_items, m->d_starts, m->grid, m->max_K_pad, m->d_err);
  }
  if (r) return mcuda(m, (cudaError_t)r, "uneven batch launch");
  r = kls_multi_launch_lu(m->stream, m->d_md, m->d_pairs, np, m->max_Na);
  if (r) return mcuda(m, (cudaError_t)r, "uneven batch LU launch");
  return KLS_OK;
}

// One eager pass (kernel attributes are set outside any capture and the
// launch shapes are checked); *ms = its device time.
int eager_pass(kls_multi* m, float* ms) {
  const size_t nz = (size_t)m->n_models * m->batch;
  for (int i = 0; i < m->n_models; ++i)
    for (int z = 0; z < m->batch; ++z) {
      m->h_omega[2 * ((size_t)i * m->batch + z)] = m->ctx[i]->cfg.m * 0.4;
      m->h_omega[2 * ((size_t)i * m->batch + z) + 1] = 0.1;
    }
  KM_CK(m, cudaMemcpyAsync(m->d_omega, m->h_omega, nz * 2 * sizeof(double),
                           cudaMemcpyHostToDevice, m->stream));
  KM_CK(m, cudaEventRecord(m->ev0, m->stream));
  int r = launch_batch(m);
  if (r) return r;
  KM_CK(m, cudaEventRecord(m->ev1, m->stream));
  KM_CK(m, cudaMemcpyAsync(m->h_err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  KM_CK(m, cudaStreamSynchronize(m->stream));
  if (*m->h_err)
    return mfail(m, KLS_ERR_CUDA,
                 "mixed contraction pipeline timed out (code " + std::to_string(*m->h_err) + ")");
  if (ms) KM_CK(m, cudaEventElapsedTime(ms, m->ev0, m->ev1));
  return KLS_OK;
}

// H2D omegas, the batch, D2H results: recorded once into a graph
int capture(kls_multi* m) {
  const size_t nz = (size_t)m->n_models * m->batch;
  int r = KLS_OK;
  KM_CK(m, cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemcpyAsync(m->d_omega, m->h_omega, nz * 2 * sizeof(double),
                                  cudaMemcpyHostToDevice, m->stream);
  if (e != cudaSuccess) r = mcuda(m, e, "cudaMemcpyAsync (omegas)");
  if (!r) r = launch_batch(m);
  if (!r && (e = cudaMemcpyAsync(m->h_det, m->d_det, nz * sizeof(double2), cudaMemcpyDeviceToHost,
                                 m->stream)) != cudaSuccess)
    r = mcuda(m, e, "cudaMemcpyAsync (dets)");
  if (!r && (e = cudaMemcpyAsync(m->h_logabs, m->d_logabs, nz * sizeof(double),
                                 cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess)
    r = mcuda(m, e, "cudaMemcpyAsync (log|det|)");
  if (!r && (e = cudaMemcpyAsync(m->h_err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                                 m->stream)) != cudaSuccess)
    r = mcuda(m, e, "cudaMemcpyAsync (error flag)");
  cudaGraph_t g = nullptr;
  cudaError_t ee = cudaStreamEndCapture(m->stream, &g);
  if (r) {
    if (g) cudaGraphDestroy(g);
    return r;
  }
  if (ee != cudaSuccess) return mcuda(m, ee, "cudaStreamEndCapture");
  m->graph = g;
  KM_CK(m, cudaGraphInstantiate(&m->exec, g, 0));
  return KLS_OK;
}

int replay(kls_multi* m) {
  KM_CK(m, cudaEventRecord(m->ev0, m->stream));
  KM_CK(m, cudaGraphLaunch(m->exec, m->stream));
  KM_CK(m, cudaEventRecord(m->ev1, m->stream));
  KM_CK(m, cudaStreamSynchronize(m->stream));
  KM_CK(m, cudaEventElapsedTime(&m->last_ms, m->ev0, m->ev1));
  m->replays++;
  if (*m->h_err) {
    int code = *m->h_err;
    *m->h_err = 0;
    cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream);
    cudaStreamSynchronize(m->stream);
    return mfail(m, KLS_ERR_CUDA,
                 "mixed contraction pipeline timed out (code " + std::to_string(code) + ")");
  }
  return KLS_OK;
}

// omegas for model i (n of them, interleaved) -> results, chunked by batch
int run_omegas(kls_multi* m, const std::function<void(int, int, double*)>& fill, int n,
               double* det_ri, double* log_abs) {
  const int B = m->batch;
  for (int b0 = 0; b0 < n; b0 += B) {
    const int nb = std::min(B, n - b0);
    for (int i = 0; i < m->n_models; ++i) {
      double* o = m->h_omega + (size_t)i * B * 2;
      for (int z = 0; z < B; ++z) fill(i, b0 + std::min(z, nb - 1), o + 2 * z);
      for (int z = 0; z < 2 * B; ++z)
        if (!std::isfinite(o[z])) return mfail(m, KLS_ERR_NONFINITE, "non-finite omega");
    }
    int r = replay(m);
    if (r) return r;
    for (int i = 0; i < m->n_models; ++i)
      for (int z = 0; z < nb; ++z) {
        const size_t src = (size_t)i * B + z, dst = (size_t)i * n + b0 + z;
        det_ri[2 * dst] = m->h_det[2 * src];
        det_ri[2 * dst + 1] = m->h_det[2 * src + 1];
        if (log_abs) log_abs[dst] = m->h_logabs[src];
      }
  }
  return KLS_OK;
}

void release(kls_multi* m) {
  if (m->exec) cudaGraphExecDestroy(m->exec);
  if (m->graph) cudaGraphDestroy(m->graph);
  for (void* p : m->bufs) cudaFree(p);
  m->bufs.clear();
  if (m->h_omega) cudaFreeHost(m->h_omega);
  if (m->h_det) cudaFreeHost(m->h_det);
  if (m->h_logabs) cudaFreeHost(m->h_logabs);
  if (m->h_err) cudaFreeHost(m->h_err);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
}

}  // namespace

extern "C" {

const char* kls_multi_last_error(const kls_multi* m) {
  return m ? m->err.c_str() : g_multi_create_err.c_str();
}

int kls_multi_create(kls_ctx* const* models, int n_models, int mode, int batch, kls_multi** out) {
  if (!out) return mfail(nullptr, KLS_ERR_CONFIG, "null output handle");
  *out = nullptr;
  if (!models || n_models < 1 || batch < 1 || batch > 4096)
    return mfail(nullptr, KLS_ERR_CONFIG, "need >= 1 model and 1 <= batch <= 4096");
  if (mode != KLS_MODE_FP64 && mode != KLS_MODE_MIXED)
    return mfail(nullptr, KLS_ERR_CONFIG, "unknown precision mode");
  for (int i = 0; i < n_models; ++i) {
    if (!models[i] || !models[i]->precomputed)
      return mfail(nullptr, KLS_ERR_STATE, "model " + std::to_string(i) + " is not precomputed");
    if (models[i]->device != models[0]->device)
      return mfail(nullptr, KLS_ERR_CONFIG, "all models of a batch must be on one device");
    if (mode == KLS_MODE_FP64 && !models[i]->d_Wre)
      return mfail(nullptr, KLS_ERR_STATE,
                   "model " + std::to_string(i) + ": the FP64 table was released");
    if (mode == KLS_MODE_FP64 && models[i]->f64_form != models[0]->f64_form)
      return mfail(nullptr, KLS_ERR_CONFIG, "FP64 models of a batch need one contraction form");
  }
  kls_multi* m = new kls_multi();
  m->device = models[0]->device;
  m->mode = mode;
  m->f64_form = models[0]->f64_form;
  m->batch = batch;
  m->n_models = n_models;
  m->ctx.assign(models, models + n_models);
  int r = KLS_OK;
  auto bail = [&](int code) {
    g_multi_create_err = m->err;
    release(m);
    delete m;
    return code;
  };
  if (cudaSetDevice(m->device) != cudaSuccess) return bail(mcuda(m, cudaGetLastError(), "cudaSetDevice"));
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&m->ev0) != cudaSuccess || cudaEventCreate(&m->ev1) != cudaSuccess)
    return bail(mcuda(m, cudaGetLastError(), "stream/event creation"));
  const size_t nz = (size_t)n_models * batch;
  if ((r = malloc_buf(m, &m->d_omega, 2 * nz)) || (r = malloc_buf(m, &m->d_det, nz)) ||
      (r = malloc_buf(m, &m->d_logabs, nz)) || (r = malloc_buf(m, &m->d_counter, 1)) ||
      (r = malloc_buf(m, &m->d_err, 1)) ||
      (r = malloc_buf(m, &m->d_tmaps, (size_t)2 * n_models * sizeof(CUtensorMap))))
    return bail(r);
  if (cudaMallocHost(&m->h_omega, 2 * nz * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&m->h_det, 2 * nz * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&m->h_logabs, nz * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&m->h_err, sizeof(int)) != cudaSuccess)
    return bail(mcuda(m, cudaErrorMemoryAllocation, "cudaMallocHost"));
  *m->h_err = 0;
  std::fill(m->h_omega, m->h_omega + 2 * nz, 0.0);
  if (cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess)
    return bail(mcuda(m, cudaGetLastError(), "cudaMemset"));

  m->md.resize(n_models);
  m->use_tm.assign(n_models, 0);
  if (mode == KLS_MODE_MIXED) {
    // each model runs its own form's kernel body: the models in the
    // TMEM-operand form share one contraction launch, the others (one-CTA or
    // pair form, which return the same bits) share the one-CTA kernel's
    for (int i = 0; i < n_models; ++i) {
      if (!models[i]->mixed && (r = kls_mixed_prepare(models[i])))
        return bail(mfail(m, r, models[i]->err));
      m->use_tm[i] = kls_mixed_tm_state(models[i], nullptr) != nullptr;
      if (m->use_tm[i]) m->tm = true;
      else m->old = true;
    }
  }
  for (int i = 0; i < n_models; ++i) {
    kls_ctx* c = models[i];
    kls_mdesc d{};
    d.Wre = c->d_Wre;
    d.Wim = c->d_Wim;
    d.Gk = c->d_Gk;
    d.Ok = c->d_Ok;
    d.Nk = c->d_N;
    d.omega = m->d_omega + (size_t)2 * i * batch;
    d.det = m->d_det + (size_t)i * batch;
    d.logabs = m->d_logabs + (size_t)i * batch;
    d.G = c->cfg.G;
    d.K_pad = c->K_pad;
    d.Na = c->Na;
    d.Na_pad = c->Na_pad;
    d.model = i;
    if ((r = malloc_buf(m, &d.wt, (size_t)batch * c->K_pad))) return bail(r);
    if ((r = malloc_buf(m, &d.A, (size_t)batch * c->Na * c->Na))) return bail(r);
    if (mode == KLS_MODE_FP64) {
      d.splits = c->splits;
      d.k_per_split = kls_f64_k_per_split(c->K_pad, c->splits);
      if ((r = malloc_buf(m, &d.part, (size_t)batch * d.splits * c->Na_pad * c->Na_pad)))
        return bail(r);
    } else {
      if (!c->mixed && (r = kls_mixed_prepare(c))) return bail(mfail(m, r, c->err));
      if (m->use_tm[i]) {
        // TMEM-operand form: FP32 weight variants and this form's partials
        unsigned long long wns = 0;
        kls_mixed_tm* t = kls_mixed_tm_state(c, &wns);
        kls_tm_model td;
        kls_tm_describe(c, t, wns, batch, &td);
        float2* w32 = nullptr;
        double* mp = nullptr;
        if ((r = malloc_buf(m, &w32, (size_t)batch * c->K_pad * KLS_TM_WVAR)) ||
            (r = malloc_buf(m, &mp, (size_t)td.n_tiles * td.splits * c->Na_pad * 128)))
          return bail(r);
        td.wt32 = w32;
        td.part = mp;
        m->tmd.push_back(td);
        d.wt32 = w32;
        d.mpart = mp;
        d.msplits = td.splits;
        m->md[i] = d;
        m->max_Na = std::max(m->max_Na, c->Na);
        m->max_K_pad = std::max(m->max_K_pad, c->K_pad);
        m->max_Npad = std::max(m->max_Npad, c->Na_pad);
        continue;
      }
      const void *xl = nullptr, *th = nullptr, *tl = nullptr;
      d.Xh = kls_mixed_tables(c, &xl, &th, &tl);
      d.Xl = xl;
      uint8_t* dm = m->d_tmaps + (size_t)2 * i * sizeof(CUtensorMap);
      if (cudaMemcpy(dm, th, sizeof(CUtensorMap), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dm + sizeof(CUtensorMap), tl, sizeof(CUtensorMap),
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(mcuda(m, cudaGetLastError(), "cudaMemcpy (tensor maps)"));
      d.tmap_h = dm;
      d.tmap_l = dm + sizeof(CUtensorMap);
      d.nkb_total = (int)(c->K_pad / MIX_BK);
      const int s = kls_mixed_legacy_splits(c);
      d.kb_per_split = (d.nkb_total + s - 1) / s;
      d.msplits = (d.nkb_total + d.kb_per_split - 1) / d.kb_per_split;   // non-empty splits
      d.om_per_item = 2;
      float2* w32 = nullptr;
      double* mp = nullptr;
      const size_t R = 2 * (size_t)c->Na_pad;
      if ((r = malloc_buf(m, &w32, (size_t)batch * c->K_pad)) ||
          (r = malloc_buf(m, &mp, (size_t)batch * d.msplits * R * R)))
        return bail(r);
      d.wt32 = w32;
      d.mpart = mp;
    }
    m->md[i] = d;
    m->max_Na = std::max(m->max_Na, c->Na);
    m->max_K_pad = std::max(m->max_K_pad, c->K_pad);
  }
  if (m->tm) {
    build_tm_items(m);
    if ((r = malloc_buf(m, &m->d_tm, m->tmd.size())) ||
        (r = malloc_buf(m, &m->d_tm_items, m->tm_items.size())))
      return bail(r);
    if (cudaMemcpy(m->d_tm, m->tmd.data(), m->tmd.size() * sizeof(kls_tm_model),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->d_tm_items, m->tm_items.data(), m->tm_items.size() * sizeof(int4),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(mcuda(m, cudaGetLastError(), "cudaMemcpy (TMEM-form descriptors)"));
  }
  if ((r = build_items(m))) return bail(r);
  const size_t n_it = std::max(m->items.size(), m->list.size());
  if ((r = malloc_buf(m, &m->d_md, m->md.size())) || (r = malloc_buf(m, &m->d_items, n_it)) ||
      (r = malloc_buf(m, &m->d_pairs, m->pairs.size())) ||
      (r = malloc_buf(m, &m->d_pairs_tm, m->pairs_tm.size())) ||
      (r = malloc_buf(m, &m->d_pairs_old, m->pairs_old.size())) ||
      (r = malloc_buf(m, &m->d_starts, n_it + 1)))
    return bail(r);
  if (cudaMemcpy(m->d_md, m->md.data(), m->md.size() * sizeof(kls_mdesc), cudaMemcpyHostToDevice) ||
      cudaMemcpy(m->d_pairs, m->pairs.data(), m->pairs.size() * sizeof(int2),
                 cudaMemcpyHostToDevice) ||
      cudaMemcpy(m->d_pairs_tm, m->pairs_tm.data(), m->pairs_tm.size() * sizeof(int2),
                 cudaMemcpyHostToDevice) ||
      cudaMemcpy(m->d_pairs_old, m->pairs_old.data(), m->pairs_old.size() * sizeof(int2),
                 cudaMemcpyHostToDevice))
    return bail(mcuda(m, cudaGetLastError(), "cudaMemcpy (descriptors)"));
  if (mode == KLS_MODE_FP64) {
    if (cudaMemcpy(m->d_items, m->items.data(), m->items.size() * sizeof(kls_item),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(mcuda(m, cudaGetLastError(), "cudaMemcpy (items)"));
    if ((r = eager_pass(m, nullptr))) return bail(r);
  } else {
    // schedule tuning, one warm-up pass first.  One-CTA / pair-form models:
    // a persistent round robin or one CTA per item; TMEM-form models: one
    // launch with a CTA pair per (model, tile pair, split) item or one launch
    // of the single-model kernel per model.  Every schedule runs the same
    // bodies on the same items, so the bits do not depend on the choice.
    if (m->old && (r = schedule_items(m, 0))) return bail(r);
    if ((r = eager_pass(m, nullptr))) return bail(r);
    if (m->old) {
      for (int p = 0; p < 2; ++p) {
        float ms = 0.f;
        if ((r = schedule_items(m, p)) || (r = eager_pass(m, &ms))) return bail(r);
        m->schedule_ms[p] = ms;
      }
      if ((r = schedule_items(m, m->schedule_ms[1] < m->schedule_ms[0] ? 1 : 0))) return bail(r);
    }
    if (m->tm) {
      for (int p = 0; p < 2; ++p) {
        float ms = 0.f;
        m->tm_schedule = p ? 2 : 1;
        if ((r = eager_pass(m, &ms))) return bail(r);
        m->tm_schedule_ms[p] = ms;
      }
      m->tm_schedule = m->tm_schedule_ms[1] < m->tm_schedule_ms[0] ? 2 : 1;
    }
  }
  if ((r = capture(m))) return bail(r);
  *out = m;
  return KLS_OK;
}

int kls_multi_destroy(kls_multi* m) {
  if (!m) return KLS_OK;
  cudaSetDevice(m->device);
  release(m);
  delete m;
  return KLS_OK;
}

int kls_multi_det(kls_multi* m, const double* omega_ri, int n, double* det_ri, double* log_abs) {
  if (!m) return KLS_ERR_CONFIG;
  if (n < 0 || (n > 0 && (!omega_ri || !det_ri)))
    return mfail(m, KLS_ERR_CONFIG, "bad omega / output buffers");
  KM_CK(m, cudaSetDevice(m->device));
  auto fill = [&](int i, int k, double* o) {
    o[0] = omega_ri[2 * ((size_t)i * n + k)];
    o[1] = omega_ri[2 * ((size_t)i * n + k) + 1];
  };
  return run_omegas(m, fill, n, det_ri, log_abs);
}

int kls_scan_multi(kls_multi* m, const kls_scan_cfg* sc, double* det_grid, double* log_abs_grid,
                   double* Op0, double* g0) {
  if (!m) return KLS_ERR_CONFIG;
  if (!sc || sc->n_Op < 1 || sc->n_gamma < 1 || !det_grid)
    return mfail(m, KLS_ERR_CONFIG, "bad scan configuration");
  if ((long long)sc->n_Op * sc->n_gamma > INT_MAX)
    return mfail(m, KLS_ERR_CONFIG, "scan grid larger than 2^31 - 1 points");
  KM_CK(m, cudaSetDevice(m->device));
  const int nO = sc->n_Op, nG = sc->n_gamma, n = nO * nG;
  // column-major grid per model, omega = m_model * Omega_p + i gamma (GridScan.jl:47, :101-104)
  auto fill = [&](int i, int q, double* o) {
    const int ig = q % nG, jo = q / nG;
    o[0] = m->ctx[i]->cfg.m * kls_lin(sc->Omega_p_min, sc->Omega_p_max, nO, jo);
    o[1] = kls_lin(sc->gamma_min, sc->gamma_max, nG, ig);
  };
  std::vector<double> la;
  double* lap = log_abs_grid;
  if (!lap) {
    la.resize((size_t)m->n_models * n);
    lap = la.data();
  }
  int r = run_omegas(m, fill, n, det_grid, lap);
  if (r) return r;
  for (int i = 0; i < m->n_models; ++i) {
    const double* d = det_grid + (size_t)2 * i * n;
    int best = 0;
    double bv = INFINITY;
    for (int q = 0; q < n; ++q) {
      double v = std::hypot(d[2 * q], d[2 * q + 1]);
      if (std::isnan(v)) { best = q; break; }
      if (v < bv) { bv = v; best = q; }
    }
    if (Op0) Op0[i] = kls_lin(sc->Omega_p_min, sc->Omega_p_max, nO, best / nG);
    if (g0) g0[i] = kls_lin(sc->gamma_min, sc->gamma_max, nG, best % nG);
  }
  return KLS_OK;
}

int kls_multi_get_info(const kls_multi* m, kls_multi_info* out) {
  if (!m || !out) return KLS_ERR_CONFIG;
  out->n_models = m->n_models;
  out->batch = m->batch;
  out->mode = m->mode;
  const bool fp64 = m->mode == KLS_MODE_FP64;
  out->n_items = (int32_t)((fp64 || m->old ? m->items.size() : 0) + (m->tm ? m->tm_items.size() : 0));
  out->grid = (fp64 || m->old ? m->grid : 0) + (m->tm ? 2 * (int32_t)m->tm_items.size() : 0);
  out->graph = m->exec ? 1 : 0;
  out->replays = m->replays;
  out->last_ms = m->last_ms;
  // kernels per replay: weights (+ FP32 copy), contraction, reduction, LU
  // FP64: weights, contraction, reduction, LU; mixed: FP64 weights, per form
  // (FP32 weights, contraction launch(es), reduction), LU
  out->launches_per_replay =
      fp64 ? 4
           : 2 + (m->old ? 3 : 0) +
                 (m->tm ? 2 + (m->tm_schedule == 2 ? (int32_t)m->tmd.size() : 1) : 0);
  // the one-CTA / pair forms' schedule when the batch has such models, else
  // the TMEM-operand form's
  const bool tm_only = !fp64 && m->tm && !m->old;
  out->schedule = tm_only ? m->tm_schedule : m->schedule;
  out->schedule_ms[0] = tm_only ? m->tm_schedule_ms[0] : m->schedule_ms[0];
  out->schedule_ms[1] = tm_only ? m->tm_schedule_ms[1] : m->schedule_ms[1];
  return KLS_OK;
}

}  // extern "C"

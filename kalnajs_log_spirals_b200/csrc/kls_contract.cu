// MatrixBuilder on the device (FP64 form).
//
//   M(omega)[b, a] = G N(a) sum_k W[k, b] w_k(omega) conj(W[k, a]),
//   w_k = DJ_p F0l[p,l] / den,  den = omega - Omega_res[p,l],
//   den := 1e-12 + 1e-12 i  when |den| < 1e-12
//
// (MatrixBuilder.jl:27-69, NL_julia_direct.jl:299-310).  The reference loops
// the n_l harmonics with one ZGEMM each, after materialising
// weight .* conj(W) for every harmonic; here the whole K = NPh * n_l
// reduction is one split-K complex contraction on the FP64 tensor pipe
// (DMMA m8n8k4) and the resonant weight is applied to the B fragment while
// it is loaded from shared memory, so the weighted copy never exists.
//
//   weights_kernel : w_k(omega) for a batch of omegas (FP64, Smith division)
//   contract_kernel: 64x64 output tile per CTA, 4 warps of 32x32, cp.async
//                    3-stage pipeline over 16-row slabs of the W table,
//                    partial tiles per K split written to a workspace
//   reduce_kernel  : deterministic sum over splits, * G * N(a), I - M
#include "kls_internal.cuh"
#include <algorithm>
#include <cmath>

namespace {

// not volatile: the scheduler may interleave independent DMMAs
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---- weights ---------------------------------------------------------------
// 1/z by Smith's algorithm (R. L. Smith, CACM 5(8), 1962), then a * (1/z):
// the same evaluation order as Julia's a / z for a real a.
__device__ __forceinline__ double2 real_over_complex(double a, double c, double d) {
  double p, q;
  if (fabs(d) <= fabs(c)) {
    double r = d / c;
    double t = 1.0 / (c + d * r);
    p = t;
    q = -r * t;
  } else {
    double r = c / d;
    double t = 1.0 / (d + c * r);
    p = r * t;
    q = -t;
  }
  return make_double2(a * p, a * q);
}

__device__ __forceinline__ double2 weight_at(double g, double ok, double wr, double wi) {
  double dr = wr - ok, di = wi;
  if (hypot(dr, di) < 1e-12) { dr = 1e-12; di = 1e-12; }
  return real_over_complex(g, dr, di);
}

__device__ __forceinline__ void weights_body(int64_t K_pad, double wr, double wi,
                                             const double* __restrict__ Gk,
                                             const double* __restrict__ Ok,
                                             double2* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K_pad;
       k += (int64_t)gridDim.x * blockDim.x)
    KLS_IF(KLS_IB(k, K_pad, KS_WEIGHTS)) out[k] = weight_at(Gk[k], Ok[k], wr, wi);
}

// anchored: w_k(omega) - w_k(omega_a), each with the denominator clamp; the
// FP64 difference loses ~|w| / |dw| ulps, far below the FP32 rounding the
// split-BF16 contraction applies next
__global__ void weights_kernel(int64_t K_pad, const double* __restrict__ omega,
                               const double* __restrict__ Gk, const double* __restrict__ Ok,
                               double2* __restrict__ wt, int anchored, double ar, double ai) {
  const int z = blockIdx.y;
  const double wr = omega[2 * z], wi = omega[2 * z + 1];
  double2* out = wt + (size_t)z * K_pad;
  if (!anchored) {
    weights_body(K_pad, wr, wi, Gk, Ok, out);
    return;
  }
  if (wr == ar && wi == ai) {                // at the anchor dM is exactly zero
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K_pad;
         k += (int64_t)gridDim.x * blockDim.x)
      KLS_IF(KLS_IB(k, K_pad, KS_WEIGHTS)) out[k] = make_double2(0.0, 0.0);
    return;
  }
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K_pad;
       k += (int64_t)gridDim.x * blockDim.x) {
    KLS_UNLESS(KLS_IB(k, K_pad, KS_WEIGHTS), continue)
    const double2 a = weight_at(Gk[k], Ok[k], wr, wi), b = weight_at(Gk[k], Ok[k], ar, ai);
    out[k] = make_double2(a.x - b.x, a.y - b.y);
  }
}

// one (model, omega) pair per grid row
__global__ void multi_weights_kernel(const kls_mdesc* __restrict__ md,
                                     const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  const double* om = d.omega + 2 * pz.y;
  weights_body(d.K_pad, om[0], om[1], d.Gk, d.Ok, d.wt + (size_t)pz.y * d.K_pad);
}

// ---- contraction -----------------------------------------------------------
constexpr int CT_BK = 16;
constexpr int CT_S = KLS_TILE + 4;          // 68 doubles: conflict-free fragment loads
constexpr int CT_STAGES = 3;
constexpr int CT_THREADS = 128;
constexpr int CT_PLANE = CT_BK * CT_S;      // doubles per plane per stage
constexpr int CT_STAGE_DOUBLES = 4 * CT_PLANE + 2 * CT_BK;
constexpr size_t CT_SMEM = (size_t)CT_STAGES * CT_STAGE_DOUBLES * sizeof(double);

struct ContractParams {
  int Na_pad, tiles_1d, splits;
  int64_t K_pad, k_per_split;
};

// One 64 x 64 output tile of one K split for one omega: the partial tile goes
// to part[(z * splits + split)][b][a].
__device__ __forceinline__ void contract_tile(const ContractParams& P,
                                              const double* __restrict__ Wre,
                                              const double* __restrict__ Wim,
                                              const double2* __restrict__ wt,
                                              double2* __restrict__ part, double* smem, int tile,
                                              int split, int z) {
  const int tm = tile / P.tiles_1d, tn = tile % P.tiles_1d;
  const int b0 = tm * KLS_TILE, a0 = tn * KLS_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int64_t kbeg = (int64_t)split * P.k_per_split;
  const int64_t kend = min(P.K_pad, kbeg + P.k_per_split);
  const int nk = kbeg < kend ? (int)((kend - kbeg) / CT_BK) : 0;
  const double2* wz = wt + (size_t)z * P.K_pad;
  const size_t ld = (size_t)P.Na_pad;

  auto stage_ptr = [&](int s) { return smem + (size_t)s * CT_STAGE_DOUBLES; };
  auto load_stage = [&](int s, int kt) {
    double* st = stage_ptr(s);
    const int64_t k0 = kbeg + (int64_t)kt * CT_BK;
#pragma unroll
    for (int it = 0; it < 16; ++it) {
      int cidx = tid + it * CT_THREADS;        // 0..2047
      int plane = cidx >> 9;                   // 0: A re, 1: A im, 2: B re, 3: B im
      int rem = cidx & 511;
      int row = rem >> 5, col = (rem & 31) * 2;
      const double* src = (plane & 1) ? Wim : Wre;
      int c0 = (plane < 2) ? b0 : a0;
      // (bounds-checked build: the copy's last element inside [K_pad][Na_pad])
      KLS_IF(KLS_IB((k0 + row) * (int64_t)ld + c0 + col + 1, P.K_pad * (int64_t)ld,
                    KS_CONTRACT_SRC))
      cp_async16(st + plane * CT_PLANE + row * CT_S + col,
                 src + (size_t)(k0 + row) * ld + c0 + col);
    }
    if (tid < CT_BK) KLS_IF(KLS_IB(k0 + tid, P.K_pad, KS_CONTRACT_SRC))
      cp_async16(st + 4 * CT_PLANE + 2 * tid, wz + k0 + tid);
  };

  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      cr[i][j][0] = cr[i][j][1] = 0.0;
      ci[i][j][0] = ci[i][j][1] = 0.0;
    }

#pragma unroll
  for (int s = 0; s < CT_STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<CT_STAGES - 2>();
    __syncthreads();
    int nxt = kt + CT_STAGES - 1;
    if (nxt < nk) load_stage(nxt % CT_STAGES, nxt);
    cp_async_commit();
    const double* st = stage_ptr(kt % CT_STAGES);
    const double* sAr = st;
    const double* sAi = st + CT_PLANE;
    const double* sBr = st + 2 * CT_PLANE;
    const double* sBi = st + 3 * CT_PLANE;
    const double* sd = st + 4 * CT_PLANE;
#pragma unroll
    for (int kk = 0; kk < CT_BK; kk += 4) {
      const int kr = kk + (lane & 3);
      const double dr = sd[2 * kr], di = sd[2 * kr + 1];
      double ar[4], ai[4], na[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int off = kr * CT_S + wm * 32 + i * 8 + (lane >> 2);
        ar[i] = sAr[off];
        ai[i] = sAi[off];
        na[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int off = kr * CT_S + wn * 32 + j * 8 + (lane >> 2);
        double xr = sBr[off], xi = sBi[off];
        // w * conj(W) = (dr xr + di xi) + i (di xr - dr xi); roundings
        // pinned so every kernel that inlines this body gives the same bits
        br[j] = __fma_rn(dr, xr, __dmul_rn(di, xi));
        bi[j] = __fma_rn(di, xr, -__dmul_rn(dr, xi));
      }
      // two passes of 32 independent DMMAs: each accumulator's second
      // update issues 32 instructions after its first
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
          dmma(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
        }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(cr[i][j][0], cr[i][j][1], na[i], bi[j]);
          dmma(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
        }
    }
  }
  cp_async_wait<0>();

  double2* out = part + ((size_t)z * P.splits + split) * ld * ld;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int b = b0 + wm * 32 + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int a = a0 + wn * 32 + j * 8 + 2 * (lane & 3);
      double2* o = out + (size_t)b * ld + a;
      KLS_UNLESS(KLS_IB((int64_t)b * ld + a + 1, (int64_t)ld * ld, KS_CONTRACT_OUT), continue)
      o[0] = make_double2(cr[i][j][0], ci[i][j][0]);
      o[1] = make_double2(cr[i][j][1], ci[i][j][1]);
    }
  }
}

__global__ void __launch_bounds__(CT_THREADS, 2)
contract_kernel(ContractParams P, const double* __restrict__ Wre, const double* __restrict__ Wim,
                const double2* __restrict__ wt, double2* __restrict__ part) {
  extern __shared__ __align__(16) double smem[];
  contract_tile(P, Wre, Wim, wt, part, smem, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---- 3M (Gauss) form: three real products per complex product -------------
// With A = W_b (ar + i ai) and B = w conj(W_a) (br + i bi):
//   P1 = ar br, P2 = ai bi, P3 = (ar + ai)(br + bi),
//   Re = P1 - P2, Im = (P3 - P1) - P2,
// so each k step takes 3 DMMAs per output fragment instead of 4.  Same tile
// and warp layout as the 4M form (4 warps of 32 x 32, 2 CTAs per SM); the
// three accumulators take 192 of the 255 registers, and the B fragment of
// each column block is formed just before its 12 DMMAs to keep the rest live
// set small.
constexpr int CT3_THREADS = 128;
constexpr int CT3_STAGES = 3;
constexpr size_t CT3_SMEM = (size_t)CT3_STAGES * CT_STAGE_DOUBLES * sizeof(double);

__device__ __forceinline__ void contract_tile_3m(const ContractParams& P,
                                                 const double* __restrict__ Wre,
                                                 const double* __restrict__ Wim,
                                                 const double2* __restrict__ wt,
                                                 double2* __restrict__ part, double* smem,
                                                 int tile, int split, int z) {
  const int tm = tile / P.tiles_1d, tn = tile % P.tiles_1d;
  const int b0 = tm * KLS_TILE, a0 = tn * KLS_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;             // 32 x 32 per warp
  const int64_t kbeg = (int64_t)split * P.k_per_split;
  const int64_t kend = min(P.K_pad, kbeg + P.k_per_split);
  const int nk = kbeg < kend ? (int)((kend - kbeg) / CT_BK) : 0;
  const double2* wz = wt + (size_t)z * P.K_pad;
  const size_t ld = (size_t)P.Na_pad;

  auto stage_ptr = [&](int s) { return smem + (size_t)s * CT_STAGE_DOUBLES; };
  auto load_stage = [&](int s, int kt) {
    double* st = stage_ptr(s);
    const int64_t k0 = kbeg + (int64_t)kt * CT_BK;
#pragma unroll
    for (int it = 0; it < 16; ++it) {
      int cidx = tid + it * CT3_THREADS;       // 0..2047
      int plane = cidx >> 9;                   // 0: A re, 1: A im, 2: B re, 3: B im
      int rem = cidx & 511;
      int row = rem >> 5, col = (rem & 31) * 2;
      const double* src = (plane & 1) ? Wim : Wre;
      int c0 = (plane < 2) ? b0 : a0;
      // (bounds-checked build: the copy's last element inside [K_pad][Na_pad])
      KLS_IF(KLS_IB((k0 + row) * (int64_t)ld + c0 + col + 1, P.K_pad * (int64_t)ld,
                    KS_CONTRACT_SRC))
      cp_async16(st + plane * CT_PLANE + row * CT_S + col,
                 src + (size_t)(k0 + row) * ld + c0 + col);
    }
    if (tid < CT_BK) KLS_IF(KLS_IB(k0 + tid, P.K_pad, KS_CONTRACT_SRC))
      cp_async16(st + 4 * CT_PLANE + 2 * tid, wz + k0 + tid);
  };

  double p1[4][4][2], p2[4][4][2], p3[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) p1[i][j][h] = p2[i][j][h] = p3[i][j][h] = 0.0;

#pragma unroll
  for (int s = 0; s < CT3_STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<CT3_STAGES - 2>();
    __syncthreads();
    int nxt = kt + CT3_STAGES - 1;
    if (nxt < nk) load_stage(nxt % CT3_STAGES, nxt);
    cp_async_commit();
    const double* st = stage_ptr(kt % CT3_STAGES);
    const double* sAr = st;
    const double* sAi = st + CT_PLANE;
    const double* sBr = st + 2 * CT_PLANE;
    const double* sBi = st + 3 * CT_PLANE;
    const double* sd = st + 4 * CT_PLANE;
#pragma unroll
    for (int kk = 0; kk < CT_BK; kk += 4) {
      const int kr = kk + (lane & 3);
      const double dr = sd[2 * kr], di = sd[2 * kr + 1];
      double ar[4], ai[4], as[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int off = kr * CT_S + wm * 32 + i * 8 + (lane >> 2);
        ar[i] = sAr[off];
        ai[i] = sAi[off];
        as[i] = __dadd_rn(ar[i], ai[i]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int off = kr * CT_S + wn * 32 + j * 8 + (lane >> 2);
        double xr = sBr[off], xi = sBi[off];
        // the same weighted fragment as the 4M form
        const double br = __fma_rn(dr, xr, __dmul_rn(di, xi));
        const double bi = __fma_rn(di, xr, -__dmul_rn(dr, xi));
        const double bs = __dadd_rn(br, bi);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          dmma(p1[i][j][0], p1[i][j][1], ar[i], br);
          dmma(p2[i][j][0], p2[i][j][1], ai[i], bi);
          dmma(p3[i][j][0], p3[i][j][1], as[i], bs);
        }
      }
    }
  }
  cp_async_wait<0>();

  double2* out = part + ((size_t)z * P.splits + split) * ld * ld;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int b = b0 + wm * 32 + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int a = a0 + wn * 32 + j * 8 + 2 * (lane & 3);
      double2* o = out + (size_t)b * ld + a;
      KLS_UNLESS(KLS_IB((int64_t)b * ld + a + 1, (int64_t)ld * ld, KS_CONTRACT_OUT), continue)
#pragma unroll
      for (int h = 0; h < 2; ++h)
        o[h] = make_double2(__dsub_rn(p1[i][j][h], p2[i][j][h]),
                            __dsub_rn(__dsub_rn(p3[i][j][h], p1[i][j][h]), p2[i][j][h]));
    }
  }
}

__global__ void __launch_bounds__(CT3_THREADS, 2)
contract3m_kernel(ContractParams P, const double* __restrict__ Wre,
                  const double* __restrict__ Wim, const double2* __restrict__ wt,
                  double2* __restrict__ part) {
  extern __shared__ __align__(16) double smem[];
  contract_tile_3m(P, Wre, Wim, wt, part, smem, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Persistent form over an uneven batch: every CTA takes work items
// (model, omega, tile, split) from an atomic counter until the list is
// exhausted.  The list runs model by model, largest first, tile fastest, so
// CTAs running together share a k-range of one table (L2 reuse) and the tail
// of the launch is made of the small models' items.  Each item computes exactly
// what contract_kernel computes for the same (tile, split, omega), so a
// determinant is bitwise the same in either form.
__global__ void __launch_bounds__(CT_THREADS, 2)
multi_contract_kernel(const kls_mdesc* __restrict__ md, const kls_item* __restrict__ items,
                      int n_items, int* __restrict__ counter) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int i = s_item;
    if (i >= n_items) break;
    const kls_item it = items[i];
    const kls_mdesc& d = md[it.model];
    ContractParams P;
    P.Na_pad = d.Na_pad;
    P.tiles_1d = d.Na_pad / KLS_TILE;
    P.splits = d.splits;
    P.K_pad = d.K_pad;
    P.k_per_split = d.k_per_split;
    contract_tile(P, d.Wre, d.Wim, d.wt, d.part, smem, it.tile, it.split, it.z);
    __syncthreads();          // shared stages and s_item are reused by the next item
  }
}

// the same persistent loop over the 3M tile
__global__ void __launch_bounds__(CT3_THREADS, 2)
multi_contract3m_kernel(const kls_mdesc* __restrict__ md, const kls_item* __restrict__ items,
                        int n_items, int* __restrict__ counter) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int i = s_item;
    if (i >= n_items) break;
    const kls_item it = items[i];
    const kls_mdesc& d = md[it.model];
    ContractParams P;
    P.Na_pad = d.Na_pad;
    P.tiles_1d = d.Na_pad / KLS_TILE;
    P.splits = d.splits;
    P.K_pad = d.K_pad;
    P.k_per_split = d.k_per_split;
    contract_tile_3m(P, d.Wre, d.Wim, d.wt, d.part, smem, it.tile, it.split, it.z);
    __syncthreads();
  }
}

// ---- split reduction + epilogue ------------------------------------------------
__device__ __forceinline__ void reduce_body(int Na, int Na_pad, int splits, double G,
                                            const double* __restrict__ Nk,
                                            const double2* __restrict__ part,
                                            double2* __restrict__ A, double2* __restrict__ Mout) {
  const size_t plane = (size_t)Na_pad * Na_pad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Na * Na; e += gridDim.x * blockDim.x) {
    int b = e / Na, a = e % Na;
    const double2* src = part + (size_t)b * Na_pad + a;
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < splits; ++s) {
      KLS_UNLESS(KLS_IB((int64_t)s * plane + (int64_t)b * Na_pad + a,
                        (int64_t)splits * plane, KS_REDUCE), continue)
      double2 v = src[(size_t)s * plane];
      sr += v.x;
      si += v.y;
    }
    double n = Nk[a];
    // unfused products: 1 - mr must not become an FMA in one kernel only
    double mr = __dmul_rn(__dmul_rn(sr, G), n), mi = __dmul_rn(__dmul_rn(si, G), n);
    KLS_UNLESS(KLS_IB(e, (int64_t)Na * Na, KS_REDUCE), continue)
    A[e] = make_double2((a == b ? 1.0 : 0.0) - mr, -mi);
    if (Mout) Mout[e] = make_double2(mr, mi);
  }
}

__global__ void reduce_kernel(int Na, int Na_pad, int splits, double G,
                              const double* __restrict__ Nk, const double2* __restrict__ part,
                              double2* __restrict__ A, double2* __restrict__ Mout) {
  const int z = blockIdx.y;
  const size_t plane = (size_t)Na_pad * Na_pad;
  reduce_body(Na, Na_pad, splits, G, Nk, part + (size_t)z * splits * plane,
              A + (size_t)z * Na * Na, z == 0 ? Mout : nullptr);
}

__global__ void multi_reduce_kernel(const kls_mdesc* __restrict__ md,
                                    const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  const size_t plane = (size_t)d.Na_pad * d.Na_pad;
  reduce_body(d.Na, d.Na_pad, d.splits, d.G, d.Nk, d.part + (size_t)pz.y * d.splits * plane,
              d.A + (size_t)pz.y * d.Na * d.Na, nullptr);
}

}  // namespace

// The split count depends on the table and the device only, never on the
// batch size, so a determinant is bitwise identical whichever batch it is
// evaluated in.  It is chosen so that tiles * splits fills a whole number q
// of waves as closely as possible (q in 1..8, at least 16 splits where the
// table allows, at least 8 slabs per split): then n omegas take n * q nearly
// full waves for every n.  At N_alpha_pad = 320 (25 tiles) on 296 slots
// that is 71 splits: 1775 CTAs per omega = 99.9% of 6 waves.
// CTAs of the FP64 contraction form `form` resident on the device at once
static int f64_slots(int device, int form, bool persistent) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const void* fn = form == KLS_F64_3M
                       ? (persistent ? (const void*)multi_contract3m_kernel
                                     : (const void*)contract3m_kernel)
                       : (persistent ? (const void*)multi_contract_kernel
                                     : (const void*)contract_kernel);
  const int threads = form == KLS_F64_3M ? CT3_THREADS : CT_THREADS;
  const size_t smem = form == KLS_F64_3M ? CT3_SMEM : CT_SMEM;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

int kls_choose_splits(const kls_ctx* c) {
  const int tiles = (c->Na_pad / KLS_TILE) * (c->Na_pad / KLS_TILE);
  const int slots = f64_slots(c->device, c->f64_form, false);
  int64_t max_s = c->K_pad / (CT_BK * 8);            // at least 8 slabs per split
  if (max_s > 512) max_s = 512;
  if (max_s < 1) max_s = 1;
  int best = (int)std::min<int64_t>(max_s, std::max(1, slots / std::max(1, tiles)));
  double best_fill = -1.0;
  for (int q = 1; q <= 8; ++q) {
    const int s = (int)std::min<int64_t>(max_s, (int64_t)q * slots / tiles);
    if (s < 1) continue;
    if (s < 16 && (int64_t)(q + 1) * slots / tiles <= max_s) continue;   // prefer >= 16 splits
    const double work = (double)tiles * s;
    const double fill = work / (std::ceil(work / slots) * slots);
    if (fill > best_fill + 1e-3) {
      best_fill = fill;
      best = s;
    }
  }
  return best;
}

int kls_run_weights(kls_ctx* c, int n, const double* anchor) {
  int blocks = (int)std::min<int64_t>((c->K_pad + 255) / 256, 2048);
  weights_kernel<<<dim3(blocks, n), 256, 0, c->stream>>>(
      c->K_pad, c->d_omega, c->d_Gk, c->d_Ok, c->d_wt, anchor ? 1 : 0, anchor ? anchor[0] : 0.0,
      anchor ? anchor[1] : 0.0);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_run_contract_f64(kls_ctx* c, int n, int splits) {
  ContractParams P{};
  P.Na_pad = c->Na_pad;
  P.tiles_1d = c->Na_pad / KLS_TILE;
  P.splits = splits;
  P.K_pad = c->K_pad;
  P.k_per_split = kls_f64_k_per_split(c->K_pad, splits);
  dim3 grid(P.tiles_1d * P.tiles_1d, splits, n);
  if (c->f64_form == KLS_F64_3M) {
    KLS_CK(c, cudaFuncSetAttribute(contract3m_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)CT3_SMEM));
    contract3m_kernel<<<grid, CT3_THREADS, CT3_SMEM, c->stream>>>(P, c->d_Wre, c->d_Wim,
                                                                  c->d_wt, c->d_part);
    KLS_LAUNCHED(c);
    return KLS_OK;
  }
  KLS_CK(c, cudaFuncSetAttribute(contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CT_SMEM));
  contract_kernel<<<grid, CT_THREADS, CT_SMEM, c->stream>>>(P, c->d_Wre, c->d_Wim, c->d_wt,
                                                            c->d_part);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_run_reduce(kls_ctx* c, int n, int splits, bool export_M) {
  int blocks = std::min((c->Na * c->Na + 255) / 256, 1024);
  reduce_kernel<<<dim3(blocks, n), 256, 0, c->stream>>>(c->Na, c->Na_pad, splits, c->cfg.G, c->d_N,
                                                        c->d_part, c->d_A,
                                                        export_M ? c->d_M : nullptr);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

// ---- uneven batch over models (kls_multi.cu) ------------------------------------
int kls_multi_launch_f64(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs, int n_pairs,
                         const kls_item* d_items, int n_items, int* d_counter, int grid,
                         int64_t max_K_pad, int form) {
  int wblocks = (int)std::min<int64_t>((max_K_pad + 255) / 256, 1024);
  multi_weights_kernel<<<dim3(wblocks, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const bool g3 = form == KLS_F64_3M;
  if ((e = cudaFuncSetAttribute(g3 ? (const void*)multi_contract3m_kernel
                                   : (const void*)multi_contract_kernel,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(g3 ? CT3_SMEM : CT_SMEM))) != cudaSuccess)
    return (int)e;
  if ((e = cudaMemsetAsync(d_counter, 0, sizeof(int), st)) != cudaSuccess) return (int)e;
  if (g3)
    multi_contract3m_kernel<<<grid, CT3_THREADS, CT3_SMEM, st>>>(d_md, d_items, n_items,
                                                                 d_counter);
  else
    multi_contract_kernel<<<grid, CT_THREADS, CT_SMEM, st>>>(d_md, d_items, n_items, d_counter);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  multi_reduce_kernel<<<dim3(256, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  return (int)cudaGetLastError();
}

int kls_multi_launch_f64_weights(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs,
                                 int n_pairs, int64_t max_K_pad) {
  int wblocks = (int)std::min<int64_t>((max_K_pad + 255) / 256, 1024);
  multi_weights_kernel<<<dim3(wblocks, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  return (int)cudaGetLastError();
}

int kls_multi_contract_slots(int device, int form) { return f64_slots(device, form, true); }

int64_t kls_f64_k_per_split(int64_t K_pad, int splits) {
  int64_t slabs = K_pad / CT_BK;
  return ((slabs + splits - 1) / splits) * CT_BK;
}

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

__global__ void weights_kernel(int64_t K_pad, const double* __restrict__ omega,
                               const double* __restrict__ Gk, const double* __restrict__ Ok,
                               double2* __restrict__ wt) {
  const int z = blockIdx.y;
  const double wr = omega[2 * z], wi = omega[2 * z + 1];
  double2* out = wt + (size_t)z * K_pad;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K_pad;
       k += (int64_t)gridDim.x * blockDim.x) {
    double dr = wr - Ok[k], di = wi;
    if (hypot(dr, di) < 1e-12) { dr = 1e-12; di = 1e-12; }
    out[k] = real_over_complex(Gk[k], dr, di);
  }
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

__global__ void __launch_bounds__(CT_THREADS, 2)
contract_kernel(ContractParams P, const double* __restrict__ Wre, const double* __restrict__ Wim,
                const double2* __restrict__ wt, double2* __restrict__ part) {
  extern __shared__ __align__(16) double smem[];
  const int tile = blockIdx.x, split = blockIdx.y, z = blockIdx.z;
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
      cp_async16(st + plane * CT_PLANE + row * CT_S + col,
                 src + (size_t)(k0 + row) * ld + c0 + col);
    }
    if (tid < CT_BK) cp_async16(st + 4 * CT_PLANE + 2 * tid, wz + k0 + tid);
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
        // w * conj(W) = (dr xr + di xi) + i (di xr - dr xi)
        br[j] = dr * xr + di * xi;
        bi[j] = di * xr - dr * xi;
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
      o[0] = make_double2(cr[i][j][0], ci[i][j][0]);
      o[1] = make_double2(cr[i][j][1], ci[i][j][1]);
    }
  }
}

// ---- split reduction + epilogue ------------------------------------------------
__global__ void reduce_kernel(int Na, int Na_pad, int splits, double G,
                              const double* __restrict__ Nk, const double2* __restrict__ part,
                              double2* __restrict__ A, double2* __restrict__ Mout) {
  const int z = blockIdx.y;
  const size_t plane = (size_t)Na_pad * Na_pad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Na * Na; e += gridDim.x * blockDim.x) {
    int b = e / Na, a = e % Na;
    const double2* src = part + (size_t)z * splits * plane + (size_t)b * Na_pad + a;
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < splits; ++s) {
      double2 v = src[(size_t)s * plane];
      sr += v.x;
      si += v.y;
    }
    double n = Nk[a];
    double mr = (sr * G) * n, mi = (si * G) * n;
    A[(size_t)z * Na * Na + e] = make_double2((a == b ? 1.0 : 0.0) - mr, -mi);
    if (Mout && z == 0) Mout[e] = make_double2(mr, mi);
  }
}

}  // namespace

// The split count depends on the table and the device only, never on the
// batch size, so a determinant is bitwise identical whichever batch it is
// evaluated in.  It is chosen so that tiles * splits fills just under a
// whole number q of waves (q the smallest giving >= 16 splits): then n
// omegas take n * q rounds with every round nearly full.
int kls_choose_splits(const kls_ctx* c) {
  const int tiles = (c->Na_pad / KLS_TILE) * (c->Na_pad / KLS_TILE);
  int sms = 148, per_sm = 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  cudaFuncSetAttribute(contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CT_SMEM);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, contract_kernel, CT_THREADS,
                                                    CT_SMEM) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int slots = sms * per_sm;
  int q = std::max(1, (16 * tiles + slots - 1) / slots);
  int s = (q * slots) / tiles;
  int64_t max_s = c->K_pad / (CT_BK * 8);            // at least 8 slabs per split
  if (s > max_s) s = (int)max_s;
  if (s < 1) s = 1;
  if (s > 256) s = 256;
  return s;
}

int kls_run_weights(kls_ctx* c, int n) {
  int blocks = (int)std::min<int64_t>((c->K_pad + 255) / 256, 2048);
  weights_kernel<<<dim3(blocks, n), 256, 0, c->stream>>>(c->K_pad, c->d_omega, c->d_Gk, c->d_Ok,
                                                         c->d_wt);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_run_contract_f64(kls_ctx* c, int n, int splits) {
  KLS_CK(c, cudaFuncSetAttribute(contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CT_SMEM));
  ContractParams P{};
  P.Na_pad = c->Na_pad;
  P.tiles_1d = c->Na_pad / KLS_TILE;
  P.splits = splits;
  P.K_pad = c->K_pad;
  int64_t slabs = c->K_pad / CT_BK;
  P.k_per_split = ((slabs + splits - 1) / splits) * CT_BK;
  dim3 grid(P.tiles_1d * P.tiles_1d, splits, n);
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

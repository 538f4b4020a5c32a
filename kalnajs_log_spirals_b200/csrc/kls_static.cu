// kls_det_lu_static: determinants of caller-supplied complex matrices with no
// device allocation.
//
// Who needs this: a caller that may not allocate device memory itself, for
// example a host program that has handed the whole GPU to its own pool
// allocator (a Julia CUDA.jl or PyTorch caching allocator that owns every
// byte and forbids outside cudaMalloc), or a latency-critical loop that
// cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.
// Such a caller allocates its inputs and outputs from its own pool and this
// entry point uses only them plus a fixed scratch array that is part of the
// library image.
//
// The scratch is a file-scope __device__ array of KLS_STATIC_LU_MAX complex
// doubles (16 MiB).  Every GPU that loads libkls.so holds it until the
// process exits.  Host code must not pass the array's name to a kernel (on
// the host it is only a stand-in symbol); the device address is fetched once
// per device with cudaGetSymbolAddress, with that device current, by the
// first call on that device.  Every call reuses the same array and leaves the
// last call's LU factors in it; nothing in it has to start at zero because
// each call overwrites the part it uses before reading it.  Calls whose
// kernels overlap on the same GPU (different streams or host threads without
// ordering between them) race on the scratch.
#include "kls_internal.cuh"
#include <cmath>
#include <mutex>

namespace {

constexpr long long KLS_STATIC_LU_MAX = 1LL << 20;   // complex elements (16 MiB)
constexpr int SLU_THREADS = 1024;
constexpr int SLU_MAX_DEVICES = 64;

static __device__ __align__(256) double2 g_lu_scratch[KLS_STATIC_LU_MAX];

std::mutex g_scratch_mu;
double2* g_scratch_ptr[SLU_MAX_DEVICES] = {nullptr};

__device__ __forceinline__ double2 s_cinv(double c, double d) {
  if (fabs(d) <= fabs(c)) {
    double r = d / c, t = 1.0 / (c + d * r);
    return make_double2(t, -r * t);
  }
  double r = c / d, t = 1.0 / (d + c * r);
  return make_double2(r * t, -t);
}

__device__ __forceinline__ double2 s_cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One CTA per matrix: copy the input into the scratch, then complex LU with
// izamax partial pivoting in place; det returned as a complex number and as
// log|det| (mantissa + binary exponent accumulation).
__global__ void __launch_bounds__(SLU_THREADS)
lu_det_static_kernel(int n, const double2* __restrict__ in, double2* __restrict__ scratch,
                     double2* __restrict__ det_out, double* __restrict__ logabs_out) {
  extern __shared__ double2 sh[];
  double2* prow = sh;
  double2* lcol = sh + n;
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  __shared__ double2 s_u;
  const size_t nn = (size_t)n * n;
  const double2* src = in + (size_t)blockIdx.x * nn;
  double2* A = scratch + (size_t)blockIdx.x * nn;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  for (size_t e = tid; e < nn; e += blockDim.x)
    KLS_IF(KLS_IB((int64_t)blockIdx.x * nn + e, KLS_STATIC_LU_MAX, KS_LU_STATIC)) A[e] = src[e];
  __syncthreads();

  double2 mant = make_double2(1.0, 0.0);
  long long expo = 0;
  bool zero = false;
  for (int j = 0; j < n; ++j) {
    double bv = -1.0;
    int bi = n;
    for (int i = j + tid; i < n; i += blockDim.x) {
      double2 v = A[(size_t)i * n + j];
      double m = fabs(v.x) + fabs(v.y);
      if (m > bv) { bv = m; bi = i; }
    }
    for (int off = 16; off; off >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, bv, off);
      int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
      bv = lane < nwarps ? red_v[lane] : -1.0;
      bi = lane < nwarps ? red_i[lane] : n;
      for (int off = 16; off; off >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, bv, off);
        int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (lane == 0) s_piv = (bi < n) ? bi : j;
    }
    __syncthreads();
    const int piv = s_piv;
    if (piv != j) {
      for (int c = j + tid; c < n; c += blockDim.x) {
        double2 t = A[(size_t)j * n + c];
        A[(size_t)j * n + c] = A[(size_t)piv * n + c];
        A[(size_t)piv * n + c] = t;
      }
    }
    __syncthreads();
    double2 u = A[(size_t)j * n + j];
    const bool nz = (u.x != 0.0 || u.y != 0.0);
    double2 ru = nz ? s_cinv(u.x, u.y) : make_double2(0.0, 0.0);
    for (int c = j + 1 + tid; c < n; c += blockDim.x) prow[c] = A[(size_t)j * n + c];
    for (int i = j + 1 + tid; i < n; i += blockDim.x) lcol[i] = s_cmul(A[(size_t)i * n + j], ru);
    if (tid == 0) s_u = u;
    __syncthreads();
    for (int i = j + 1 + warp; i < n; i += nwarps) {
      double2 l = lcol[i];
      double2* row = A + (size_t)i * n;
      for (int c = j + 1 + lane; c < n; c += 32) {
        double2 p = prow[c];
        double2 a = row[c];
        a.x -= l.x * p.x - l.y * p.y;
        a.y -= l.x * p.y + l.y * p.x;
        row[c] = a;
      }
    }
    if (tid == 0) {
      double2 uu = s_u;
      if (piv != j) { mant.x = -mant.x; mant.y = -mant.y; }
      if (uu.x == 0.0 && uu.y == 0.0) zero = true;
      mant = s_cmul(mant, uu);
      double mx = fmax(fabs(mant.x), fabs(mant.y));
      if (mx != 0.0 && isfinite(mx)) {
        int e = ilogb(mx);
        mant.x = scalbn(mant.x, -e);
        mant.y = scalbn(mant.y, -e);
        expo += e;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    double2 d;
    double la;
    if (zero) {
      d = make_double2(0.0, 0.0);
      la = -INFINITY;
    } else {
      long long e = expo;
      if (e > 4000) e = 4000;
      if (e < -4000) e = -4000;
      d = make_double2(scalbn(mant.x, (int)e), scalbn(mant.y, (int)e));
      la = log(hypot(mant.x, mant.y)) + (double)expo * 0.69314718055994530942;
    }
    det_out[blockIdx.x] = d;
    if (logabs_out) logabs_out[blockIdx.x] = la;
  }
}

// failures are reported like kls_create's: status code + kls_create_error()
int static_fail(int code, const std::string& m) { return kls_fail(nullptr, code, m); }

}  // namespace

extern "C" {

int kls_det_lu_static(const double* d_A_ri, int n_matrices, int N, double* d_det_ri,
                      double* d_log_abs, void* stream) {
  if (n_matrices < 0 || N < 1 || (n_matrices > 0 && (!d_A_ri || !d_det_ri)))
    return static_fail(KLS_ERR_CONFIG, "kls_det_lu_static: bad arguments");
  if (n_matrices == 0) return KLS_OK;
  // One matrix of 1024^2 complex elements fills the scratch, so N <= 1024;
  // the kernel's two row buffers then take at most 2 * 1024 * 16 B = 32 KiB
  // of shared memory, inside the default 48 KiB (no opt-in needed).
  if (N > 1024)
    return static_fail(KLS_ERR_CONFIG, "kls_det_lu_static: N = " + std::to_string(N) +
                                           " > 1024: one matrix exceeds the fixed scratch");
  if ((long long)n_matrices * N * N > KLS_STATIC_LU_MAX) {
    return static_fail(KLS_ERR_CONFIG,
                       "kls_det_lu_static: n_matrices * N * N = " +
                           std::to_string((long long)n_matrices * N * N) +
                           " exceeds the fixed scratch of " + std::to_string(KLS_STATIC_LU_MAX) +
                           " complex elements");
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return static_fail(KLS_ERR_CUDA, std::string("kls_det_lu_static: cudaGetDevice: ") +
                                         cudaGetErrorString(e));
  if (dev < 0 || dev >= SLU_MAX_DEVICES)
    return static_fail(KLS_ERR_UNSUPPORTED,
                       "kls_det_lu_static: device index " + std::to_string(dev) +
                           " is beyond the " + std::to_string(SLU_MAX_DEVICES) +
                           " devices whose scratch addresses are cached");
  double2* scratch;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      // one-time set-up on this device (the current one): device address of
      // the library's scratch array
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_lu_scratch);
      if (e != cudaSuccess || !p)
        return static_fail(KLS_ERR_CUDA, std::string("kls_det_lu_static: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
      g_scratch_ptr[dev] = (double2*)p;
    }
    scratch = g_scratch_ptr[dev];
  }
  const size_t sm = 2 * (size_t)N * sizeof(double2);
  lu_det_static_kernel<<<n_matrices, SLU_THREADS, sm, (cudaStream_t)stream>>>(
      N, reinterpret_cast<const double2*>(d_A_ri), scratch, reinterpret_cast<double2*>(d_det_ri),
      d_log_abs);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return static_fail(KLS_ERR_CUDA, std::string("kls_det_lu_static: launch: ") +
                                         cudaGetErrorString(e));
  return KLS_OK;
}

}  // extern "C"

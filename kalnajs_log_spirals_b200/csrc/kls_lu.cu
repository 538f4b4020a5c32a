// det(I - M(omega)) for a batch of matrices: complex FP64 LU with partial
// pivoting, one CTA per matrix (the reference moves M to the host and calls
// LinearAlgebra.det -> LAPACK zgetrf, MatrixBuilder.jl:173-182).
//
// Pivot choice follows LAPACK's izamax (largest |re| + |im|, first index on
// ties); the column is scaled by the reciprocal of the pivot as zgetf2 does.
// The determinant is accumulated as a mantissa and a binary exponent so that
// products of ~N_alpha pivots neither overflow nor underflow; the result is
// returned both as a complex number and as log|det|.
#include "kls_internal.cuh"
#include <cfloat>

namespace {

constexpr int LU_THREADS = 1024;

__device__ __forceinline__ double2 cinv(double c, double d) {
  // Smith's algorithm for 1/(c + i d)
  if (fabs(d) <= fabs(c)) {
    double r = d / c, t = 1.0 / (c + d * r);
    return make_double2(t, -r * t);
  }
  double r = c / d, t = 1.0 / (d + c * r);
  return make_double2(r * t, -t);
}

// roundings pinned (no compiler choice of which product joins an FMA), so
// every kernel that inlines the LU body gives the same bits
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__fma_rn(a.x, b.x, -__dmul_rn(a.y, b.y)),
                      __fma_rn(a.x, b.y, __dmul_rn(a.y, b.x)));
}

// LU of one n x n row-major matrix A by the whole CTA; writes *det_out and,
// if given, *logabs_out.  sh holds 2 n complex values.
__device__ __forceinline__ void lu_det_body(int n, double2* __restrict__ A, double2* sh,
                                            double2* __restrict__ det_out,
                                            double* __restrict__ logabs_out) {
  double2* prow = sh;
  double2* lcol = sh + n;
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  __shared__ double2 s_u;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;

  double2 mant = make_double2(1.0, 0.0);
  long long expo = 0;
  bool zero = false;

  for (int j = 0; j < n; ++j) {
    // ---- pivot search: izamax over rows j..n-1 of column j
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
      if (lane == 0) s_piv = (bi < n) ? bi : j;   // NaN column: keep the diagonal
    }
    __syncthreads();
    const int piv = s_piv;
    // ---- row interchange (columns j..n-1; L columns are not needed for det)
    if (piv != j) {
      for (int c = j + tid; c < n; c += blockDim.x) {
        double2 t = A[(size_t)j * n + c];
        A[(size_t)j * n + c] = A[(size_t)piv * n + c];
        A[(size_t)piv * n + c] = t;
      }
    }
    __syncthreads();
    // ---- pivot row and scaled column to shared memory
    double2 u = A[(size_t)j * n + j];
    const bool nz = (u.x != 0.0 || u.y != 0.0);
    double2 ru = nz ? cinv(u.x, u.y) : make_double2(0.0, 0.0);
    for (int c = j + 1 + tid; c < n; c += blockDim.x) prow[c] = A[(size_t)j * n + c];
    for (int i = j + 1 + tid; i < n; i += blockDim.x) lcol[i] = cmul(A[(size_t)i * n + j], ru);
    if (tid == 0) s_u = u;
    __syncthreads();
    // ---- rank-1 update of the trailing matrix
    for (int i = j + 1 + warp; i < n; i += nwarps) {
      double2 l = lcol[i];
      double2* row = A + (size_t)i * n;
      for (int c = j + 1 + lane; c < n; c += 32) {
        double2 p = prow[c];
        double2 a = row[c];
        a.x = __dsub_rn(a.x, __fma_rn(l.x, p.x, -__dmul_rn(l.y, p.y)));
        a.y = __dsub_rn(a.y, __fma_rn(l.x, p.y, __dmul_rn(l.y, p.x)));
        row[c] = a;
      }
    }
    // ---- determinant accumulation (thread 0)
    if (tid == 0) {
      double2 uu = s_u;
      if (piv != j) { mant.x = -mant.x; mant.y = -mant.y; }
      if (uu.x == 0.0 && uu.y == 0.0) zero = true;
      mant = cmul(mant, uu);
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
    *det_out = d;
    if (logabs_out) *logabs_out = la;
  }
}

__global__ void __launch_bounds__(LU_THREADS)
lu_det_kernel(int n, double2* __restrict__ Aall, double2* __restrict__ det_out,
              double* __restrict__ logabs_out) {
  extern __shared__ double2 sh[];        // prow[n], lcol[n]
  lu_det_body(n, Aall + (size_t)blockIdx.x * n * n, sh, det_out + blockIdx.x,
              logabs_out ? logabs_out + blockIdx.x : nullptr);
}

// one (model, omega) pair per CTA, matrices of different sizes
__global__ void __launch_bounds__(LU_THREADS)
multi_lu_kernel(const kls_mdesc* __restrict__ md, const int2* __restrict__ pairs) {
  extern __shared__ double2 sh[];
  const int2 pz = pairs[blockIdx.x];
  const kls_mdesc& d = md[pz.x];
  lu_det_body(d.Na, d.A + (size_t)pz.y * d.Na * d.Na, sh, d.det + pz.y, d.logabs + pz.y);
}

}  // namespace

int kls_run_lu(kls_ctx* c, int n) {
  size_t sm = 2 * (size_t)c->Na * sizeof(double2);
  if (sm > 48 * 1024)
    KLS_CK(c, cudaFuncSetAttribute(lu_det_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sm));
  lu_det_kernel<<<n, LU_THREADS, sm, c->stream>>>(c->Na, c->d_A, c->d_det, c->d_logabs);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_multi_launch_lu(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs, int n_pairs,
                        int max_Na) {
  size_t sm = 2 * (size_t)max_Na * sizeof(double2);
  cudaError_t e;
  if (sm > 48 * 1024 &&
      (e = cudaFuncSetAttribute(multi_lu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sm)) != cudaSuccess)
    return (int)e;
  multi_lu_kernel<<<n_pairs, LU_THREADS, sm, st>>>(d_md, d_pairs);
  return (int)cudaGetLastError();
}

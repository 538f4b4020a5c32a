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
#include <cooperative_groups.h>
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

// element (i, c) of the n x n matrix A, guarded in the bounds-checked build
#define LU_IN(i, c) KLS_IB((int64_t)(i) * n + (c), (int64_t)n * n, KS_LU)
#define LU_A(i, c) KLS_LD(LU_IN(i, c), A[(size_t)i * n + c], make_double2(0.0, 0.0))

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
      double2 v = LU_A(i, j);
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
        KLS_UNLESS(LU_IN(j, c) && LU_IN(piv, c), continue)
        double2 t = A[(size_t)j * n + c];
        A[(size_t)j * n + c] = A[(size_t)piv * n + c];
        A[(size_t)piv * n + c] = t;
      }
    }
    __syncthreads();
    // ---- pivot row and scaled column to shared memory
    double2 u = LU_A(j, j);
    const bool nz = (u.x != 0.0 || u.y != 0.0);
    double2 ru = nz ? cinv(u.x, u.y) : make_double2(0.0, 0.0);
    for (int c = j + 1 + tid; c < n; c += blockDim.x) prow[c] = LU_A(j, c);
    for (int i = j + 1 + tid; i < n; i += blockDim.x) lcol[i] = cmul(LU_A(i, j), ru);
    if (tid == 0) s_u = u;
    __syncthreads();
    // ---- rank-1 update of the trailing matrix
    for (int i = j + 1 + warp; i < n; i += nwarps) {
      double2 l = lcol[i];
      double2* row = A + (size_t)i * n;
      for (int c = j + 1 + lane; c < n; c += 32) {
        KLS_UNLESS(LU_IN(i, c), continue)
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

// ---- cluster form: one thread-block cluster per matrix ---------------------------
// The matrix is distributed by columns over the C CTAs of a cluster (column g
// in CTA g mod C, column-major in shared memory), so the whole factorisation
// stays on chip: per step j the owner of column j searches the pivot, swaps,
// scales its column into multipliers; after one cluster barrier every CTA
// reads the pivot row index and the multipliers from the owner's shared
// memory (DSMEM) and updates its own trailing columns.  Pivot rule, multiplier
// and update arithmetic and the order of the determinant product are those of
// lu_det_kernel, so both kernels return the same bits.
namespace cg = cooperative_groups;
constexpr int LUC_THREADS = 512;

__host__ __device__ inline size_t luc_smem_bytes(int n, int C) {
  const size_t nc = (size_t)((n + C - 1) / C);
  return (nc * n + 3 * (size_t)n) * sizeof(double2) + (size_t)n * sizeof(int);
}

__global__ void __launch_bounds__(LUC_THREADS)
lu_cluster_kernel(int n, const double2* __restrict__ Aall, double2* __restrict__ det_out,
                  double* __restrict__ logabs_out) {
  extern __shared__ __align__(16) double2 smem[];
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int mat = blockIdx.x / C;
  const int nc = (n + C - 1) / C;
  double2* col = smem;                        // [nc][n] owned columns g = rank + C lc
  double2* lvec = col + (size_t)nc * n;       // multipliers of the steps this CTA owns
  double2* lbuf = lvec + n;                   // copy of the current owner's multipliers
  double2* rec_u = lbuf + n;                  // rank 0: pivot of every step
  int* rec_s = reinterpret_cast<int*>(rec_u + n);   // rank 0: row interchange flags
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int T = blockDim.x, nwarps = T >> 5;
  const int my_nc = rank < n ? (n - 1 - rank) / C + 1 : 0;
  const double2* A = Aall + (size_t)mat * n * n;
  for (int e = tid; e < my_nc * n; e += T) {
    const int lc = e / n, i = e % n;
    KLS_UNLESS(KLS_IB((int64_t)i * n + rank + C * lc, (int64_t)n * n, KS_LU), continue)
    col[(size_t)lc * n + i] = A[(size_t)i * n + rank + C * lc];
  }
  double2* rec_u0 = cl.map_shared_rank(rec_u, 0);
  int* rec_s0 = cl.map_shared_rank(rec_s, 0);
  __syncthreads();

  for (int j = 0; j < n; ++j) {
    const int owner = j % C;
    if (rank == owner) {
      double2* cj = col + (size_t)(j / C) * n;
      double bv = -1.0;
      int bi = n;
      for (int i = j + tid; i < n; i += T) {
        const double2 v = cj[i];
        const double m = fabs(v.x) + fabs(v.y);
        if (m > bv) { bv = m; bi = i; }
      }
      for (int off = 16; off; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
      __syncthreads();
      if (warp == 0) {
        bv = lane < nwarps ? red_v[lane] : -1.0;
        bi = lane < nwarps ? red_i[lane] : n;
        for (int off = 16; off; off >>= 1) {
          const double ov = __shfl_down_sync(0xffffffffu, bv, off);
          const int oi = __shfl_down_sync(0xffffffffu, bi, off);
          if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) s_piv = (bi < n) ? bi : j;   // NaN column: keep the diagonal
      }
      __syncthreads();
      const int piv = s_piv;
      if (tid == 0 && piv != j) {
        const double2 t = cj[j];
        cj[j] = cj[piv];
        cj[piv] = t;
      }
      __syncthreads();
      const double2 u = cj[j];
      const bool nz = (u.x != 0.0 || u.y != 0.0);
      const double2 ru = nz ? cinv(u.x, u.y) : make_double2(0.0, 0.0);
      for (int i = j + 1 + tid; i < n; i += T) lvec[i] = cmul(cj[i], ru);
      if (tid == 0) {
        rec_u0[j] = u;
        rec_s0[j] = piv != j;
      }
    }
    cl.sync();                                  // owner's pivot and multipliers visible
    const int piv = *cl.map_shared_rank(&s_piv, owner);
    const double2* ol = cl.map_shared_rank(lvec, owner);
    for (int i = j + 1 + tid; i < n; i += T) lbuf[i] = ol[i];
    // owned columns right of j: g = rank + C lc > j
    const int lc0 = j >= rank ? (j - rank) / C + 1 : 0;
    if (piv != j)
      for (int lc = lc0 + tid; lc < my_nc; lc += T) {
        double2* cc = col + (size_t)lc * n;
        const double2 t = cc[j];
        cc[j] = cc[piv];
        cc[piv] = t;
      }
    __syncthreads();
    const int nr = n - j - 1, ncols = my_nc - lc0;
    for (int e = tid; e < nr * ncols; e += T) {
      const int i = j + 1 + e % nr;
      double2* cc = col + (size_t)(lc0 + e / nr) * n;
      const double2 l = lbuf[i], p = cc[j];
      double2 a = cc[i];
      a.x = __dsub_rn(a.x, __fma_rn(l.x, p.x, -__dmul_rn(l.y, p.y)));
      a.y = __dsub_rn(a.y, __fma_rn(l.x, p.y, __dmul_rn(l.y, p.x)));
      cc[i] = a;
    }
    __syncthreads();
  }
  cl.sync();                                    // every record landed in rank 0
  if (rank == 0 && tid == 0) {
    double2 mant = make_double2(1.0, 0.0);
    long long expo = 0;
    bool zero = false;
    for (int j = 0; j < n; ++j) {
      const double2 uu = rec_u[j];
      if (rec_s[j]) { mant.x = -mant.x; mant.y = -mant.y; }
      if (uu.x == 0.0 && uu.y == 0.0) zero = true;
      mant = cmul(mant, uu);
      const double mx = fmax(fabs(mant.x), fabs(mant.y));
      if (mx != 0.0 && isfinite(mx)) {
        const int e = ilogb(mx);
        mant.x = scalbn(mant.x, -e);
        mant.y = scalbn(mant.y, -e);
        expo += e;
      }
    }
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
    det_out[mat] = d;
    if (logabs_out) logabs_out[mat] = la;
  }
}

}  // namespace

// Cluster size for an n x n factorisation (0: does not fit): the smallest of
// 8 (portable) and 16 whose column slab fits the shared memory of one CTA and
// of which the device can co-schedule a cluster.
static int lu_cluster_size(int device, int n) {
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  for (int C : {8, 16}) {
    const size_t bytes = luc_smem_bytes(n, C);
    if (bytes + 2048 > (size_t)max_smem) continue;
    if (cudaFuncSetAttribute(lu_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes) != cudaSuccess)
      return 0;
    if (C > 8 && cudaFuncSetAttribute(lu_cluster_kernel,
                                      cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                     cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(LUC_THREADS);
    cfg.dynamicSmemBytes = bytes;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, lu_cluster_kernel, &cfg) == cudaSuccess &&
        clusters > 0)
      return C;
    cudaGetLastError();
  }
  return 0;
}

static int run_lu_cluster(kls_ctx* c, int n, int C) {
  const size_t bytes = luc_smem_bytes(c->Na, C);
  // the limit is a property of the kernel shared by all contexts: set it for
  // this context's N right before its launch (another context may have set
  // a smaller one)
  KLS_CK(c, cudaFuncSetAttribute(lu_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(n * C);
  cfg.blockDim = dim3(LUC_THREADS);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = c->stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  KLS_CK(c, cudaLaunchKernelEx(&cfg, lu_cluster_kernel, c->Na, (const double2*)c->d_A, c->d_det,
                               c->d_logabs));
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_run_lu(kls_ctx* c, int n) {
  // latency form (a cluster per matrix) for the N_alpha of the benchmark
  // sizes when the batch fits one wave; otherwise one CTA per matrix
  if (c->lu_mode != KLS_LU_CTA) {
    if (c->lu_cluster < 0) c->lu_cluster = lu_cluster_size(c->device, c->Na);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const bool want = c->lu_mode == KLS_LU_CLUSTER ||
                      (c->Na >= 128 && (int64_t)n * c->lu_cluster <= sms);
    if (want && c->lu_cluster > 0) return run_lu_cluster(c, n, c->lu_cluster);
    if (c->lu_mode == KLS_LU_CLUSTER)
      return kls_fail(c, KLS_ERR_UNSUPPORTED, "cluster LU does not fit this N_alpha");
  }
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

// Learned root proposer: a small MLP trained on the device by this file's own
// BF16 tensor-core kernels (no library GEMM).
//
//   features (5) -> [W1, b1, GELU] -> width -> ... -> [W_L, b_L] -> outputs (3)
//
// Parameters are FP32 masters (Adam moments FP32); every GEMM runs on BF16
// copies with FP32 accumulation (mma.sync m16n8k16 bf16 -> f32).  Each GEMM
// computes C[M x N] = A[M x K] * B[N x K]^T with both operands K-contiguous:
//   forward   Z_l  = H_{l-1} W_l^T + b_l        (A = H_{l-1}, B = W_l)
//   backward  dW_l = dZ_l^T H_{l-1}             (A = dZ_l^T, B = H_{l-1}^T)
//             dH   = dZ_l W_l                   (A = dZ_l,   B = W_l^T)
// so the epilogues also write transposed BF16 copies (H^T, dZ^T) and the
// update writes W and W^T in BF16.  GELU is the erf form
// 0.5 x (1 + erf(x / sqrt 2)).  The loss is the mean squared error over the
// batch and the outputs.
#include "kls_internal.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

struct kls_mlp;

namespace {

constexpr int ML_IN = 5, ML_OUT = 3;
constexpr int ML_PAD = 16;            // input / output dims padded to 16 for the MMA
constexpr int GT_BM = 64, GT_BN = 64, GT_BK = 32, GT_THREADS = 128;
constexpr int GT_LDS = GT_BK + 8;     // bf16 row stride in shared memory

enum Epi { EPI_STORE = 0, EPI_BIAS_GELU = 1, EPI_BIAS = 2, EPI_GELU_BWD = 3 };

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16* A; int lda;     // A[m][k] at A[m * lda + k]
  const __nv_bfloat16* B; int ldb;     // B[n][k] at B[n * ldb + k]
  float* C; int ldc;                   // fp32 output (may be null)
  const float* bias;                   // [N]
  const float* Zin; int ldz;           // pre-activations for EPI_GELU_BWD
  __nv_bfloat16* H; int ldh;           // bf16 output [M][N]
  __nv_bfloat16* Ht; int ldht;         // bf16 transposed output [N][M]
};

__device__ __forceinline__ float gelu_f(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int EPI>
__global__ void __launch_bounds__(GT_THREADS) gemm_bf16_kernel(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 sA[GT_BM * GT_LDS];
  __shared__ __align__(16) __nv_bfloat16 sB[GT_BN * GT_LDS];
  const int m0 = blockIdx.y * GT_BM, n0 = blockIdx.x * GT_BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int gid = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int t = 0; t < 4; ++t) acc[i][j][t] = 0.f;

  for (int k0 = 0; k0 < g.K; k0 += GT_BK) {
    // stage tiles (zero outside the matrices)
    for (int e = tid; e < GT_BM * GT_BK; e += GT_THREADS) {
      int r = e / GT_BK, kk = e % GT_BK;
      int gm = m0 + r, gk = k0 + kk;
      sA[r * GT_LDS + kk] = (gm < g.M && gk < g.K) ? g.A[(size_t)gm * g.lda + gk]
                                                   : __float2bfloat16(0.f);
      int gn = n0 + r;
      sB[r * GT_LDS + kk] = (gn < g.N && gk < g.K) ? g.B[(size_t)gn * g.ldb + gk]
                                                   : __float2bfloat16(0.f);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GT_BK; ks += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const __nv_bfloat16* p = sA + (wm + i * 16 + gid) * GT_LDS + ks + tig * 2;
        af[i][0] = *reinterpret_cast<const uint32_t*>(p);
        af[i][1] = *reinterpret_cast<const uint32_t*>(p + 8 * GT_LDS);
        af[i][2] = *reinterpret_cast<const uint32_t*>(p + 8);
        af[i][3] = *reinterpret_cast<const uint32_t*>(p + 8 * GT_LDS + 8);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat16* p = sB + (wn + j * 8 + gid) * GT_LDS + ks + tig * 2;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(p);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(p + 8);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
  // epilogue: fragment element t at row gid (+8 for t >= 2), col 2 tig + (t & 1)
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int r = m0 + wm + i * 16 + gid + (t >= 2 ? 8 : 0);
        const int cidx = n0 + wn + j * 8 + 2 * tig + (t & 1);
        if (r >= g.M || cidx >= g.N) continue;
        float v = acc[i][j][t];
        if (EPI == EPI_BIAS_GELU || EPI == EPI_BIAS) v += g.bias[cidx];
        if (g.C) g.C[(size_t)r * g.ldc + cidx] = v;
        float h = v;
        if (EPI == EPI_BIAS_GELU) h = gelu_f(v);
        if (EPI == EPI_GELU_BWD) h = v * gelu_d(g.Zin[(size_t)r * g.ldz + cidx]);
        if (EPI == EPI_GELU_BWD && g.C) g.C[(size_t)r * g.ldc + cidx] = h;
        if (g.H) g.H[(size_t)r * g.ldh + cidx] = __float2bfloat16(h);
        if (g.Ht) g.Ht[(size_t)cidx * g.ldht + r] = __float2bfloat16(h);
      }
}

// dY = 2 (Y - T) / (B * OUT) into fp32, bf16 and bf16^T; loss partial sums
__global__ void mse_grad_kernel(int Bn, const float* __restrict__ Y, const float* __restrict__ T,
                                float* __restrict__ dY, __nv_bfloat16* __restrict__ dYb,
                                __nv_bfloat16* __restrict__ dYt, int ldt, float* __restrict__ loss) {
  float s = 0.f;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Bn * ML_PAD; e += gridDim.x * blockDim.x) {
    const int r = e / ML_PAD, c = e % ML_PAD;
    float g = 0.f;
    if (c < ML_OUT) {
      const float d = Y[(size_t)r * ML_PAD + c] - T[(size_t)r * ML_OUT + c];
      s += d * d;
      g = 2.f * d / (float)(Bn * ML_OUT);
    }
    dY[e] = g;
    dYb[e] = __float2bfloat16(g);
    dYt[(size_t)c * ldt + r] = __float2bfloat16(g);
  }
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (float)(Bn * ML_OUT));
}

// column sums of dZ [B][N] -> db[N] (deterministic: one thread per column)
__global__ void colsum_kernel(int Bn, int N, int ld, const float* __restrict__ dZ,
                              float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.f;
  for (int r = 0; r < Bn; ++r) s += dZ[(size_t)r * ld + c];
  db[c] = s;
}

__global__ void adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// fp32 weights [rows][cols] -> bf16 W [rows_pad][cols_pad] and W^T [cols_pad][rows_pad]
__global__ void pack_weights_kernel(int rows, int cols, int rows_pad, int cols_pad,
                                    const float* __restrict__ w, __nv_bfloat16* __restrict__ Wb,
                                    __nv_bfloat16* __restrict__ Wt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows_pad * cols_pad;
       e += gridDim.x * blockDim.x) {
    const int r = e / cols_pad, c = e % cols_pad;
    const float x = (r < rows && c < cols) ? w[(size_t)r * cols + c] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16(x);
    Wb[e] = b;
    Wt[(size_t)c * rows_pad + r] = b;
  }
}

// features fp32 [B][5] -> bf16 [B][16] and its transpose [16][B]
__global__ void pack_input_kernel(int Bn, const float* __restrict__ X, __nv_bfloat16* __restrict__ Xb,
                                  __nv_bfloat16* __restrict__ Xt, int ldt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Bn * ML_PAD; e += gridDim.x * blockDim.x) {
    const int r = e / ML_PAD, c = e % ML_PAD;
    const __nv_bfloat16 b = __float2bfloat16(c < ML_IN ? X[(size_t)r * ML_IN + c] : 0.f);
    Xb[e] = b;
    Xt[(size_t)c * ldt + r] = b;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
struct kls_mlp {
  int device = 0, width = 256, depth = 4, cap = 0;  // depth = number of linear layers
  std::vector<int> din, dout, din_pad, dout_pad;    // per layer
  std::vector<int64_t> woff, boff;                  // offsets into the flat fp32 params
  int64_t nparams = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  std::vector<__nv_bfloat16*> Wb, Wt;
  // activations for a batch of `cap` rows
  std::vector<float*> Z;                             // pre-activations [cap][dout_pad]
  std::vector<__nv_bfloat16*> H, Ht;                 // H[l]: input of layer l [cap][din_pad]
  float *dZ = nullptr, *dZ2 = nullptr;               // fp32 [cap][width]
  __nv_bfloat16 *dZb = nullptr, *dZb2 = nullptr;    // bf16 [cap][width] (ping-pong)
  __nv_bfloat16 *dZt = nullptr;                      // bf16 [width][cap]
  float *Xd = nullptr, *Td = nullptr, *loss = nullptr;
  int64_t step = 0;
  cudaStream_t stream = nullptr;
  std::string err;
};

namespace {

int mfail(kls_mlp* m, const std::string& s) {
  if (m) m->err = s;
  return kls_fail(nullptr, KLS_ERR_CUDA, s);
}
#define ML_CK(m, call)                                                            \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) return mfail(m, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int ensure_cap(kls_mlp* m, int n) {
  if (n <= m->cap) return KLS_OK;
  int cap = ((n + 63) / 64) * 64;
  auto fr = [](void* p) { if (p) cudaFree(p); };
  for (auto* z : m->Z) fr(z);
  for (auto* h : m->H) fr(h);
  for (auto* h : m->Ht) fr(h);
  fr(m->dZ); fr(m->dZ2); fr(m->dZb); fr(m->dZb2); fr(m->dZt); fr(m->Xd); fr(m->Td);
  const int L = m->depth;
  m->Z.assign(L, nullptr);
  m->H.assign(L + 1, nullptr);
  m->Ht.assign(L + 1, nullptr);
  for (int l = 0; l < L; ++l) ML_CK(m, cudaMalloc(&m->Z[l], (size_t)cap * m->dout_pad[l] * 4));
  for (int l = 0; l <= L; ++l) {
    int w = l < L ? m->din_pad[l] : ML_PAD;
    ML_CK(m, cudaMalloc(&m->H[l], (size_t)cap * w * 2));
    ML_CK(m, cudaMalloc(&m->Ht[l], (size_t)cap * w * 2));
  }
  ML_CK(m, cudaMalloc(&m->dZ, (size_t)cap * m->width * 4));
  ML_CK(m, cudaMalloc(&m->dZ2, (size_t)cap * m->width * 4));
  ML_CK(m, cudaMalloc(&m->dZb, (size_t)cap * m->width * 2));
  ML_CK(m, cudaMalloc(&m->dZb2, (size_t)cap * m->width * 2));
  ML_CK(m, cudaMalloc(&m->dZt, (size_t)cap * m->width * 2));
  ML_CK(m, cudaMalloc(&m->Xd, (size_t)cap * ML_IN * 4));
  ML_CK(m, cudaMalloc(&m->Td, (size_t)cap * ML_OUT * 4));
  m->cap = cap;
  return KLS_OK;
}

template <int EPI>
int gemm(kls_mlp* m, const GemmArgs& g) {
  dim3 grid((g.N + GT_BN - 1) / GT_BN, (g.M + GT_BM - 1) / GT_BM);
  gemm_bf16_kernel<EPI><<<grid, GT_THREADS, 0, m->stream>>>(g);
  ML_CK(m, cudaGetLastError());
  return KLS_OK;
}

int pack_all(kls_mlp* m) {
  for (int l = 0; l < m->depth; ++l) {
    int n = m->dout_pad[l] * m->din_pad[l];
    pack_weights_kernel<<<(n + 255) / 256, 256, 0, m->stream>>>(
        m->dout[l], m->din[l], m->dout_pad[l], m->din_pad[l], m->p + m->woff[l], m->Wb[l], m->Wt[l]);
    ML_CK(m, cudaGetLastError());
  }
  return KLS_OK;
}

// forward over n rows already in m->Xd; output Z[L-1] [n][16]
int forward(kls_mlp* m, int n) {
  pack_input_kernel<<<(n * ML_PAD + 255) / 256, 256, 0, m->stream>>>(n, m->Xd, m->H[0], m->Ht[0],
                                                                     m->cap);
  ML_CK(m, cudaGetLastError());
  const int L = m->depth;
  for (int l = 0; l < L; ++l) {
    GemmArgs g{};
    g.M = n; g.N = m->dout_pad[l]; g.K = m->din_pad[l];
    g.A = m->H[l]; g.lda = m->din_pad[l];
    g.B = m->Wb[l]; g.ldb = m->din_pad[l];
    g.C = m->Z[l]; g.ldc = m->dout_pad[l];
    g.bias = nullptr;
    int r;
    if (l < L - 1) {
      g.bias = m->p + m->boff[l];
      g.H = m->H[l + 1]; g.ldh = m->din_pad[l + 1];
      g.Ht = m->Ht[l + 1]; g.ldht = m->cap;
      r = gemm<EPI_BIAS_GELU>(m, g);
    } else {
      // the last layer's bias covers only the 3 real outputs; padded columns
      // of the bias vector are zero-filled by a separate padded bias copy
      g.bias = m->p + m->boff[l];
      r = gemm<EPI_BIAS>(m, g);
    }
    if (r) return r;
  }
  return KLS_OK;
}

// backward from dZ_last (fp32 [n][16] in m->dZ2 reinterpreted, bf16 copies ready)
int backward(kls_mlp* m, int n) {
  const int L = m->depth;
  float* dZcur = m->dZ2;           // fp32 dZ of layer l, [n][dout_pad[l]]
  __nv_bfloat16* dZbcur = m->dZb;  // its bf16 copy (the GEMM below reads one, writes the other)
  for (int l = L - 1; l >= 0; --l) {
    // dW_l [dout][din] = dZ_l^T (dout x n) * H_l (n x din): A = dZt [dout_pad][cap], B = Ht_l
    {
      GemmArgs g{};
      g.M = m->dout[l]; g.N = m->din[l]; g.K = n;
      g.A = m->dZt; g.lda = m->cap;
      g.B = m->Ht[l]; g.ldb = m->cap;
      g.C = m->g + m->woff[l]; g.ldc = m->din[l];
      int r = gemm<EPI_STORE>(m, g);
      if (r) return r;
    }
    colsum_kernel<<<(m->dout[l] + 127) / 128, 128, 0, m->stream>>>(n, m->dout[l], m->dout_pad[l],
                                                                   dZcur, m->g + m->boff[l]);
    ML_CK(m, cudaGetLastError());
    if (l == 0) break;
    // dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1}): A = dZb [n][dout_pad], B = Wt_l [din_pad][dout_pad]
    float* dZnext = (dZcur == m->dZ) ? m->dZ2 : m->dZ;
    __nv_bfloat16* dZbnext = (dZbcur == m->dZb) ? m->dZb2 : m->dZb;
    GemmArgs g{};
    g.M = n; g.N = m->din_pad[l]; g.K = m->dout_pad[l];
    g.A = dZbcur; g.lda = m->dout_pad[l];
    g.B = m->Wt[l]; g.ldb = m->dout_pad[l];
    g.C = dZnext; g.ldc = m->din_pad[l];
    g.Zin = m->Z[l - 1]; g.ldz = m->dout_pad[l - 1];
    // dZ^T is read only by the dW GEMM that already ran, so it is rewritten
    // in place; the bf16 dZ ping-pongs because this GEMM reads the other one
    g.H = dZbnext; g.ldh = m->din_pad[l];
    g.Ht = m->dZt; g.ldht = m->cap;
    int r = gemm<EPI_GELU_BWD>(m, g);
    if (r) return r;
    dZcur = dZnext;
    dZbcur = dZbnext;
  }
  return KLS_OK;
}

// loss + gradients over rows [0, n) of Xd/Td into m->g; loss into *loss_out (device)
int grad_batch(kls_mlp* m, int n) {
  int r;
  if ((r = forward(m, n))) return r;
  mse_grad_kernel<<<std::min((n * ML_PAD + 255) / 256, 1024), 256, 0, m->stream>>>(
      n, m->Z[m->depth - 1], m->Td, m->dZ2, m->dZb, m->dZt, m->cap, m->loss);
  ML_CK(m, cudaGetLastError());
  return backward(m, n);
}

}  // namespace

extern "C" {

int kls_mlp_create(int device, int width, int depth, uint64_t seed, kls_mlp** out) {
  if (!out || width < 16 || width % 16 || depth < 2 || depth > 16)
    return kls_fail(nullptr, KLS_ERR_CONFIG, "kls_mlp_create: bad arguments");
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return kls_fail(nullptr, KLS_ERR_CUDA, cudaGetErrorString(e));
  kls_mlp* m = new kls_mlp();
  m->device = device; m->width = width; m->depth = depth;
  for (int l = 0; l < depth; ++l) {
    int di = l == 0 ? ML_IN : width, dO = l == depth - 1 ? ML_OUT : width;
    m->din.push_back(di); m->dout.push_back(dO);
    m->din_pad.push_back(l == 0 ? ML_PAD : width);
    m->dout_pad.push_back(l == depth - 1 ? ML_PAD : width);
    m->woff.push_back(m->nparams); m->nparams += (int64_t)di * dO;
    m->boff.push_back(m->nparams); m->nparams += dO;
  }
  // the last bias is read for all 16 padded outputs: reserve 13 zero floats after it
  const int64_t alloc = m->nparams + ML_PAD;
  std::vector<float> h(alloc, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < depth; ++l) {
    const float bound = 1.0f / std::sqrt((float)m->din[l]);   // uniform(-1/sqrt(fan_in), ..)
    std::uniform_real_distribution<float> U(-bound, bound);
    for (int64_t i = 0; i < (int64_t)m->din[l] * m->dout[l]; ++i) h[m->woff[l] + i] = U(rng);
    for (int i = 0; i < m->dout[l]; ++i) h[m->boff[l] + i] = U(rng);
  }
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&m->p, alloc * 4) != cudaSuccess || cudaMalloc(&m->g, alloc * 4) != cudaSuccess ||
      cudaMalloc(&m->m, alloc * 4) != cudaSuccess || cudaMalloc(&m->v, alloc * 4) != cudaSuccess ||
      cudaMalloc(&m->loss, 4) != cudaSuccess) {
    delete m;
    return kls_fail(nullptr, KLS_ERR_OOM, "kls_mlp_create: device allocation failed");
  }
  cudaMemcpy(m->p, h.data(), alloc * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->g, 0, alloc * 4);
  cudaMemset(m->m, 0, alloc * 4);
  cudaMemset(m->v, 0, alloc * 4);
  for (int l = 0; l < depth; ++l) {
    __nv_bfloat16 *a = nullptr, *b = nullptr;
    size_t n = (size_t)m->dout_pad[l] * m->din_pad[l];
    if (cudaMalloc(&a, n * 2) != cudaSuccess || cudaMalloc(&b, n * 2) != cudaSuccess)
      return kls_fail(nullptr, KLS_ERR_OOM, "kls_mlp_create: device allocation failed");
    m->Wb.push_back(a); m->Wt.push_back(b);
  }
  int r = pack_all(m);
  if (r) return r;
  if (cudaStreamSynchronize(m->stream) != cudaSuccess)
    return kls_fail(nullptr, KLS_ERR_CUDA, "kls_mlp_create: init failed");
  *out = m;
  return KLS_OK;
}

int kls_mlp_destroy(kls_mlp* m) {
  if (!m) return KLS_OK;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(m->p); fr(m->g); fr(m->m); fr(m->v); fr(m->loss);
  for (auto* x : m->Wb) fr(x);
  for (auto* x : m->Wt) fr(x);
  for (auto* z : m->Z) fr(z);
  for (auto* x : m->H) fr(x);
  for (auto* x : m->Ht) fr(x);
  fr(m->dZ); fr(m->dZ2); fr(m->dZb); fr(m->dZb2); fr(m->dZt); fr(m->Xd); fr(m->Td);
  cudaStreamDestroy(m->stream);
  delete m;
  return KLS_OK;
}

int kls_mlp_num_params(const kls_mlp* m, int64_t* n) {
  if (!m || !n) return KLS_ERR_CONFIG;
  *n = m->nparams;
  return KLS_OK;
}

int kls_mlp_get_params(kls_mlp* m, float* params) {
  if (!m || !params) return KLS_ERR_CONFIG;
  cudaSetDevice(m->device);
  ML_CK(m, cudaMemcpy(params, m->p, m->nparams * 4, cudaMemcpyDeviceToHost));
  return KLS_OK;
}

int kls_mlp_set_params(kls_mlp* m, const float* params) {
  if (!m || !params) return KLS_ERR_CONFIG;
  cudaSetDevice(m->device);
  ML_CK(m, cudaMemcpy(m->p, params, m->nparams * 4, cudaMemcpyHostToDevice));
  int r = pack_all(m);
  if (r) return r;
  ML_CK(m, cudaStreamSynchronize(m->stream));
  return KLS_OK;
}

// Inference: X [n][5] host -> Y [n][3] host
int kls_mlp_forward(kls_mlp* m, const float* X, int n, float* Y) {
  if (!m || n < 0 || (n && (!X || !Y))) return KLS_ERR_CONFIG;
  cudaSetDevice(m->device);
  const int chunk = 1 << 16;
  std::vector<float> z((size_t)std::min(n, chunk) * ML_PAD);
  for (int s = 0; s < n; s += chunk) {
    int nb = std::min(chunk, n - s);
    int r = ensure_cap(m, nb);
    if (r) return r;
    ML_CK(m, cudaMemcpyAsync(m->Xd, X + (size_t)s * ML_IN, (size_t)nb * ML_IN * 4,
                             cudaMemcpyHostToDevice, m->stream));
    if ((r = forward(m, nb))) return r;
    ML_CK(m, cudaMemcpyAsync(z.data(), m->Z[m->depth - 1], (size_t)nb * ML_PAD * 4,
                             cudaMemcpyDeviceToHost, m->stream));
    ML_CK(m, cudaStreamSynchronize(m->stream));
    for (int i = 0; i < nb; ++i)
      for (int c = 0; c < ML_OUT; ++c) Y[(size_t)(s + i) * ML_OUT + c] = z[(size_t)i * ML_PAD + c];
  }
  return KLS_OK;
}

// Loss and full-batch gradients (no update), for gradient checks
int kls_mlp_grad(kls_mlp* m, const float* X, const float* T, int n, float* grads, float* loss) {
  if (!m || n < 1 || !X || !T) return KLS_ERR_CONFIG;
  cudaSetDevice(m->device);
  int r = ensure_cap(m, n);
  if (r) return r;
  ML_CK(m, cudaMemcpyAsync(m->Xd, X, (size_t)n * ML_IN * 4, cudaMemcpyHostToDevice, m->stream));
  ML_CK(m, cudaMemcpyAsync(m->Td, T, (size_t)n * ML_OUT * 4, cudaMemcpyHostToDevice, m->stream));
  ML_CK(m, cudaMemsetAsync(m->loss, 0, 4, m->stream));
  if ((r = grad_batch(m, n))) return r;
  if (grads) ML_CK(m, cudaMemcpyAsync(grads, m->g, m->nparams * 4, cudaMemcpyDeviceToHost, m->stream));
  if (loss) ML_CK(m, cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
  ML_CK(m, cudaStreamSynchronize(m->stream));
  return KLS_OK;
}

// Adam training: epochs over shuffled minibatches; loss_hist[e] = mean batch loss
int kls_mlp_train(kls_mlp* m, const float* X, const float* T, int n, int epochs, int batch,
                  float lr, uint64_t seed, float* loss_hist) {
  if (!m || n < 1 || batch < 1 || epochs < 0 || !X || !T) return KLS_ERR_CONFIG;
  cudaSetDevice(m->device);
  batch = std::min(batch, n);
  int r = ensure_cap(m, batch);
  if (r) return r;
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::mt19937_64 rng(seed);
  std::vector<float> xb((size_t)batch * ML_IN), tb((size_t)batch * ML_OUT);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(idx.begin(), idx.end(), rng);
    double lsum = 0.0;
    int nb_count = 0;
    for (int s = 0; s + batch <= n; s += batch) {
      for (int i = 0; i < batch; ++i) {
        std::memcpy(&xb[(size_t)i * ML_IN], X + (size_t)idx[s + i] * ML_IN, ML_IN * 4);
        std::memcpy(&tb[(size_t)i * ML_OUT], T + (size_t)idx[s + i] * ML_OUT, ML_OUT * 4);
      }
      ML_CK(m, cudaMemcpyAsync(m->Xd, xb.data(), xb.size() * 4, cudaMemcpyHostToDevice, m->stream));
      ML_CK(m, cudaMemcpyAsync(m->Td, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice, m->stream));
      ML_CK(m, cudaMemsetAsync(m->loss, 0, 4, m->stream));
      if ((r = grad_batch(m, batch))) return r;
      ++m->step;
      const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
      adam_kernel<<<256, 256, 0, m->stream>>>(m->nparams, m->p, m->g, m->m, m->v, lr, b1, b2, eps,
                                             c1, c2);
      ML_CK(m, cudaGetLastError());
      if ((r = pack_all(m))) return r;
      float l = 0.f;
      ML_CK(m, cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
      ML_CK(m, cudaStreamSynchronize(m->stream));
      lsum += l;
      ++nb_count;
    }
    if (loss_hist) loss_hist[ep] = nb_count ? (float)(lsum / nb_count) : 0.f;
  }
  return KLS_OK;
}

}  // extern "C"

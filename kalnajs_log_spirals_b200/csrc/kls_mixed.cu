// Split-BF16 tensor-core contraction (KLS_MODE_MIXED) on tcgen05 / TMEM.
//
// M(omega) = W^T diag(w(omega)) conj(W) as one real GEMM per omega:
//
//   X = [Re W | Im W]                 (rows c in [0, 2 Npad), K-major, omega-independent)
//   Y = [U_r | U_i], U = w * conj(W)  (rows n = 2 a + part, K-major, per omega)
//   P = X Y^T (2 Npad x 2 Npad)
//   M_r[b,a] = P[b, 2a] - P[Npad+b, 2a+1],  M_i[b,a] = P[b, 2a+1] + P[Npad+b, 2a]
//
// Both operands are split error-free into BF16 high and low parts
// (x = hi + lo to ~2^-17 relative) and P accumulates hi*hi + hi*lo + lo*hi on
// the tensor cores with FP32 accumulation in TMEM (the lo*lo term, ~2^-18
// relative, is dropped).  FP32 accumulation error grows with the length of
// the accumulation chain, so TMEM is flushed every MX_CHUNK_KB k-blocks into
// an FP64 partial in global memory (deterministic order); the split-K
// reduction, the weights w(omega), the LU and the determinant are FP64.
//
// Table: Xh/Xl BF16 in 64-k blocks, element (row r, k) at
// (k / 64) * (2 Npad * 64) + r * 64 + k % 64 (each block of 64 k over all
// rows contiguous, so that one stage reads a few pages rather than one page
// per table row), built once by split_table_kernel from
// the FP64 table.  Contraction CTA (one per SM, 16 warps):
//   warp 0       TMA: X tile 128 rows x 64 k (hi, lo; 128B swizzle)
//   warp 3       bulk copies of the FP32 weights into their own 8-deep ring,
//                so the producers never wait for them on the critical path
//   warp 1       MMA issuer: tcgen05.mma kind::f16 M=128 N=128 K=16, 3
//                products per k-step per omega, 2 TMEM accumulator buffers
//   warp 2       TMEM allocation / release (512 columns)
//   warps 4-11   producers: U = w conj(W) in FP32 from the table rows of the
//                CTA's alpha block (prefetched one stage ahead), split to
//                BF16 hi/lo, stored 128B-swizzled (K-major) for 2 omegas
//   warps 12-15  drain: per chunk, tcgen05.ld -> add into the FP64 partial
// Every mbarrier wait is bounded by %globaltimer; a timeout aborts the CTA
// (error flag for the host), and TMEM is released only after all issued MMAs
// have completed.
#include "kls_internal.cuh"
#include "kls_tcgen05.cuh"
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstring>

namespace {

constexpr int MX_BM = 128;                 // X rows per CTA
constexpr int MX_AB = 64;                  // alphas per CTA -> 128 Y rows per omega
constexpr int MX_BN = 2 * MX_AB;           // 128
constexpr int MX_OMEGA = 2;                // omegas per CTA
constexpr int MX_BK = 64;                  // k per stage: one 128-byte swizzle row of BF16
constexpr int MX_STAGES = 2;
constexpr int MX_CHUNK_KB = 32;            // k-blocks per TMEM accumulation chunk
constexpr int MX_PRODUCERS = 256;          // warps 4..11
constexpr int MX_DRAIN0 = 12;              // first drain warp (warps 12..15)
constexpr int MX_THREADS = 512;
constexpr int MX_TILE_X = MX_BM * MX_BK * 2;            // 16 KB per part
constexpr int MX_TILE_Y = MX_BN * MX_BK * 2;            // 16 KB per part per omega
constexpr int MX_W_BYTES = MX_BK * 8;                   // float2 weights per omega per stage
constexpr int MX_WSTAGES = 8;              // weights ring: filled up to 8 k-blocks ahead
constexpr int MX_STAGE_BYTES = 2 * MX_TILE_X + 2 * MX_OMEGA * MX_TILE_Y;          // 96 KB
constexpr int MX_WRING_BYTES = MX_WSTAGES * MX_OMEGA * MX_W_BYTES;                // 8 KB
constexpr size_t MX_SMEM = (size_t)MX_STAGES * MX_STAGE_BYTES + MX_WRING_BYTES + 1024;
constexpr int MX_ACC_COLS = MX_OMEGA * MX_BN;          // 256 fp32 columns per buffer
constexpr int MX_TMEM_COLS = 2 * MX_ACC_COLS;          // 512
constexpr unsigned long long MX_WAIT_NS = 2000000000ull;   // 2 s per wait

using namespace kls_tc;

// bounded waits of the legacy kernels: the fixed MX_WAIT_NS bound
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int* abort,
                                          int* err, int code) {
  return mbar_wait_lim(a, parity, abort, err, code, MX_WAIT_NS);
}
__device__ __forceinline__ bool mbar_wait_cl(uint32_t a, uint32_t parity, volatile int* abort,
                                             int* err, int code) {
  return mbar_wait_cl_lim(a, parity, abort, err, code, MX_WAIT_NS);
}

struct MixedParams {
  int Npad;            // N_alpha_pad
  int rows;            // 2 * Npad
  int64_t K_pad;
  int nkb_total;       // K_pad / MX_BK
  int kb_per_split;
  int splits;
  int n_omega;
  int tiles_a;
};

// ---- error-free split of the FP64 table --------------------------------------
__device__ __forceinline__ void split2(double v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn((float)v);
  lo = __float2bfloat16_rn((float)(v - (double)__bfloat162float(hi)));
}

// [K_pad][Npad] FP64 planes -> X{h,l}, rows a (Re) and Npad + a (Im), in
// 64-k blocks: element (r, k) at (k / 64) * (2 Npad * 64) + r * 64 + k % 64
__global__ void split_table_kernel(const double* __restrict__ Wre, const double* __restrict__ Wim,
                                   int Npad, int64_t K_pad, __nv_bfloat16* __restrict__ Xh,
                                   __nv_bfloat16* __restrict__ Xl) {
  (void)K_pad;
  const size_t blk = (size_t)2 * Npad * MX_BK;      // elements of one 64-k block
  __shared__ double tr[32][33], ti[32][33];
  const int64_t k0 = (int64_t)blockIdx.x * 32;
  const int a0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < 32; i += 8) {
    tr[i][tx] = Wre[(size_t)(k0 + i) * Npad + a0 + tx];
    ti[i][tx] = Wim[(size_t)(k0 + i) * Npad + a0 + tx];
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    __nv_bfloat16 h, l;
    split2(tr[tx][i], h, l);
    const int64_t k = k0 + tx;
    size_t o = (size_t)(k >> 6) * blk + (size_t)(a0 + i) * MX_BK + (k & 63);
    Xh[o] = h;
    Xl[o] = l;
    split2(ti[tx][i], h, l);
    o = (size_t)(k >> 6) * blk + (size_t)(Npad + a0 + i) * MX_BK + (k & 63);
    Xh[o] = h;
    Xl[o] = l;
  }
}

// FP32 copy of the weights, permuted inside each 64-k block so that the
// producers' 16-byte reads (k-chunk c of 8, pair q of 2) are conflict-free:
// k = 8c + 2q + h is stored at position 2 (8q + c) + h of its block.
__global__ void weights32_kernel(int64_t total, const double2* __restrict__ wt,
                                 float2* __restrict__ wt32) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = wt[i];
    const int k = (int)(i & (MX_BK - 1));
    const int c = k >> 3, q = (k >> 1) & 3, h = k & 1;
    wt32[(i & ~(int64_t)(MX_BK - 1)) + 2 * (8 * q + c) + h] = make_float2((float)v.x, (float)v.y);
  }
}

// ---- contraction -------------------------------------------------------------
__global__ void __launch_bounds__(MX_THREADS, 1)
mixed_contract_kernel(const __grid_constant__ CUtensorMap tm_h,
                      const __grid_constant__ CUtensorMap tm_l, MixedParams P,
                      const __nv_bfloat16* __restrict__ Xh, const __nv_bfloat16* __restrict__ Xl,
                      const float2* __restrict__ wt32, double* __restrict__ part,
                      int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full_x[MX_STAGES], bar_full_y[MX_STAGES],
      bar_empty[MX_STAGES], bar_w_full[MX_WSTAGES], bar_w_empty[MX_WSTAGES], bar_acc_full[2],
      bar_acc_empty[2], bar_done;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x, split = blockIdx.y, grp = blockIdx.z;
  const int tm = tile / P.tiles_a, ta = tile % P.tiles_a;
  const int m0 = tm * MX_BM;             // first X row
  const int a0 = ta * MX_AB;             // first alpha
  const int om0 = grp * MX_OMEGA;
  const int n_om = min(MX_OMEGA, P.n_omega - om0);
  const int kb0 = split * P.kb_per_split;
  const int nkb = max(0, min(P.nkb_total, kb0 + P.kb_per_split) - kb0);
  const int nch = (nkb + MX_CHUNK_KB - 1) / MX_CHUNK_KB;

  auto xh_s = [&](int s) { return smem + (size_t)s * MX_STAGE_BYTES; };
  auto xl_s = [&](int s) { return smem + (size_t)s * MX_STAGE_BYTES + MX_TILE_X; };
  auto yh_s = [&](int s, int j) {
    return smem + (size_t)s * MX_STAGE_BYTES + 2 * MX_TILE_X + (size_t)j * MX_TILE_Y;
  };
  auto yl_s = [&](int s, int j) {
    return smem + (size_t)s * MX_STAGE_BYTES + 2 * MX_TILE_X + (size_t)(MX_OMEGA + j) * MX_TILE_Y;
  };
  auto w_s = [&](int ws, int j) {
    return reinterpret_cast<float2*>(smem + (size_t)MX_STAGES * MX_STAGE_BYTES +
                                     (size_t)ws * MX_OMEGA * MX_W_BYTES) + j * MX_BK;
  };

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < MX_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full_x[s]), 1);
      mbar_init(smem_u32(&bar_full_y[s]), MX_PRODUCERS / 32);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int s = 0; s < MX_WSTAGES; ++s) {
      mbar_init(smem_u32(&bar_w_full[s]), 1);
      mbar_init(smem_u32(&bar_w_empty[s]), MX_PRODUCERS / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_acc_full[b]), 1);
      mbar_init(smem_u32(&bar_acc_empty[b]), 4);
    }
    mbar_init(smem_u32(&bar_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2 && nkb > 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(MX_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const size_t R = (size_t)P.rows;

  if (warp == 0) {
    // ---------------- TMA: X tiles
    if (lane == 0 && nkb > 0) {
      int issued = 0;
      for (int i = 0; i < nkb; ++i) {
        const int s = i % MX_STAGES, r = i / MX_STAGES;
        if (!mbar_wait(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort, err, 1)) break;
        const uint32_t fb = smem_u32(&bar_full_x[s]);
        mbar_arrive_tx(fb, 2 * MX_TILE_X);
        tma_load_3d(smem_u32(xh_s(s)), &tm_h, 0, m0, kb0 + i, fb);
        tma_load_3d(smem_u32(xl_s(s)), &tm_l, 0, m0, kb0 + i, fb);
        issued = i + 1;
      }
      // the last copies into each stage land before the CTA may exit
      for (int i = max(0, issued - MX_STAGES); i < issued; ++i)
        mbar_wait(smem_u32(&bar_full_x[i % MX_STAGES]), (i / MX_STAGES) & 1, nullptr, err, 6);
    }
  } else if (warp == 3) {
    // ---------------- weights ring: bulk copies up to MX_WSTAGES k-blocks ahead
    if (lane == 0 && nkb > 0) {
      int issued = 0;
      for (int i = 0; i < nkb; ++i) {
        const int ws = i % MX_WSTAGES, r = i / MX_WSTAGES;
        if (!mbar_wait(smem_u32(&bar_w_empty[ws]), (r & 1) ^ 1, &s_abort, err, 10)) break;
        const int64_t kx = (int64_t)(kb0 + i) * MX_BK;
        const uint32_t wb = smem_u32(&bar_w_full[ws]);
        mbar_arrive_tx(wb, n_om * MX_W_BYTES);
        for (int j = 0; j < n_om; ++j)
          bulk_load(smem_u32(w_s(ws, j)), wt32 + (size_t)(om0 + j) * P.K_pad + kx, MX_W_BYTES, wb);
        issued = i + 1;
      }
      for (int i = max(0, issued - MX_WSTAGES); i < issued; ++i)
        mbar_wait(smem_u32(&bar_w_full[i % MX_WSTAGES]), (i / MX_WSTAGES) & 1, nullptr, err, 6);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0 && nkb > 0) {
      // the Y tiles of the CTA's omegas are adjacent in shared memory and the
      // accumulators adjacent in TMEM, so one MMA with N = 128 * n_om covers all
      // omegas (the operand reads per MAC bound this kernel: N = 256 halves the
      // A-tile reads of N = 128)
      const uint32_t idesc = idesc_bf16(MX_BM, MX_BN * n_om);
      for (int i = 0; i < nkb; ++i) {
        const int s = i % MX_STAGES, r = i / MX_STAGES;
        const int ch = i / MX_CHUNK_KB, b = ch & 1;
        const bool first = (i % MX_CHUNK_KB) == 0;
        const bool last = (i % MX_CHUNK_KB) == MX_CHUNK_KB - 1 || i == nkb - 1;
        if (first && !mbar_wait(smem_u32(&bar_acc_empty[b]), ((ch >> 1) & 1) ^ 1, &s_abort, err, 7))
          break;
        if (!mbar_wait(smem_u32(&bar_full_x[s]), r & 1, &s_abort, err, 2)) break;
        if (!mbar_wait(smem_u32(&bar_full_y[s]), r & 1, &s_abort, err, 3)) break;
        tc_fence_after();
        const uint64_t dxh = sw128_desc(smem_u32(xh_s(s)));
        const uint64_t dxl = sw128_desc(smem_u32(xl_s(s)));
        const uint32_t d = tmem + (uint32_t)(b * MX_ACC_COLS);
        const uint64_t dyh0 = sw128_desc(smem_u32(yh_s(s, 0)));
        const uint64_t dyl0 = sw128_desc(smem_u32(yl_s(s, 0)));
#pragma unroll
        for (int kk = 0; kk < MX_BK / 16; ++kk) {
          const uint64_t koff = (uint64_t)(kk * 32) >> 4;    // +32 bytes per k-step
          umma(d, dxh + koff, dyh0 + koff, idesc, (first && kk == 0) ? 0u : 1u);
          umma(d, dxh + koff, dyl0 + koff, idesc, 1u);
          umma(d, dxl + koff, dyh0 + koff, idesc, 1u);
        }
        umma_commit(smem_u32(&bar_empty[s]));
        if (last) umma_commit(smem_u32(&bar_acc_full[b]));
      }
      // completion of every issued MMA (also on the abort path)
      umma_commit(smem_u32(&bar_done));
    }
  } else if (warp >= 4 && warp < MX_DRAIN0) {
    // ---------------- producers: U = w conj(W), split, swizzled store
    const int pt = tid - 128;                 // 0..255
    // 64 alphas x 8 chunks of 8 k = 512 units, 2 per thread with the same
    // k-chunk (alphas al and al + 32), so the stage weights are read once
    int al_u[2], c_u[2];
    const __nv_bfloat16* rows_u[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      al_u[u] = (pt >> 3) + 32 * u;
      c_u[u] = pt & 7;
      const size_t a = (size_t)(a0 + al_u[u]);
      rows_u[u][0] = Xh + a * MX_BK;
      rows_u[u][1] = Xl + a * MX_BK;
      rows_u[u][2] = Xh + (P.Npad + a) * MX_BK;
      rows_u[u][3] = Xl + (P.Npad + a) * MX_BK;
    }
    uint4 pre[2][4];
    auto prefetch = [&](int i) {
      const int64_t kb = (int64_t)(kb0 + i) * P.rows * MX_BK;    // 64-k block
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          pre[u][q] = __ldg(reinterpret_cast<const uint4*>(rows_u[u][q] + kb + c_u[u] * 8));
    };
    if (nkb > 0) prefetch(0);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % MX_STAGES, r = i / MX_STAGES;
      // warp-uniform outcomes: a warp leaves the loop as a whole
      if (!__all_sync(0xffffffffu,
                      mbar_wait(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort, err, 4)))
        break;
      const int ws = i % MX_WSTAGES;
      if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&bar_w_full[ws]), (i / MX_WSTAGES) & 1,
                                             &s_abort, err, 8)))
        break;
      // W of both units in FP32 (hi + lo is exact in FP32)
      float wr[2][8], wi[2][8];
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t ah = (&pre[u][0].x)[q], al = (&pre[u][1].x)[q];
          const uint32_t bh = (&pre[u][2].x)[q], bl = (&pre[u][3].x)[q];
          wr[u][2 * q] = bf_lo(ah) + bf_lo(al);
          wr[u][2 * q + 1] = bf_hi(ah) + bf_hi(al);
          wi[u][2 * q] = bf_lo(bh) + bf_lo(bl);
          wi[u][2 * q + 1] = bf_hi(bh) + bf_hi(bl);
        }
      // the next k-block's rows load while this one's U is formed and stored
      if (i + 1 < nkb) prefetch(i + 1);
      const int c = c_u[0];
      // weights of k = 2q, 2q+1 of the chunk, both omegas loaded up front
      float4 wq[MX_OMEGA][4];
#pragma unroll
      for (int j = 0; j < MX_OMEGA; ++j) {
        // permuted block layout: pair q of chunk c is float4 number 8q + c
        const float4* wz = reinterpret_cast<const float4*>(w_s(ws, j)) + c;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          wq[j][q] = j < n_om ? wz[8 * q] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int j = 0; j < MX_OMEGA; ++j) {
        if (j >= n_om) break;
        const float4* w = wq[j];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int a_l = al_u[u];
          uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            // w conj(W) = (dr Wr + di Wi) + i (di Wr - dr Wi), roundings pinned
            // so both contraction kernels give the same bits
            const float ur0 = __fmaf_rn(w[q].x, wr[u][2 * q], __fmul_rn(w[q].y, wi[u][2 * q]));
            const float ui0 = __fmaf_rn(w[q].y, wr[u][2 * q], -__fmul_rn(w[q].x, wi[u][2 * q]));
            const float ur1 =
                __fmaf_rn(w[q].z, wr[u][2 * q + 1], __fmul_rn(w[q].w, wi[u][2 * q + 1]));
            const float ui1 =
                __fmaf_rn(w[q].w, wr[u][2 * q + 1], -__fmul_rn(w[q].z, wi[u][2 * q + 1]));
            rh[q] = pack_split(ur0, ur1, rl[q]);
            ih[q] = pack_split(ui0, ui1, il[q]);
          }
          const uint32_t offr = sw128_off(2 * a_l, c), offi = sw128_off(2 * a_l + 1, c);
          *reinterpret_cast<uint4*>(yh_s(s, j) + offr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
          *reinterpret_cast<uint4*>(yl_s(s, j) + offr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
          *reinterpret_cast<uint4*>(yh_s(s, j) + offi) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
          *reinterpret_cast<uint4*>(yl_s(s, j) + offi) = make_uint4(il[0], il[1], il[2], il[3]);
        }
      }
      // one arrival per warp (weights slot read, Y tiles written): 256
      // same-address arrivals per stage would serialise on the shared port
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(smem_u32(&bar_w_empty[ws]));
        mbar_arrive(smem_u32(&bar_full_y[s]));
      }
    }
  } else if (warp >= MX_DRAIN0) {
    // ---------------- drain: TMEM chunk -> FP64 partial (row per thread)
    const int q = warp & 3;                   // TMEM lane quadrant of this warp
    const int row = m0 + q * 32 + lane;
    for (int ch = 0; ch < max(nch, 1); ++ch) {
      const int b = ch & 1;
      bool ok = nkb > 0;
      if (ok) ok = mbar_wait(smem_u32(&bar_acc_full[b]), (ch >> 1) & 1, &s_abort, err, 9);
      ok = __all_sync(0xffffffffu, ok);
      if (nkb > 0 && !ok) break;
      tc_fence_after();
      for (int j = 0; j < n_om; ++j) {
        // partial plane of (omega, split), stored column by column (element
        // (row, col) at col * R + row): a warp's 32 rows are 256 contiguous bytes
        double* out = part + ((size_t)(om0 + j) * P.splits + split) * R * R + row;
        for (int cc = 0; cc < MX_BN / 32; ++cc) {
          uint32_t v[32];
          if (nkb > 0) {
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) +
                                   (uint32_t)(b * MX_ACC_COLS + j * MX_BN + cc * 32);
            TMEM_LD32(taddr, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          } else {
#pragma unroll
            for (int t = 0; t < 32; ++t) v[t] = 0u;
          }
          double* o = out + (size_t)(2 * a0 + cc * 32) * R;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            double old[16];
            if (ch > 0) {
#pragma unroll
              for (int t = 0; t < 16; ++t) old[t] = o[(size_t)(16 * h + t) * R];
            } else {
#pragma unroll
              for (int t = 0; t < 16; ++t) old[t] = 0.0;
            }
#pragma unroll
            for (int t = 0; t < 16; ++t)
              o[(size_t)(16 * h + t) * R] = old[t] + (double)__uint_as_float(v[16 * h + t]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (nkb > 0 && lane == 0) mbar_arrive(smem_u32(&bar_acc_empty[b]));
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  // every role has finished; all MMAs complete before TMEM is released
  // (bounded, ignores abort; the wait starts only now, so its bound does not
  // depend on how long the CTA worked)
  if (warp == 2 && nkb > 0) {
    mbar_wait(smem_u32(&bar_done), 0, nullptr, err, 5);
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(MX_TMEM_COLS));
  }
}

// ---- CTA-pair form (tcgen05 cta_group::2) ------------------------------------
// Two CTAs of a cluster compute a 256-row x 2-omega tile with M = 256,
// N = 128 x omegas MMAs issued by the even CTA ("leader"):
//   A (X rows): CTA c holds rows m0_c = (2 tp + c) 128 .. +127 (its own TMA);
//   B (Y rows): CTA c produces the Y rows of alphas a0 + 32c .. +31 for both
//               omegas (row omega 64 + 2 alpha + part), so each SM forms half
//               as much of Y per output as the one-CTA kernel;
//   D: CTA c's TMEM holds its 128 rows; column j < N/2 comes from the
//      leader's Y tile, j >= N/2 from the peer's.
// The peer's TMA completes on the leader's full barrier (cta_group::2 form),
// its producer and drain warps arrive on the leader's barriers through
// shared::cluster addresses, and the leader's commits multicast to both CTAs.
// A final cluster barrier keeps both CTAs resident until the last remote
// access.  When 2 Npad is not a multiple of 256 the last pair's odd CTA has
// no X rows: it loads nothing, still produces its half of Y, and its drain
// writes nothing.  Same k-blocks, chunks, flush order and U arithmetic as
// mixed_contract_kernel.
constexpr int MP_STAGES = 3;
constexpr int MP_AH = MX_AB / 2;                               // alphas per CTA
constexpr int MP_TILE_Y = MX_OMEGA * 2 * MP_AH * MX_BK * 2;    // 16 KB per part
constexpr int MP_STAGE_BYTES = 2 * MX_TILE_X + 2 * MP_TILE_Y;  // 64 KB
constexpr size_t MP_SMEM = (size_t)MP_STAGES * MP_STAGE_BYTES + MX_WRING_BYTES + 1024;

struct PairParams {
  int Npad, rows;
  int64_t K_pad;
  int nkb_total, kb_per_split, splits, n_omega, tiles_a;
};

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(MX_THREADS, 1)
mixed_pair_kernel(const __grid_constant__ CUtensorMap tm_h, const __grid_constant__ CUtensorMap tm_l,
                  PairParams P, const __nv_bfloat16* __restrict__ Xh,
                  const __nv_bfloat16* __restrict__ Xl, const float2* __restrict__ wt32,
                  double* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full_x[MP_STAGES], bar_full_y[MP_STAGES],
      bar_empty[MP_STAGES], bar_w_full[MX_WSTAGES], bar_w_empty[MX_WSTAGES], bar_acc_full[2],
      bar_acc_empty[2], bar_done;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t crank;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(crank));
  const bool leader = crank == 0;
  const int pair_tile = blockIdx.x >> 1;
  const int tp = pair_tile / P.tiles_a, ta = pair_tile % P.tiles_a;
  const int R = P.rows;
  const int m0 = (2 * tp + (int)crank) * MX_BM;       // this CTA's first X row
  const bool has_rows = m0 < R;
  const bool peer_rows = (2 * tp + 1) * MX_BM < R;      // the odd CTA of the pair has rows
  const int a0 = ta * MX_AB;
  const int ah0 = a0 + MP_AH * (int)crank;               // this CTA's alphas
  const int split = blockIdx.y, grp = blockIdx.z;
  const int om0 = grp * MX_OMEGA;
  const int n_om = min(MX_OMEGA, P.n_omega - om0);
  const int kb0 = split * P.kb_per_split;
  const int nkb = max(0, min(P.nkb_total, kb0 + P.kb_per_split) - kb0);
  const int nch = (nkb + MX_CHUNK_KB - 1) / MX_CHUNK_KB;
  const int NB = MX_BN * n_om;                            // MMA N
  const int half = NB / 2;                                // columns per CTA

  auto xh_s = [&](int s) { return smem + (size_t)s * MP_STAGE_BYTES; };
  auto xl_s = [&](int s) { return smem + (size_t)s * MP_STAGE_BYTES + MX_TILE_X; };
  auto yh_s = [&](int s) { return smem + (size_t)s * MP_STAGE_BYTES + 2 * MX_TILE_X; };
  auto yl_s = [&](int s) {
    return smem + (size_t)s * MP_STAGE_BYTES + 2 * MX_TILE_X + MP_TILE_Y;
  };
  auto w_s = [&](int ws, int j) {
    return reinterpret_cast<float2*>(smem + (size_t)MP_STAGES * MP_STAGE_BYTES +
                                     (size_t)ws * MX_OMEGA * MX_W_BYTES) + j * MX_BK;
  };

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < MP_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full_x[s]), 1);
      mbar_init(smem_u32(&bar_full_y[s]), 2 * (MX_PRODUCERS / 32));
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int s = 0; s < MX_WSTAGES; ++s) {
      mbar_init(smem_u32(&bar_w_full[s]), 1);
      mbar_init(smem_u32(&bar_w_empty[s]), MX_PRODUCERS / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_acc_full[b]), 1);
      mbar_init(smem_u32(&bar_acc_empty[b]), 2 * 4);
    }
    mbar_init(smem_u32(&bar_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2 && nkb > 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(MX_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();            // both CTAs' barriers initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    // ---------------- TMA: this CTA's X tile, completing on the leader's barrier
    if (lane == 0 && nkb > 0) {
      for (int i = 0; i < nkb; ++i) {
        const int s = i % MP_STAGES, r = i / MP_STAGES;
        if (!mbar_wait_cl(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort, err, 1)) break;
        const uint32_t fb = mapa_u32(smem_u32(&bar_full_x[s]), 0);
        if (leader) mbar_arrive_tx(smem_u32(&bar_full_x[s]), (peer_rows ? 2 : 1) * 2 * MX_TILE_X);
        if (has_rows) {
          tma_load_3d_pair(smem_u32(xh_s(s)), &tm_h, 0, m0, kb0 + i, fb);
          tma_load_3d_pair(smem_u32(xl_s(s)), &tm_l, 0, m0, kb0 + i, fb);
        }
      }
    }
  } else if (warp == 3) {
    // ---------------- weights ring (this CTA's producers)
    if (lane == 0 && nkb > 0) {
      int issued = 0;
      for (int i = 0; i < nkb; ++i) {
        const int ws = i % MX_WSTAGES, r = i / MX_WSTAGES;
        if (!mbar_wait(smem_u32(&bar_w_empty[ws]), (r & 1) ^ 1, &s_abort, err, 10)) break;
        const int64_t kx = (int64_t)(kb0 + i) * MX_BK;
        const uint32_t wb = smem_u32(&bar_w_full[ws]);
        mbar_arrive_tx(wb, n_om * MX_W_BYTES);
        for (int j = 0; j < n_om; ++j)
          bulk_load(smem_u32(w_s(ws, j)), wt32 + (size_t)(om0 + j) * P.K_pad + kx, MX_W_BYTES, wb);
        issued = i + 1;
      }
      for (int i = max(0, issued - MX_WSTAGES); i < issued; ++i)
        mbar_wait(smem_u32(&bar_w_full[i % MX_WSTAGES]), (i / MX_WSTAGES) & 1, nullptr, err, 6);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader only)
    if (leader && lane == 0 && nkb > 0) {
      const uint32_t idesc = idesc_bf16(2 * MX_BM, NB);
      for (int i = 0; i < nkb; ++i) {
        const int s = i % MP_STAGES, r = i / MP_STAGES;
        const int ch = i / MX_CHUNK_KB, b = ch & 1;
        const bool first = (i % MX_CHUNK_KB) == 0;
        const bool last = (i % MX_CHUNK_KB) == MX_CHUNK_KB - 1 || i == nkb - 1;
        if (first &&
            !mbar_wait_cl(smem_u32(&bar_acc_empty[b]), ((ch >> 1) & 1) ^ 1, &s_abort, err, 7))
          break;
        if (!mbar_wait_cl(smem_u32(&bar_full_x[s]), r & 1, &s_abort, err, 2)) break;
        if (!mbar_wait_cl(smem_u32(&bar_full_y[s]), r & 1, &s_abort, err, 3)) break;
        tc_fence_after();
        const uint64_t dxh = sw128_desc(smem_u32(xh_s(s)));
        const uint64_t dxl = sw128_desc(smem_u32(xl_s(s)));
        const uint64_t dyh = sw128_desc(smem_u32(yh_s(s)));
        const uint64_t dyl = sw128_desc(smem_u32(yl_s(s)));
        const uint32_t d = tmem + (uint32_t)(b * MX_ACC_COLS);
#pragma unroll
        for (int kk = 0; kk < MX_BK / 16; ++kk) {
          const uint64_t koff = (uint64_t)(kk * 32) >> 4;
          umma_pair(d, dxh + koff, dyh + koff, idesc, (first && kk == 0) ? 0u : 1u);
          umma_pair(d, dxh + koff, dyl + koff, idesc, 1u);
          umma_pair(d, dxl + koff, dyh + koff, idesc, 1u);
        }
        umma_pair_commit(smem_u32(&bar_empty[s]));
        if (last) umma_pair_commit(smem_u32(&bar_acc_full[b]));
      }
      umma_pair_commit(smem_u32(&bar_done));
    }
  } else if (warp >= 4 && warp < MX_DRAIN0) {
    // ---------------- producers: this CTA's 32 alphas x 8 k-chunks, both omegas
    const int pt = tid - 128;
    const int al = pt >> 3, c = pt & 7;
    const size_t a = (size_t)(ah0 + al);
    const __nv_bfloat16* rows_u[4] = {Xh + a * MX_BK, Xl + a * MX_BK,
                                      Xh + (P.Npad + a) * MX_BK, Xl + (P.Npad + a) * MX_BK};
    uint4 pre[4];
    auto prefetch = [&](int i) {
      const int64_t kb = (int64_t)(kb0 + i) * R * MX_BK;         // 64-k block
#pragma unroll
      for (int q = 0; q < 4; ++q)
        pre[q] = __ldg(reinterpret_cast<const uint4*>(rows_u[q] + kb + c * 8));
    };
    const uint32_t offr = sw128_off(2 * al, c), offi = sw128_off(2 * al + 1, c);
    if (nkb > 0) prefetch(0);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % MP_STAGES, r = i / MP_STAGES;
      if (!__all_sync(0xffffffffu, mbar_wait_cl(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort,
                                                err, 4)))
        break;
      const int ws = i % MX_WSTAGES;
      if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&bar_w_full[ws]), (i / MX_WSTAGES) & 1,
                                             &s_abort, err, 8)))
        break;
      float wr[8], wi[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t ah = (&pre[0].x)[q], all = (&pre[1].x)[q];
        const uint32_t bh = (&pre[2].x)[q], bl = (&pre[3].x)[q];
        wr[2 * q] = bf_lo(ah) + bf_lo(all);
        wr[2 * q + 1] = bf_hi(ah) + bf_hi(all);
        wi[2 * q] = bf_lo(bh) + bf_lo(bl);
        wi[2 * q + 1] = bf_hi(bh) + bf_hi(bl);
      }
#pragma unroll
      for (int j = 0; j < MX_OMEGA; ++j) {
        if (j >= n_om) break;
        const float4* wz = reinterpret_cast<const float4*>(w_s(ws, j)) + c;
        float4 w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = wz[8 * q];
        uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float ur0 = __fmaf_rn(w[q].x, wr[2 * q], __fmul_rn(w[q].y, wi[2 * q]));
          const float ui0 = __fmaf_rn(w[q].y, wr[2 * q], -__fmul_rn(w[q].x, wi[2 * q]));
          const float ur1 = __fmaf_rn(w[q].z, wr[2 * q + 1], __fmul_rn(w[q].w, wi[2 * q + 1]));
          const float ui1 = __fmaf_rn(w[q].w, wr[2 * q + 1], -__fmul_rn(w[q].z, wi[2 * q + 1]));
          rh[q] = pack_split(ur0, ur1, rl[q]);
          ih[q] = pack_split(ui0, ui1, il[q]);
        }
        // rows omega 64 + 2 alpha + part: omega j's block starts 8 swizzle atoms on
        const uint32_t ob = (uint32_t)j * 8 * 1024;
        *reinterpret_cast<uint4*>(yh_s(s) + ob + offr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(yl_s(s) + ob + offr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4*>(yh_s(s) + ob + offi) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4*>(yl_s(s) + ob + offi) = make_uint4(il[0], il[1], il[2], il[3]);
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(smem_u32(&bar_w_empty[ws]));
        if (leader) mbar_arrive(smem_u32(&bar_full_y[s]));
        else mbar_arrive_remote(mapa_u32(smem_u32(&bar_full_y[s]), 0));
      }
      if (i + 1 < nkb) prefetch(i + 1);
    }
  } else if (warp >= MX_DRAIN0) {
    // ---------------- drain: this CTA's 128 rows x N columns -> FP64 partial
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
    const bool row_ok = row < R;
    const size_t RR = (size_t)R;
    for (int ch = 0; ch < max(nch, 1); ++ch) {
      const int b = ch & 1;
      bool ok = nkb > 0;
      if (ok) ok = mbar_wait_cl(smem_u32(&bar_acc_full[b]), (ch >> 1) & 1, &s_abort, err, 9);
      ok = __all_sync(0xffffffffu, ok);
      if (nkb > 0 && !ok) break;
      tc_fence_after();
      for (int cc = 0; cc < NB / 32; ++cc) {
        const int col0 = cc * 32;
        const int h = col0 / half, n = col0 % half;
        const int om = n / 64;
        const int dcol = 2 * a0 + 64 * h + (n % 64);     // output column of TMEM column col0
        uint32_t v[32];
        if (nkb > 0) {
          const uint32_t taddr =
              tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * MX_ACC_COLS + col0);
          TMEM_LD32(taddr, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
          for (int t = 0; t < 32; ++t) v[t] = 0u;
        }
        if (!row_ok) continue;
        double* o = part + ((size_t)(om0 + om) * P.splits + split) * RR * RR + row +
                    (size_t)dcol * RR;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          double old[16];
          if (ch > 0) {
#pragma unroll
            for (int t = 0; t < 16; ++t) old[t] = o[(size_t)(16 * hh + t) * RR];
          } else {
#pragma unroll
            for (int t = 0; t < 16; ++t) old[t] = 0.0;
          }
#pragma unroll
          for (int t = 0; t < 16; ++t)
            o[(size_t)(16 * hh + t) * RR] = old[t] + (double)__uint_as_float(v[16 * hh + t]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (nkb > 0 && lane == 0) {
        if (leader) mbar_arrive(smem_u32(&bar_acc_empty[b]));
        else mbar_arrive_remote(mapa_u32(smem_u32(&bar_acc_empty[b]), 0));
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  // every role has finished; every MMA of the pair completes (bounded from
  // now, ignores abort) before the cluster barrier that both CTAs leave by
  if (warp == 2 && nkb > 0) mbar_wait_cl(smem_u32(&bar_done), 0, nullptr, err, 5);
  cluster_sync_all();            // no CTA leaves while its peer may still touch it
  if (warp == 2 && nkb > 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(MX_TMEM_COLS));
  }
}

// ---- reduction of the FP64 partial tiles -----------------------------------------
__device__ __forceinline__ void mixed_reduce_body(int Na, int Npad, int splits, double G,
                                                  const double* __restrict__ Nk,
                                                  const double* __restrict__ part,
                                                  double2* __restrict__ A,
                                                  double2* __restrict__ Mout,
                                                  const double2* __restrict__ Ma) {
  const size_t R = 2 * (size_t)Npad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Na * Na; e += gridDim.x * blockDim.x) {
    const int b = e % Na, a = e / Na;          // consecutive threads: consecutive rows b
    double mr = 0.0, mi = 0.0;
    for (int s = 0; s < splits; ++s) {
      // plane of (omega, split), element (row c, column n) at n * R + c
      const double* P = part + (size_t)s * R * R;
      const double pr_r = P[(size_t)(2 * a) * R + b], pr_i = P[(size_t)(2 * a + 1) * R + b];
      const double pi_r = P[(size_t)(2 * a) * R + Npad + b];
      const double pi_i = P[(size_t)(2 * a + 1) * R + Npad + b];
      mr += pr_r - pi_i;
      mi += pr_i + pi_r;
    }
    const double n = Nk[a];
    // unfused products: 1 - Mr must not become an FMA in one kernel only
    double Mr = __dmul_rn(__dmul_rn(mr, G), n), Mi = __dmul_rn(__dmul_rn(mi, G), n);
    if (Ma) {                                  // anchored: M(omega_a) + delta M
      const double2 v = Ma[(size_t)b * Na + a];
      Mr = __dadd_rn(v.x, Mr);
      Mi = __dadd_rn(v.y, Mi);
    }
    A[(size_t)b * Na + a] = make_double2((a == b ? 1.0 : 0.0) - Mr, -Mi);
    if (Mout) Mout[(size_t)b * Na + a] = make_double2(Mr, Mi);
  }
}

__global__ void mixed_reduce_kernel(int Na, int Npad, int splits, double G,
                                    const double* __restrict__ Nk, const double* __restrict__ part,
                                    double2* __restrict__ A, double2* __restrict__ Mout,
                                    const double2* __restrict__ Ma) {
  const int z = blockIdx.y;
  const size_t R = 2 * (size_t)Npad;
  mixed_reduce_body(Na, Npad, splits, G, Nk, part + (size_t)z * splits * R * R,
                    A + (size_t)z * Na * Na, z == 0 ? Mout : nullptr, Ma);
}

// ---- uneven batch over models -------------------------------------------------
__global__ void multi_weights32_kernel(const kls_mdesc* __restrict__ md,
                                       const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  const double2* wt = d.wt + (size_t)pz.y * d.K_pad;
  float2* w32 = reinterpret_cast<float2*>(d.wt32) + (size_t)pz.y * d.K_pad;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.K_pad;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = wt[i];
    const int k = (int)(i & (MX_BK - 1));
    const int c = k >> 3, q = (k >> 1) & 3, h = k & 1;
    w32[(i & ~(int64_t)(MX_BK - 1)) + 2 * (8 * q + c) + h] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void multi_mixed_reduce_kernel(const kls_mdesc* __restrict__ md,
                                          const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  const size_t R = 2 * (size_t)d.Na_pad;
  mixed_reduce_body(d.Na, d.Na_pad, d.msplits, d.G, d.Nk,
                    d.mpart + (size_t)pz.y * d.msplits * R * R, d.A + (size_t)pz.y * d.Na * d.Na,
                    nullptr, nullptr);
}


// Persistent form of mixed_contract_kernel over an uneven batch of models.
// CTA b takes items [starts[b], starts[b+1]) of a list the host ordered
// (round robin over a model-major list, so CTAs running at the same time
// share a k-range of one table); every role walks the same items, and the stage, weights-slot and
// accumulator phases run on counters that continue across items, so the
// pipeline never drains between items.  An item computes exactly what the
// one-model kernel computes for the same (tile, split, omegas): the same
// k-blocks, chunks and FP64 flush order, hence the same bits.
__global__ void __launch_bounds__(MX_THREADS, 1)
mixed_multi_kernel(const kls_mdesc* __restrict__ md, const kls_item* __restrict__ items,
                   const int* __restrict__ starts, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full_x[MX_STAGES], bar_full_y[MX_STAGES],
      bar_empty[MX_STAGES], bar_w_full[MX_WSTAGES], bar_w_empty[MX_WSTAGES], bar_acc_full[2],
      bar_acc_empty[2], bar_done;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t_beg = starts[blockIdx.x], t_end = starts[blockIdx.x + 1];
  const bool any = t_end > t_beg;

  auto xh_s = [&](int s) { return smem + (size_t)s * MX_STAGE_BYTES; };
  auto xl_s = [&](int s) { return smem + (size_t)s * MX_STAGE_BYTES + MX_TILE_X; };
  auto yh_s = [&](int s, int j) {
    return smem + (size_t)s * MX_STAGE_BYTES + 2 * MX_TILE_X + (size_t)j * MX_TILE_Y;
  };
  auto yl_s = [&](int s, int j) {
    return smem + (size_t)s * MX_STAGE_BYTES + 2 * MX_TILE_X + (size_t)(MX_OMEGA + j) * MX_TILE_Y;
  };
  auto w_s = [&](int ws, int j) {
    return reinterpret_cast<float2*>(smem + (size_t)MX_STAGES * MX_STAGE_BYTES +
                                     (size_t)ws * MX_OMEGA * MX_W_BYTES) + j * MX_BK;
  };

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < MX_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full_x[s]), 1);
      mbar_init(smem_u32(&bar_full_y[s]), MX_PRODUCERS / 32);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int s = 0; s < MX_WSTAGES; ++s) {
      mbar_init(smem_u32(&bar_w_full[s]), 1);
      mbar_init(smem_u32(&bar_w_empty[s]), MX_PRODUCERS / 32);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_acc_full[b]), 1);
      mbar_init(smem_u32(&bar_acc_empty[b]), 4);
    }
    mbar_init(smem_u32(&bar_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2 && any) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(MX_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    // ---------------- TMA: X tiles
    if (lane == 0 && any) {
      uint32_t g = 0;
      bool ok = true;
      for (int t = t_beg; t < t_end && ok; ++t) {
        const kls_item it = items[t];
        const kls_mdesc& d = md[it.model];
        const CUtensorMap* mh = reinterpret_cast<const CUtensorMap*>(d.tmap_h);
        const CUtensorMap* ml = reinterpret_cast<const CUtensorMap*>(d.tmap_l);
        tensormap_acquire(mh);
        tensormap_acquire(ml);
        const int m0 = (it.tile / (d.Na_pad / MX_AB)) * MX_BM;
        for (int i = 0; i < it.nkb; ++i) {
          const int s = g % MX_STAGES, r = g / MX_STAGES;
          if (!mbar_wait(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort, err, 1)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&bar_full_x[s]);
          mbar_arrive_tx(fb, 2 * MX_TILE_X);
          tma_load_3d(smem_u32(xh_s(s)), mh, 0, m0, it.kb0 + i, fb);
          tma_load_3d(smem_u32(xl_s(s)), ml, 0, m0, it.kb0 + i, fb);
          ++g;
        }
      }
      for (uint32_t i = g > MX_STAGES ? g - MX_STAGES : 0; i < g; ++i)
        mbar_wait(smem_u32(&bar_full_x[i % MX_STAGES]), (i / MX_STAGES) & 1, nullptr, err, 6);
    }
  } else if (warp == 3) {
    // ---------------- weights ring
    if (lane == 0 && any) {
      uint32_t g = 0;
      bool ok = true;
      for (int t = t_beg; t < t_end && ok; ++t) {
        const kls_item it = items[t];
        const kls_mdesc& d = md[it.model];
        const float2* wt32 = reinterpret_cast<const float2*>(d.wt32);
        for (int i = 0; i < it.nkb; ++i) {
          const int ws = g % MX_WSTAGES, r = g / MX_WSTAGES;
          if (!mbar_wait(smem_u32(&bar_w_empty[ws]), (r & 1) ^ 1, &s_abort, err, 10)) {
            ok = false;
            break;
          }
          const int64_t kx = (int64_t)(it.kb0 + i) * MX_BK;
          const uint32_t wb = smem_u32(&bar_w_full[ws]);
          mbar_arrive_tx(wb, it.n_om * MX_W_BYTES);
          for (int j = 0; j < it.n_om; ++j)
            bulk_load(smem_u32(w_s(ws, j)), wt32 + (size_t)(it.z + j) * d.K_pad + kx, MX_W_BYTES,
                      wb);
          ++g;
        }
      }
      for (uint32_t i = g > MX_WSTAGES ? g - MX_WSTAGES : 0; i < g; ++i)
        mbar_wait(smem_u32(&bar_w_full[i % MX_WSTAGES]), (i / MX_WSTAGES) & 1, nullptr, err, 6);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0 && any) {
      uint32_t g = 0, gch = 0;
      bool ok = true;
      for (int t = t_beg; t < t_end && ok; ++t) {
        const kls_item it = items[t];
        const uint32_t idesc = idesc_bf16(MX_BM, MX_BN * it.n_om);
        for (int i = 0; i < it.nkb; ++i) {
          const int s = g % MX_STAGES, r = g / MX_STAGES;
          const uint32_t ch = gch + (uint32_t)(i / MX_CHUNK_KB), b = ch & 1;
          const bool first = (i % MX_CHUNK_KB) == 0;
          const bool last = (i % MX_CHUNK_KB) == MX_CHUNK_KB - 1 || i == it.nkb - 1;
          if (first &&
              !mbar_wait(smem_u32(&bar_acc_empty[b]), ((ch >> 1) & 1) ^ 1, &s_abort, err, 7)) {
            ok = false;
            break;
          }
          if (!mbar_wait(smem_u32(&bar_full_x[s]), r & 1, &s_abort, err, 2) ||
              !mbar_wait(smem_u32(&bar_full_y[s]), r & 1, &s_abort, err, 3)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t dxh = sw128_desc(smem_u32(xh_s(s)));
          const uint64_t dxl = sw128_desc(smem_u32(xl_s(s)));
          const uint32_t d = tmem + (uint32_t)(b * MX_ACC_COLS);
          const uint64_t dyh0 = sw128_desc(smem_u32(yh_s(s, 0)));
          const uint64_t dyl0 = sw128_desc(smem_u32(yl_s(s, 0)));
#pragma unroll
          for (int kk = 0; kk < MX_BK / 16; ++kk) {
            const uint64_t koff = (uint64_t)(kk * 32) >> 4;
            umma(d, dxh + koff, dyh0 + koff, idesc, (first && kk == 0) ? 0u : 1u);
            umma(d, dxh + koff, dyl0 + koff, idesc, 1u);
            umma(d, dxl + koff, dyh0 + koff, idesc, 1u);
          }
          umma_commit(smem_u32(&bar_empty[s]));
          if (last) umma_commit(smem_u32(&bar_acc_full[b]));
          ++g;
        }
        gch += (uint32_t)((it.nkb + MX_CHUNK_KB - 1) / MX_CHUNK_KB);
      }
      umma_commit(smem_u32(&bar_done));
    }
  } else if (warp >= 4 && warp < MX_DRAIN0) {
    // ---------------- producers
    const int pt = tid - 128;
    const int c = pt & 7;
    uint32_t g = 0;
    bool ok = true;
    for (int t = t_beg; t < t_end && ok; ++t) {
      const kls_item it = items[t];
      const kls_mdesc& d = md[it.model];
      const __nv_bfloat16* Xh = reinterpret_cast<const __nv_bfloat16*>(d.Xh);
      const __nv_bfloat16* Xl = reinterpret_cast<const __nv_bfloat16*>(d.Xl);
      const int a0 = (it.tile % (d.Na_pad / MX_AB)) * MX_AB;
      const int n_om = it.n_om;
      int al_u[2];
      const __nv_bfloat16* rows_u[2][4];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        al_u[u] = (pt >> 3) + 32 * u;
        const size_t a = (size_t)(a0 + al_u[u]);
        rows_u[u][0] = Xh + a * MX_BK;
        rows_u[u][1] = Xl + a * MX_BK;
        rows_u[u][2] = Xh + (d.Na_pad + a) * MX_BK;
        rows_u[u][3] = Xl + (d.Na_pad + a) * MX_BK;
      }
      uint4 pre[2][4];
      auto prefetch = [&](int i) {
        const int64_t kb = (int64_t)(it.kb0 + i) * 2 * d.Na_pad * MX_BK;   // 64-k block
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int q = 0; q < 4; ++q)
            pre[u][q] = __ldg(reinterpret_cast<const uint4*>(rows_u[u][q] + kb + c * 8));
      };
      prefetch(0);
      for (int i = 0; i < it.nkb; ++i) {
        const int s = g % MX_STAGES, r = g / MX_STAGES;
        if (!__all_sync(0xffffffffu,
                        mbar_wait(smem_u32(&bar_empty[s]), (r & 1) ^ 1, &s_abort, err, 4))) {
          ok = false;
          break;
        }
        const int ws = g % MX_WSTAGES;
        if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&bar_w_full[ws]), (g / MX_WSTAGES) & 1,
                                               &s_abort, err, 8))) {
          ok = false;
          break;
        }
        float wr[2][8], wi[2][8];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t ah = (&pre[u][0].x)[q], al = (&pre[u][1].x)[q];
            const uint32_t bh = (&pre[u][2].x)[q], bl = (&pre[u][3].x)[q];
            wr[u][2 * q] = bf_lo(ah) + bf_lo(al);
            wr[u][2 * q + 1] = bf_hi(ah) + bf_hi(al);
            wi[u][2 * q] = bf_lo(bh) + bf_lo(bl);
            wi[u][2 * q + 1] = bf_hi(bh) + bf_hi(bl);
          }
        float4 wq[MX_OMEGA][4];
#pragma unroll
        for (int j = 0; j < MX_OMEGA; ++j) {
          const float4* wz = reinterpret_cast<const float4*>(w_s(ws, j)) + c;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            wq[j][q] = j < n_om ? wz[8 * q] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < MX_OMEGA; ++j) {
          if (j >= n_om) break;
          const float4* w = wq[j];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int a_l = al_u[u];
            uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float ur0 = __fmaf_rn(w[q].x, wr[u][2 * q], __fmul_rn(w[q].y, wi[u][2 * q]));
              const float ui0 = __fmaf_rn(w[q].y, wr[u][2 * q], -__fmul_rn(w[q].x, wi[u][2 * q]));
              const float ur1 =
                  __fmaf_rn(w[q].z, wr[u][2 * q + 1], __fmul_rn(w[q].w, wi[u][2 * q + 1]));
              const float ui1 =
                  __fmaf_rn(w[q].w, wr[u][2 * q + 1], -__fmul_rn(w[q].z, wi[u][2 * q + 1]));
              rh[q] = pack_split(ur0, ur1, rl[q]);
              ih[q] = pack_split(ui0, ui1, il[q]);
            }
            const uint32_t offr = sw128_off(2 * a_l, c), offi = sw128_off(2 * a_l + 1, c);
            *reinterpret_cast<uint4*>(yh_s(s, j) + offr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
            *reinterpret_cast<uint4*>(yl_s(s, j) + offr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
            *reinterpret_cast<uint4*>(yh_s(s, j) + offi) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
            *reinterpret_cast<uint4*>(yl_s(s, j) + offi) = make_uint4(il[0], il[1], il[2], il[3]);
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(smem_u32(&bar_w_empty[ws]));
          mbar_arrive(smem_u32(&bar_full_y[s]));
        }
        ++g;
        if (i + 1 < it.nkb) prefetch(i + 1);
      }
    }
  } else if (warp >= MX_DRAIN0) {
    // ---------------- drain
    const int q = warp & 3;
    uint32_t gch = 0;
    bool ok = true;
    for (int t = t_beg; t < t_end && ok; ++t) {
      const kls_item it = items[t];
      const kls_mdesc& d = md[it.model];
      const size_t R = 2 * (size_t)d.Na_pad;
      const int tiles_a = d.Na_pad / MX_AB;
      const int row = (it.tile / tiles_a) * MX_BM + q * 32 + lane;
      const int a0 = (it.tile % tiles_a) * MX_AB;
      const int nch = (it.nkb + MX_CHUNK_KB - 1) / MX_CHUNK_KB;
      for (int ch = 0; ch < nch; ++ch) {
        const uint32_t G = gch + (uint32_t)ch, b = G & 1;
        bool w = mbar_wait(smem_u32(&bar_acc_full[b]), (G >> 1) & 1, &s_abort, err, 9);
        w = __all_sync(0xffffffffu, w);
        if (!w) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int j = 0; j < it.n_om; ++j) {
          double* out = d.mpart + ((size_t)(it.z + j) * d.msplits + it.split) * R * R + row;
          for (int cc = 0; cc < MX_BN / 32; ++cc) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) +
                                   (uint32_t)(b * MX_ACC_COLS + j * MX_BN + cc * 32);
            TMEM_LD32(taddr, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            double* o = out + (size_t)(2 * a0 + cc * 32) * R;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              double old[16];
              if (ch > 0) {
#pragma unroll
                for (int t2 = 0; t2 < 16; ++t2) old[t2] = o[(size_t)(16 * h + t2) * R];
              } else {
#pragma unroll
                for (int t2 = 0; t2 < 16; ++t2) old[t2] = 0.0;
              }
#pragma unroll
              for (int t2 = 0; t2 < 16; ++t2)
                o[(size_t)(16 * h + t2) * R] = old[t2] + (double)__uint_as_float(v[16 * h + t2]);
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&bar_acc_empty[b]));
      }
      gch += (uint32_t)nch;
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  // the wait for the last commit starts after every role has finished: a
  // persistent CTA may work for longer than any single wait's bound
  if (warp == 2 && any) {
    mbar_wait(smem_u32(&bar_done), 0, nullptr, err, 5);
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(MX_TMEM_COLS));
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct kls_mixed {
  __nv_bfloat16* Xh = nullptr;
  __nv_bfloat16* Xl = nullptr;
  CUtensorMap tm_h, tm_l;
  double* part = nullptr;       // FP64 partials [n][splits][2 Npad][2 Npad]
  size_t part_elems = 0;
  float2* wt32 = nullptr;       // FP32 weights [n][K_pad]
  size_t wt32_elems = 0;
  int* err = nullptr;
  int splits = 1;
  int form = KLS_MIXED_ONE_CTA;   // contraction kernel (KLS_MIXED_*)
  kls_mixed_tm* tm = nullptr;     // TMEM-operand form (N_alpha_pad <= 384)
  unsigned long long wait_ns = 2000000000ull;   // its wait bound
  int fault_mode = 0;             // test hook of the failure path (one-shot)
};

static int mixed_splits(const kls_ctx* c) {
  const int tiles = (2 * c->Na_pad / MX_BM) * (c->Na_pad / MX_AB);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  int q = std::max(1, (16 * tiles + sms - 1) / sms);
  int s = (q * sms) / tiles;
  int nkb = (int)(c->K_pad / MX_BK);
  s = std::max(1, std::min(s, nkb));
  return s;
}

int kls_mixed_prepare(kls_ctx* c) {
  if (c->mixed) return KLS_OK;
  if (!c->precomputed) return kls_fail(c, KLS_ERR_STATE, "kls_precompute has not run");
  if ((2 * c->Na_pad) % MX_BM != 0 || c->Na_pad % MX_AB != 0 || c->K_pad % MX_BK != 0)
    return kls_fail(c, KLS_ERR_CONFIG, "table padding incompatible with the mixed tiles");
  kls_mixed* m = new kls_mixed();
  const size_t rows = 2 * (size_t)c->Na_pad;
  const size_t n = rows * (size_t)c->K_pad;
  cudaError_t e;
  if ((e = cudaMalloc(&m->Xh, n * sizeof(__nv_bfloat16))) != cudaSuccess ||
      (e = cudaMalloc(&m->Xl, n * sizeof(__nv_bfloat16))) != cudaSuccess ||
      (e = cudaMalloc(&m->err, sizeof(int))) != cudaSuccess) {
    cudaFree(m->Xh); cudaFree(m->Xl); cudaFree(m->err);
    delete m;
    return kls_cuda_fail(c, e, "cudaMalloc (split table)");
  }
  c->device_bytes += (int64_t)(2 * n * sizeof(__nv_bfloat16));
  c->mixed = m;
  KLS_CK(c, cudaMemsetAsync(m->err, 0, sizeof(int), c->stream));
  dim3 grid((unsigned)(c->K_pad / 32), c->Na_pad / 32);
  split_table_kernel<<<grid, dim3(32, 8), 0, c->stream>>>(c->d_Wre, c->d_Wim, c->Na_pad, c->K_pad,
                                                          m->Xh, m->Xl);
  KLS_LAUNCHED(c);
  // TMA descriptors over X{h,l}: box {64 k, 128 rows, 1 block}, 128B swizzle
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  KLS_CK(c, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess)
    return kls_fail(c, KLS_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn encode = (EncodeTiledFn)fn;
  // 3-D view of the blocked table: {64 k, rows, 64-k blocks}
  cuuint64_t dims[3] = {(cuuint64_t)MX_BK, (cuuint64_t)rows, (cuuint64_t)(c->K_pad / MX_BK)};
  cuuint64_t strides[2] = {(cuuint64_t)MX_BK * sizeof(__nv_bfloat16),
                           (cuuint64_t)rows * MX_BK * sizeof(__nv_bfloat16)};
  cuuint32_t box[3] = {MX_BK, MX_BM, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  for (int t = 0; t < 2; ++t) {
    CUresult r = encode(t == 0 ? &m->tm_h : &m->tm_l, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                        t == 0 ? (void*)m->Xh : (void*)m->Xl, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return kls_fail(c, KLS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  }
  m->splits = mixed_splits(c);
  if (kls_tm_supported(c)) {
    int r = kls_tm_create(c, m->Xh, m->Xl, &m->tm);
    if (r) return r;
    m->form = KLS_MIXED_TMEM;
  }
  KLS_CK(c, cudaFuncSetAttribute(mixed_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)MX_SMEM));
  KLS_CK(c, cudaFuncSetAttribute(mixed_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)MP_SMEM));
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  return KLS_OK;
}

int kls_mixed_contract(kls_ctx* c, int n, int) {
  kls_mixed* m = c->mixed;
  if (m->form == KLS_MIXED_TMEM) {
    const int fault = m->fault_mode;
    m->fault_mode = 0;
    return kls_tm_contract(c, m->tm, n, m->err, m->wait_ns, fault);
  }
  const size_t R = 2 * (size_t)c->Na_pad;
  const size_t need = (size_t)n * m->splits * R * R;
  if (need > m->part_elems) {
    cudaFree(m->part);
    m->part = nullptr;
    m->part_elems = 0;
    KLS_CK(c, cudaMalloc(&m->part, need * sizeof(double)));
    m->part_elems = need;
  }
  const size_t nw = (size_t)n * c->K_pad;
  if (nw > m->wt32_elems) {
    cudaFree(m->wt32);
    m->wt32 = nullptr;
    m->wt32_elems = 0;
    KLS_CK(c, cudaMalloc(&m->wt32, nw * sizeof(float2)));
    m->wt32_elems = nw;
  }
  weights32_kernel<<<(unsigned)std::min<size_t>((nw + 255) / 256, 4096), 256, 0, c->stream>>>(
      (int64_t)nw, c->d_wt, m->wt32);
  KLS_LAUNCHED(c);
  if (m->form == KLS_MIXED_PAIR) {
    PairParams Q{};
    Q.Npad = c->Na_pad;
    Q.rows = (int)R;
    Q.K_pad = c->K_pad;
    Q.nkb_total = (int)(c->K_pad / MX_BK);
    Q.splits = m->splits;
    Q.kb_per_split = (Q.nkb_total + m->splits - 1) / m->splits;
    Q.n_omega = n;
    Q.tiles_a = c->Na_pad / MX_AB;
    const int row_pairs = (int)((R + 2 * MX_BM - 1) / (2 * MX_BM));
    dim3 grid((unsigned)(2 * row_pairs * Q.tiles_a), m->splits, (n + MX_OMEGA - 1) / MX_OMEGA);
    mixed_pair_kernel<<<grid, MX_THREADS, MP_SMEM, c->stream>>>(m->tm_h, m->tm_l, Q, m->Xh, m->Xl,
                                                                m->wt32, m->part, m->err);
    KLS_LAUNCHED(c);
    return KLS_OK;
  }
  MixedParams P{};
  P.Npad = c->Na_pad;
  P.rows = (int)R;
  P.K_pad = c->K_pad;
  P.nkb_total = (int)(c->K_pad / MX_BK);
  P.splits = m->splits;
  P.kb_per_split = (P.nkb_total + m->splits - 1) / m->splits;
  P.n_omega = n;
  P.tiles_a = c->Na_pad / MX_AB;
  dim3 grid((unsigned)((R / MX_BM) * P.tiles_a), m->splits, (n + MX_OMEGA - 1) / MX_OMEGA);
  mixed_contract_kernel<<<grid, MX_THREADS, MX_SMEM, c->stream>>>(m->tm_h, m->tm_l, P, m->Xh,
                                                                  m->Xl, m->wt32, m->part, m->err);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_mixed_reduce(kls_ctx* c, int n, bool export_M, const double2* Ma) {
  kls_mixed* m = c->mixed;
  if (m->form == KLS_MIXED_TMEM) return kls_tm_reduce(c, m->tm, n, export_M, Ma);
  int blocks = std::min((c->Na * c->Na + 255) / 256, 1024);
  mixed_reduce_kernel<<<dim3(blocks, n), 256, 0, c->stream>>>(
      c->Na, c->Na_pad, m->splits, c->cfg.G, c->d_N, m->part, c->d_A, export_M ? c->d_M : nullptr,
      Ma);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

int kls_mixed_check(kls_ctx* c) {
  if (!c->mixed) return KLS_OK;
  int h = 0;
  KLS_CK(c, cudaMemcpy(&h, c->mixed->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(c->mixed->err, 0, sizeof(int));
    return kls_fail(c, KLS_ERR_TIMEOUT,
                    "mixed contraction pipeline: a bounded wait ran out (code " +
                        std::to_string(h) + "); results of this call are invalid");
  }
  return KLS_OK;
}

void kls_mixed_free(kls_ctx* c) {
  if (!c->mixed) return;
  cudaFree(c->mixed->Xh);
  cudaFree(c->mixed->Xl);
  cudaFree(c->mixed->part);
  cudaFree(c->mixed->wt32);
  cudaFree(c->mixed->err);
  kls_tm_destroy(c->mixed->tm);
  delete c->mixed;
  c->mixed = nullptr;
}

// ---- uneven batch hooks (kls_multi.cu) ----------------------------------------
int kls_multi_launch_mixed(cudaStream_t st, const kls_mdesc* d_md, const int2* d_pairs,
                           int n_pairs, const kls_item* d_items, const int* d_starts, int grid,
                           int64_t max_K_pad, int* d_err) {
  cudaError_t e;
  int wblocks = (int)std::min<int64_t>((max_K_pad + 255) / 256, 1024);
  multi_weights32_kernel<<<dim3(wblocks, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  if ((e = cudaFuncSetAttribute(mixed_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)MX_SMEM)) != cudaSuccess)
    return (int)e;
  mixed_multi_kernel<<<grid, MX_THREADS, MX_SMEM, st>>>(d_md, d_items, d_starts, d_err);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  multi_mixed_reduce_kernel<<<dim3(256, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  return (int)cudaGetLastError();
}

int kls_mixed_slots(int device) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaFuncSetAttribute(mixed_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)MX_SMEM);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_multi_kernel, MX_THREADS,
                                                    MX_SMEM) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

int kls_mixed_splits_of(const kls_ctx* c) {
  if (!c->mixed) return 0;
  return c->mixed->form == KLS_MIXED_TMEM ? kls_tm_splits(c->mixed->tm) : c->mixed->splits;
}

int kls_mixed_legacy_splits(const kls_ctx* c) { return c->mixed ? c->mixed->splits : 0; }

kls_mixed_tm* kls_mixed_tm_state(const kls_ctx* c, unsigned long long* wait_ns) {
  if (!c->mixed || c->mixed->form != KLS_MIXED_TMEM) return nullptr;
  if (wait_ns) *wait_ns = c->mixed->wait_ns;
  return c->mixed->tm;
}

int kls_mixed_default_splits(const kls_ctx* c) {
  if (c->mixed && c->mixed->form == KLS_MIXED_TMEM) return kls_tm_default_splits(c);
  return mixed_splits(c);
}

int kls_mixed_set_form(kls_ctx* c, int form) {
  if (!c->mixed) return KLS_ERR_STATE;
  if (form == KLS_MIXED_TMEM && !c->mixed->tm)
    return kls_fail(c, KLS_ERR_UNSUPPORTED, "KLS_MIXED_TMEM needs N_alpha_pad <= 384");
  c->mixed->form = form;
  return KLS_OK;
}

int kls_mixed_set_chunk(kls_ctx* c, int stages) {
  if (!c->mixed) return KLS_ERR_STATE;
  if (!c->mixed->tm) return kls_fail(c, KLS_ERR_UNSUPPORTED, "KLS_MIXED_TMEM needs N_alpha_pad <= 384");
  kls_tm_set_chunk(c->mixed->tm, stages);
  return KLS_OK;
}

int kls_mixed_set_wait(kls_ctx* c, unsigned long long ns, int fault_mode) {
  if (!c->mixed) return KLS_ERR_STATE;
  if (ns) c->mixed->wait_ns = ns;
  if (fault_mode >= 0) c->mixed->fault_mode = fault_mode;
  return KLS_OK;
}

int kls_mixed_form_of(const kls_ctx* c) { return c->mixed ? c->mixed->form : 0; }

int kls_mixed_set_splits(kls_ctx* c, int splits) {
  if (!c->mixed) return KLS_ERR_STATE;
  if (c->mixed->form == KLS_MIXED_TMEM) {
    kls_tm_set_splits(c, c->mixed->tm, splits);
    return KLS_OK;
  }
  const int nkb = (int)(c->K_pad / MX_BK);
  c->mixed->splits = std::max(1, std::min(splits, nkb));
  return KLS_OK;
}

const void* kls_mixed_tables(const kls_ctx* c, const void** Xl, const void** tmap_h,
                             const void** tmap_l) {
  if (!c->mixed) return nullptr;
  *Xl = c->mixed->Xl;
  *tmap_h = &c->mixed->tm_h;
  *tmap_l = &c->mixed->tm_l;
  return c->mixed->Xh;
}

// Split-BF16 contraction with the omega-dependent operand in tensor memory
// (KLS_MIXED_TMEM, the default form of KLS_MODE_MIXED for N_alpha_pad <= 384).
//
//   M(omega)[b, a] = sum_k W[k, b] U[k, a],   U = w(omega) conj(W)
//   M_r = sum_k ReW_b ReU_a - ImW_b ImU_a,    M_i = sum_k ReW_b ImU_a + ImW_b ReU_a
//
// A stage covers 32 complex k and 64 real contraction indices k': the first
// 32 pair Re W with the coefficient rows, the next 32 pair Im W.  With
//   B row b     = [ReW_b(k) | ImW_b(k)]            (omega-independent table)
//   A row (a,r) = [ReU_a(k) | -ImU_a(k)],  A row (a,i) = [ImU_a(k) | ReU_a(k)]
// one real GEMM D = A B^T gives M_r[b, a] = D[(a,r), b], M_i[b, a] = D[(a,i), b]
// with every A row formed exactly once per omega (the older forms re-form the
// omega-dependent operand once per 128-row output tile).
//
// CTA pair (cluster of 2, tcgen05 cta_group::2, MMA M = 256).  Each CTA owns
// one "tile": 64 alphas of one omega = 128 A rows.  Its producer warps form
// the A rows in FP32 from the table rows of its alphas (TMA-staged), split
// them error-free into BF16 hi + lo and store them straight into tensor
// memory (tcgen05.st); the MMA reads A from TMEM and B from shared memory.
// B is the whole table row range [0, Npad) for the stage: each CTA loads half
// of it (64-byte swizzled TMA tiles of the split table Xh / Xl, Re rows a and
// Im rows Npad + a), so each SM reads Npad / 2 table rows per stage.  The
// accumulator (128 lanes x Npad FP32 columns per CTA) holds every output row
// b and is flushed every `chunk` stages (default TM_CHUNK) into an FP64
// partial per (tile, K split) in deterministic order; the split sum, G N(a)
// scaling, I - M, the weights and the LU are FP64.  Products hi*hi + lo*hi + hi*lo (the lo*lo
// term, ~2^-18 relative, is dropped).
//
// Warps (640 threads):
//   0       TMA: both B half tiles (completing on the leader's barrier; a
//           ring of 4 stages, 3 at Npad = 384) and this CTA's A-source tiles
//           (its 64 alphas; a ring of 3 stages)
//   1       MMA issuer (leader CTA; the warp waits, one elected lane issues)
//   2       TMEM allocation / release (512 columns: D at [0, Npad), A stages
//           of 64 columns at the top: three for Npad <= 320, else two)
//   3       weights ring: bulk copies of the FP32 w(omega) of the CTA's omega,
//           two pre-signed coefficient pairs per two k
//   4..11   producers, 2 per TMEM lane quadrant (halves of the stage's k);
//           lane 2a holds row (a, r), lane 2a + 1 row (a, i); each lane forms
//           one component of U (packed f32x2 arithmetic) and takes the other
//           half of its row from its partner lane
//   12..19  drain, 2 per lane quadrant (halves of the D columns): TMEM ->
//           FP64 partial (stores for the first chunk, L2 reductions after)
// Every wait is bounded (the context's wait limit, 2 s by default); a wait
// that runs out records a code in the error flag (KLS_ERR_TIMEOUT on the
// host) and the CTA pair winds down; TMEM is released after all issued MMAs
// completed.
#include "kls_internal.cuh"
#include "kls_tcgen05.cuh"
#include <algorithm>

namespace {
using namespace kls_tc;

constexpr int TM_AB = 64;              // alphas per CTA (128 A rows)
constexpr int TM_KB = 32;              // complex k per stage
constexpr int TM_BSTAGES_MAX = 4;      // shared-memory stages of the B halves (4 or 3)
constexpr int TM_YSTAGES = 3;          // shared-memory stages of the A-source tiles
constexpr int TM_ASTAGES_MAX = 3;      // TMEM stages of A (3 when Npad <= 320, else 2)
constexpr int TM_WSTAGES = 8;          // weights ring
constexpr int TM_CHUNK = 128;          // default stages per FP32 accumulation chunk (4096 k)
constexpr int TM_THREADS = 640;
constexpr int TM_NPROD = 8;            // producer warps 4..11
constexpr int TM_NDRAIN = 8;           // drain warps 12..19
constexpr int TM_TMEM_COLS = 512;
constexpr int TM_YTILE = TM_AB * TM_KB * 2;   // 4 KB: 64 rows x 64 B
constexpr int TM_WVAR = KLS_TM_WVAR;          // coefficient variants per k pair
constexpr int TM_WBYTES = TM_KB / 2 * TM_WVAR * 16;   // 512 B: weights of one stage

__host__ __device__ constexpr int tm_astages(int Npad) { return Npad <= 320 ? 3 : 2; }

__host__ __device__ constexpr int tm_btile(int Npad) { return (Npad / 2) * TM_KB * 2; }
// B ring depth: 4 stages up to Npad = 320 (224 KB of shared memory in all),
// 3 at Npad = 384
__host__ __device__ constexpr int tm_bstages(int Npad) { return Npad <= 320 ? 4 : 3; }
size_t tm_smem(int Npad) {
  return (size_t)tm_bstages(Npad) * 4 * tm_btile(Npad) + (size_t)TM_YSTAGES * 4 * TM_YTILE +
         TM_WSTAGES * TM_WBYTES + 1024;
}

struct TmParams {
  int Npad;                 // N_alpha_pad (<= 384, multiple of 64)
  int tiles_a;              // Npad / 64
  int n_tiles;              // n_omega * tiles_a
  int splits, kb_per_split, nkb_total;
  int64_t K_pad;
  unsigned long long wait_ns;
  int fault_skip;           // test hook: one producer arrival is skipped
  int chunk;                // stages per FP32 accumulation chunk
};

// output row b of the table for accumulator column j (the pair splits each
// MMA's N columns: the first half from the leader's B rows, the rest from the
// peer's; CTA c holds table rows [c Npad/2, (c+1) Npad/2))
__device__ __forceinline__ int tm_brow(int j, int Nh, int Nh2) {
  const int nh = j / Nh, jj = j - nh * Nh, h2 = Nh >> 1;
  return jj < h2 ? nh * h2 + jj : Nh2 + nh * h2 + (jj - h2);
}

// One CTA of a pair: tile `tile_pair` x 2 + its cluster rank, K split `split`.
__device__ __forceinline__ void tm_body(const CUtensorMap* tbh, const CUtensorMap* tbl,
                                        const CUtensorMap* tyh, const CUtensorMap* tyl,
                                        const TmParams& P, int tile_pair, int split,
                                        const float2* __restrict__ wt32,
                                        double* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_b_full[TM_BSTAGES_MAX], bar_b_empty[TM_BSTAGES_MAX],
      bar_y_full[TM_YSTAGES], bar_y_empty[TM_YSTAGES], bar_w_full[TM_WSTAGES],
      bar_w_empty[TM_WSTAGES], bar_a_full[TM_ASTAGES_MAX], bar_a_empty[TM_ASTAGES_MAX], bar_acc_full,
      bar_acc_empty, bar_done;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t crank;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(crank));
  const bool leader = crank == 0;
  const int tile = 2 * tile_pair + (int)crank;
  const bool dummy = tile >= P.n_tiles;      // odd tile count: the last peer only loads B
  const int tile_e = dummy ? 0 : tile;
  const int om = tile_e / P.tiles_a;
  const int a0 = (tile_e % P.tiles_a) * TM_AB;
  const int kb0 = split * P.kb_per_split;
  const int nkb = max(0, min(P.nkb_total, kb0 + P.kb_per_split) - kb0);
  const int CH = P.chunk;
  const int nch = (nkb + CH - 1) / CH;
  const int Nh2 = P.Npad / 2;                // table rows per CTA
  const int nmma = P.Npad > 256 ? 2 : 1;     // MMAs along N
  const int NA = tm_astages(P.Npad);         // TMEM stages of A
  const uint32_t acol = (uint32_t)(TM_TMEM_COLS - 64 * NA);
  const int Nh = P.Npad / nmma;              // N of each MMA
  const int BT = tm_btile(P.Npad), NB = tm_bstages(P.Npad);
  const unsigned long long lim = P.wait_ns;

  // B tile (part 0 hi / 1 lo, sub 0 Re rows / 1 Im rows) of B stage s, and
  // A-source tile of A-source stage s
  uint8_t* yring = smem + (size_t)NB * 4 * BT;
  auto b_tile = [&](int s, int pt, int sub) {
    return smem + (size_t)(4 * s + 2 * pt + sub) * BT;
  };
  auto y_tile = [&](int s, int pt, int sub) {
    return yring + (size_t)(4 * s + 2 * pt + sub) * TM_YTILE;
  };
  uint8_t* wring = yring + (size_t)TM_YSTAGES * 4 * TM_YTILE;

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < NB; ++s) {
      mbar_init(smem_u32(&bar_b_full[s]), 1);
      mbar_init(smem_u32(&bar_b_empty[s]), 1);
    }
    for (int s = 0; s < TM_YSTAGES; ++s) {
      mbar_init(smem_u32(&bar_y_full[s]), 1);
      mbar_init(smem_u32(&bar_y_empty[s]), TM_NPROD);
    }
    for (int s = 0; s < TM_WSTAGES; ++s) {
      mbar_init(smem_u32(&bar_w_full[s]), 1);
      mbar_init(smem_u32(&bar_w_empty[s]), TM_NPROD);
    }
    for (int s = 0; s < NA; ++s) {
      mbar_init(smem_u32(&bar_a_full[s]), 2 * TM_NPROD);
      mbar_init(smem_u32(&bar_a_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_acc_full), 1);
    mbar_init(smem_u32(&bar_acc_empty), 2 * TM_NDRAIN);
    mbar_init(smem_u32(&bar_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2 && nkb > 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(TM_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();            // both CTAs' barriers initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    // ---------------- TMA: B halves (leader's barrier) + A-source tiles (own)
    if (lane == 0 && nkb > 0) {
      int issued = 0;
      const int yb = (int)crank * Nh2;
      for (int i = 0; i < nkb; ++i) {
        const int sb = i % NB, rb = i / NB, sy = i % TM_YSTAGES, ry = i / TM_YSTAGES;
        if (!mbar_wait_cl_lim(smem_u32(&bar_b_empty[sb]), (rb & 1) ^ 1, &s_abort, err, 1, lim))
          break;
        if (!mbar_wait_lim(smem_u32(&bar_y_empty[sy]), (ry & 1) ^ 1, &s_abort, err, 11, lim)) break;
        // stage g of 32 k: half (g & 1) of the table's 64-k block g >> 1
        const int g = kb0 + i, kx = (g & 1) * TM_KB, kz = g >> 1;
        if (leader) mbar_arrive_tx(smem_u32(&bar_b_full[sb]), 2 * 4 * BT);
        const uint32_t fb = mapa_u32(smem_u32(&bar_b_full[sb]), 0);
        tma_load_3d_pair(smem_u32(b_tile(sb, 0, 0)), tbh, kx, yb, kz, fb);
        tma_load_3d_pair(smem_u32(b_tile(sb, 0, 1)), tbh, kx, P.Npad + yb, kz, fb);
        tma_load_3d_pair(smem_u32(b_tile(sb, 1, 0)), tbl, kx, yb, kz, fb);
        tma_load_3d_pair(smem_u32(b_tile(sb, 1, 1)), tbl, kx, P.Npad + yb, kz, fb);
        const uint32_t yf = smem_u32(&bar_y_full[sy]);
        mbar_arrive_tx(yf, 4 * TM_YTILE);
        tma_load_3d(smem_u32(y_tile(sy, 0, 0)), tyh, kx, a0, kz, yf);
        tma_load_3d(smem_u32(y_tile(sy, 0, 1)), tyh, kx, P.Npad + a0, kz, yf);
        tma_load_3d(smem_u32(y_tile(sy, 1, 0)), tyl, kx, a0, kz, yf);
        tma_load_3d(smem_u32(y_tile(sy, 1, 1)), tyl, kx, P.Npad + a0, kz, yf);
        issued = i + 1;
      }
      // the last copies into this CTA's shared memory land before it may exit
      // (the peer's B copies complete on the leader's barrier, which the
      // leader checks; the final cluster barrier orders the peer's exit)
      for (int i = max(0, issued - TM_YSTAGES); i < issued; ++i)
        mbar_wait_lim(smem_u32(&bar_y_full[i % TM_YSTAGES]), (i / TM_YSTAGES) & 1, nullptr, err,
                      6, lim);
      if (leader)
        for (int i = max(0, issued - NB); i < issued; ++i)
          mbar_wait_cl_lim(smem_u32(&bar_b_full[i % NB]), (i / NB) & 1, nullptr, err, 6, lim);
    }
  } else if (warp == 3) {
    // ---------------- weights ring
    if (lane == 0 && nkb > 0) {
      int issued = 0;
      // weights of omega om: TM_WVAR float2 per k (the pre-signed variants)
      const float2* wz = wt32 + (size_t)om * P.K_pad * TM_WVAR;
      for (int i = 0; i < nkb; ++i) {
        const int ws = i % TM_WSTAGES, r = i / TM_WSTAGES;
        if (!mbar_wait_lim(smem_u32(&bar_w_empty[ws]), (r & 1) ^ 1, &s_abort, err, 10, lim)) break;
        const uint32_t wb = smem_u32(&bar_w_full[ws]);
        mbar_arrive_tx(wb, TM_WBYTES);
        bulk_load(smem_u32(wring + ws * TM_WBYTES), wz + (size_t)(kb0 + i) * TM_KB * TM_WVAR,
                  TM_WBYTES, wb);
        issued = i + 1;
      }
      for (int i = max(0, issued - TM_WSTAGES); i < issued; ++i)
        mbar_wait_lim(smem_u32(&bar_w_full[i % TM_WSTAGES]), (i / TM_WSTAGES) & 1, nullptr, err,
                      6, lim);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader): the whole warp waits, one elected
    // lane issues.  B descriptors are formed once: a tile's descriptor is the
    // first tile's plus (byte offset >> 4) (shared addresses stay below
    // 256 KB, so the add never carries out of the 14-bit start field).
    if (leader && nkb > 0) {
      const uint32_t idesc = idesc_bf16(256, Nh);
      const uint64_t d00 = sw64_desc(smem_u32(b_tile(0, 0, 0)));
      const uint32_t t16 = (uint32_t)BT >> 4;                  // one B tile
      const uint32_t nh16 = (uint32_t)((Nh >> 1) * 64) >> 4;   // second N half
      const bool issuer = elect_one();
      for (int i = 0; i < nkb; ++i) {
        const int s = i % NB, as = i % NA;
        const int ci = i % CH, ch = i / CH;
        const bool first = ci == 0;
        const bool last = ci == CH - 1 || i == nkb - 1;
        bool ok = true;
        if (first && ch > 0)
          ok = mbar_wait_cl_lim(smem_u32(&bar_acc_empty), (ch - 1) & 1, &s_abort, err, 7, lim);
        if (ok) ok = mbar_wait_cl_lim(smem_u32(&bar_b_full[s]), (i / NB) & 1, &s_abort, err, 2, lim);
        if (ok) ok = mbar_wait_cl_lim(smem_u32(&bar_a_full[as]), (i / NA) & 1, &s_abort, err, 3, lim);
        if (!__all_sync(0xffffffffu, ok)) break;
        tc_fence_after();
        if (issuer) {
          // tile (s, part, sub) sits at (4 s + 2 part + sub) tiles; k 16..31
          // of a 64-byte row start 32 bytes in
          const uint64_t ds = d00 + (uint64_t)(4 * s) * t16;
          const uint32_t a_s = tmem + acol + (uint32_t)(as * 64);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t bh = ds + (uint64_t)((kk >> 1) * t16 + (kk & 1) * 2);   // Re, then Im rows
            const uint64_t bl = bh + 2 * t16;
            const uint32_t a_hi = a_s + (uint32_t)(kk * 8), a_lo = a_hi + 32;
            const uint32_t acc0 = (first && kk == 0) ? 0u : 1u;
#pragma unroll
            for (int nh = 0; nh < 2; ++nh) {
              if (nh < nmma) {
                const uint32_t d = tmem + (uint32_t)(nh * Nh);
                const uint64_t o = (uint64_t)(nh * nh16);
                umma_pair_ts(d, a_hi, bh + o, idesc, acc0);
                umma_pair_ts(d, a_lo, bh + o, idesc, 1u);
                umma_pair_ts(d, a_hi, bl + o, idesc, 1u);
              }
            }
          }
          umma_pair_commit(smem_u32(&bar_b_empty[s]));
          umma_pair_commit(smem_u32(&bar_a_empty[as]));
          if (last) umma_pair_commit(smem_u32(&bar_acc_full));
        }
        __syncwarp();
      }
      // completion of every issued MMA (also on the abort path)
      if (issuer) umma_pair_commit(smem_u32(&bar_done));
    }
  } else if (warp >= 4 && warp < 4 + TM_NPROD) {
    // ---------------- producers: A rows of this CTA's 64 alphas into TMEM
    const int pw = warp - 4, q = pw & 3, kh = pw >> 2;
    const int l = 32 * q + lane;               // TMEM lane = A row
    const int al = l >> 1, p = l & 1;          // rows (a, r) at lane 2a, (a, i) at 2a + 1
    // With U = w conj(W): row (a, r) is [Re U | -Im U] and (a, i) is
    // [Im U | Re U] over the halves (Re W columns | Im W columns) of the
    // stage.  Each lane forms its own component over this warp's 16 k
    // (k pairs j = 8 kh .. 8 kh + 7), c1 ReW + c2 ImW with (c1, c2) = (wr, wi)
    // (Re U, lane 2a) or (wi, -wr) (Im U, lane 2a + 1), for half 0, and takes
    // its half-1 values from its partner lane, negated for the (a, r) row
    // (the split of -x is the negated split of x, so the bits are those the
    // formula would give).
    const int var = p;                         // weight variant 0 or 1
    const uint32_t neg = p ? 0u : 0x80008000u; // sign bits of a BF16 pair
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16) + acol + (uint32_t)(kh * 8);
    const bool skip_one = P.fault_skip && leader && tile_pair == 0 && split == 0 && pw == 0;
    for (int i = 0; i < nkb; ++i) {
      const int s = i % TM_YSTAGES, as = i % NA, ws = i % TM_WSTAGES;
      bool ok = mbar_wait_lim(smem_u32(&bar_y_full[s]), (i / TM_YSTAGES) & 1, &s_abort, err, 4, lim);
      if (ok) ok = mbar_wait_lim(smem_u32(&bar_w_full[ws]), (i / TM_WSTAGES) & 1, &s_abort, err, 8,
                                 lim);
      if (ok) ok = mbar_wait_cl_lim(smem_u32(&bar_a_empty[as]), ((i / NA) & 1) ^ 1, &s_abort, err,
                                    12, lim);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      // (c1 pair, c2 pair) of k = 2j, 2j + 1 at float4 number TM_WVAR j + var
      const float4* wz = reinterpret_cast<const float4*>(wring + ws * TM_WBYTES) + var;
      uint32_t hi[8], lo[8], hi1[8], lo1[8];
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        // 16-byte chunk c of the alpha's table rows: k = 8c .. 8c + 7
        const int c = 2 * kh + cc;
        const uint32_t off = sw64_off(al, c);
        const uint4 Rh = *reinterpret_cast<const uint4*>(y_tile(s, 0, 0) + off);
        const uint4 Ih = *reinterpret_cast<const uint4*>(y_tile(s, 0, 1) + off);
        const uint4 Rl = *reinterpret_cast<const uint4*>(y_tile(s, 1, 0) + off);
        const uint4 Il = *reinterpret_cast<const uint4*>(y_tile(s, 1, 1) + off);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int j = 4 * c + e;               // k = 2j, 2j + 1
          const uint64_t wr = f2_add(f2_bf16x2((&Rh.x)[e]), f2_bf16x2((&Rl.x)[e]));
          const uint64_t wi = f2_add(f2_bf16x2((&Ih.x)[e]), f2_bf16x2((&Il.x)[e]));
          const float4 cw = wz[TM_WVAR * j];
          const uint64_t v = f2_fma(f2_pack(cw.x, cw.y), wr, f2_mul(f2_pack(cw.z, cw.w), wi));
          hi[4 * cc + e] = pack_split2(v, lo[4 * cc + e]);
        }
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        hi1[t] = __shfl_xor_sync(0xffffffffu, hi[t], 1) ^ neg;
        lo1[t] = __shfl_xor_sync(0xffffffffu, lo[t], 1) ^ neg;
      }
      TMEM_ST8(tl + (uint32_t)(as * 64), hi);
      TMEM_ST8(tl + (uint32_t)(as * 64 + 32), lo);
      TMEM_ST8(tl + (uint32_t)(as * 64 + 16), hi1);
      TMEM_ST8(tl + (uint32_t)(as * 64 + 48), lo1);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(smem_u32(&bar_y_empty[s]));
        mbar_arrive(smem_u32(&bar_w_empty[ws]));
        if (!(skip_one && i == 0)) {
          if (leader) mbar_arrive(smem_u32(&bar_a_full[as]));
          else mbar_arrive_remote_cta(mapa_u32(smem_u32(&bar_a_full[as]), 0));
        }
      }
    }
  } else if (warp >= 4 + TM_NPROD) {
    // ---------------- drain: D chunk -> FP64 partial [tile][split][b][A row]
    const int dw = warp - 4 - TM_NPROD, q = dw & 3, half = dw >> 2;
    const int l = 32 * q + lane;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    double* out = part + ((size_t)tile_e * P.splits + split) * (size_t)P.Npad * 128 + l;
    const int c0 = half * Nh2;
    for (int ch = 0; ch < nch; ++ch) {
      const bool ok =
          mbar_wait_cl_lim(smem_u32(&bar_acc_full), ch & 1, &s_abort, err, 9, lim);
      if (!__all_sync(0xffffffffu, ok)) break;
      tc_fence_after();
      for (int cb = 0; cb < Nh2 / 16; ++cb) {
        const int j0 = c0 + 16 * cb;
        uint32_t v[16];
        TMEM_LD16(tl + (uint32_t)j0, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (dummy) continue;
        // first chunk: plain stores; later chunks: FP64 reductions in L2
        // (fire-and-forget, so the accumulator is free again as soon as it
        // is read).  Each partial element is written by this one thread, in
        // chunk order (same-thread, same-address operations are ordered), so
        // the sums are deterministic: ((c0 + c1) + c2) + ...
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          double* dst = out + (size_t)tm_brow(j0 + t, Nh, Nh2) * 128;
          const double x = (double)__uint_as_float(v[t]);
          if (ch == 0) *dst = x;
          else asm volatile("red.global.add.f64 [%0], %1;" ::"l"(dst), "d"(x) : "memory");
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (leader) mbar_arrive(smem_u32(&bar_acc_empty));
        else mbar_arrive_remote_cta(mapa_u32(smem_u32(&bar_acc_empty), 0));
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  // every role has finished; all MMAs complete before TMEM is released
  if (warp == 2 && nkb > 0) mbar_wait_cl_lim(smem_u32(&bar_done), 0, nullptr, err, 5, lim);
  cluster_sync_all();            // no CTA leaves while its peer may still touch it
  if (warp == 2 && nkb > 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TM_TMEM_COLS));
  }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TM_THREADS, 1)
mixed_tm_kernel(const __grid_constant__ CUtensorMap tb_h, const __grid_constant__ CUtensorMap tb_l,
                const __grid_constant__ CUtensorMap ty_h, const __grid_constant__ CUtensorMap ty_l,
                TmParams P, const float2* __restrict__ wt32, double* __restrict__ part,
                int* __restrict__ err) {
  tm_body(&tb_h, &tb_l, &ty_h, &ty_l, P, (int)(blockIdx.x >> 1), (int)blockIdx.y, wt32, part, err);
}

// Uneven batch: one cluster per work item (model, tile pair, K split); the
// model's tensor maps and parameters come from device descriptors.  Each
// item runs exactly the one-model kernel's body, so a determinant is bitwise
// what the model's own context returns in this form.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TM_THREADS, 1)
mixed_tm_multi_kernel(const kls_tm_model* __restrict__ md, const int4* __restrict__ items,
                      int* __restrict__ err) {
  const int4 it = items[blockIdx.x >> 1];
  const kls_tm_model& d = md[it.x];
  tensormap_acquire(&d.tb_h);
  tensormap_acquire(&d.tb_l);
  tensormap_acquire(&d.ty_h);
  tensormap_acquire(&d.ty_l);
  TmParams P;
  P.Npad = d.Npad;
  P.tiles_a = d.tiles_a;
  P.n_tiles = d.n_tiles;
  P.splits = d.splits;
  P.kb_per_split = d.kb_per_split;
  P.nkb_total = d.nkb_total;
  P.K_pad = d.K_pad;
  P.wait_ns = d.wait_ns;
  P.fault_skip = 0;
  P.chunk = d.chunk;
  tm_body(&d.tb_h, &d.tb_l, &d.ty_h, &d.ty_l, P, it.y, it.z, d.wt32, d.part, err);
}

// FP32 weights as the producers read them: for k = 2j, 2j + 1 two float4
// (c1 pair, c2 pair) = (wr, wi) and (wi, -wr); negation is exact, so each
// variant rounds like the plain FP32 weight
__device__ __forceinline__ void tm_weight_variants(int64_t K_pad, const double2* __restrict__ wt,
                                                   float4* __restrict__ out) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < K_pad / 2;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = wt[2 * j], b = wt[2 * j + 1];
    const float r0 = (float)a.x, i0 = (float)a.y, r1 = (float)b.x, i1 = (float)b.y;
    out[2 * j] = make_float4(r0, r1, i0, i1);
    out[2 * j + 1] = make_float4(i0, i1, -r0, -r1);
  }
}

// uneven batch: FP32 weight variants of every (model, omega) pair
__global__ void tm_multi_weights32_kernel(const kls_mdesc* __restrict__ md,
                                          const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  tm_weight_variants(d.K_pad, d.wt + (size_t)pz.y * d.K_pad,
                     reinterpret_cast<float4*>(d.wt32) + (size_t)pz.y * (d.K_pad / 2) * TM_WVAR);
}

// uneven batch: split sum, * G * N(a), I - M per (model, omega) pair; mpart is
// the model's TMEM-form partial [batch * tiles_a][splits][Npad][128]
__global__ void tm_multi_reduce_kernel(const kls_mdesc* __restrict__ md,
                                       const int2* __restrict__ pairs) {
  const int2 pz = pairs[blockIdx.y];
  const kls_mdesc& d = md[pz.x];
  const int Na = d.Na, tiles_a = d.Na_pad / TM_AB;
  const size_t plane = (size_t)d.Na_pad * 128;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Na * Na; e += gridDim.x * blockDim.x) {
    const int b = e / Na, a = e % Na;
    const int at = a / TM_AB, la = 2 * (a % TM_AB);   // rows (a, r) at 2a, (a, i) at 2a + 1
    const double* src =
        d.mpart + (size_t)(pz.y * tiles_a + at) * d.msplits * plane + (size_t)b * 128 + la;
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < d.msplits; ++s) {
      sr += src[(size_t)s * plane];
      si += src[(size_t)s * plane + 1];
    }
    const double n = d.Nk[a];
    const double mr = __dmul_rn(__dmul_rn(sr, d.G), n), mi = __dmul_rn(__dmul_rn(si, d.G), n);
    d.A[(size_t)pz.y * Na * Na + e] = make_double2((a == b ? 1.0 : 0.0) - mr, -mi);
  }
}

// FP32 weight variants, [omega][K_pad / 2][TM_WVAR] float4
__global__ void tm_weights32_kernel(int64_t K_pad, const double2* __restrict__ wt,
                                    float4* __restrict__ wt32) {
  const int z = blockIdx.y;
  tm_weight_variants(K_pad, wt + (size_t)z * K_pad, wt32 + (size_t)z * (K_pad / 2) * TM_WVAR);
}

// split sum, * G * N(a), I - M: partial [tile][split][b][A row], A row
// 2 a_local (Re) or 2 a_local + 1 (Im)
__global__ void tm_reduce_kernel(int Na, int Npad, int tiles_a, int splits, double G,
                                 const double* __restrict__ Nk, const double* __restrict__ part,
                                 double2* __restrict__ A, double2* __restrict__ Mout,
                                 const double2* __restrict__ Ma) {
  const int z = blockIdx.y;
  const size_t plane = (size_t)Npad * 128;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Na * Na; e += gridDim.x * blockDim.x) {
    const int b = e / Na, a = e % Na;
    const int at = a / TM_AB, la = 2 * (a % TM_AB);   // rows (a, r) at 2a, (a, i) at 2a + 1
    const double* src = part + (size_t)(z * tiles_a + at) * splits * plane + (size_t)b * 128 + la;
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < splits; ++s) {
      sr += src[(size_t)s * plane];
      si += src[(size_t)s * plane + 1];
    }
    const double n = Nk[a];
    double mr = __dmul_rn(__dmul_rn(sr, G), n), mi = __dmul_rn(__dmul_rn(si, G), n);
    if (Ma) {                                  // anchored: M(omega_a) + delta M
      mr = __dadd_rn(Ma[e].x, mr);
      mi = __dadd_rn(Ma[e].y, mi);
    }
    A[(size_t)z * Na * Na + e] = make_double2((a == b ? 1.0 : 0.0) - mr, -mi);
    if (Mout && z == 0) Mout[e] = make_double2(mr, mi);
  }
}

// The dynamic shared-memory limit is a property of the kernel, shared by
// every context in the process: set it once to the largest stage layout of
// any N_alpha_pad (64 .. 384), so that contexts of any size can launch.
size_t tm_smem_max() {
  size_t mx = 0;
  for (int n = 64; n <= 384; n += 64) mx = std::max(mx, tm_smem(n));
  return mx;
}
cudaError_t tm_set_smem_limits() {
  cudaError_t e = cudaFuncSetAttribute(mixed_tm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tm_smem_max());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(mixed_tm_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tm_smem_max());
  return e;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct kls_mixed_tm {
  CUtensorMap tb_h, tb_l, ty_h, ty_l;
  int splits = 1;
  int chunk = TM_CHUNK;         // stages per FP32 accumulation chunk
  double* part = nullptr;       // [n tiles][splits][Npad][128]
  size_t part_elems = 0;
  float2* wt32 = nullptr;       // [n][K_pad / 2][TM_WVAR] float4 weight variants
  size_t wt32_elems = 0;
};

bool kls_tm_supported(const kls_ctx* c) {
  return c->Na_pad % TM_AB == 0 && c->Na_pad <= 384 && c->K_pad % 64 == 0;
}

// K splits of the form: fixed per context (determinants do not depend on the
// batch).  With as many splits as CTA pairs can be resident at once, every
// batch fills whole waves: (tile pairs of the batch) x splits is a multiple
// of the resident pairs for any number of omegas.
int kls_tm_default_splits(const kls_ctx* c) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  int pairs = sms / 2;
  tm_set_smem_limits();
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(2 * pairs, 1, 1);
  lc.blockDim = dim3(TM_THREADS, 1, 1);
  lc.dynamicSmemBytes = tm_smem(c->Na_pad);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, (void*)mixed_tm_kernel, &lc) == cudaSuccess &&
      clusters > 0)
    pairs = clusters;
  else
    cudaGetLastError();
  const int nkb = (int)(c->K_pad / TM_KB);
  return std::max(1, std::min(nkb, pairs));
}

int kls_tm_create(kls_ctx* c, const void* Xh, const void* Xl, kls_mixed_tm** out) {
  *out = nullptr;
  if (!kls_tm_supported(c)) return kls_fail(c, KLS_ERR_UNSUPPORTED, "N_alpha_pad > 384");
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  KLS_CK(c, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess)
    return kls_fail(c, KLS_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn encode = (EncodeTiledFn)fn;
  kls_mixed_tm* t = new kls_mixed_tm();
  // the split table in 64-k blocks: {64 k, 2 Na_pad rows, K_pad / 64 blocks}
  const cuuint64_t rows = (cuuint64_t)(2 * c->Na_pad);
  const cuuint64_t dims[3] = {64, rows, (cuuint64_t)(c->K_pad / 64)};
  const cuuint64_t strides[2] = {64 * sizeof(__nv_bfloat16), rows * 64 * sizeof(__nv_bfloat16)};
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box_b[3] = {TM_KB, (cuuint32_t)(c->Na_pad / 2), 1};
  const cuuint32_t box_y[3] = {TM_KB, TM_AB, 1};
  struct { CUtensorMap* m; const void* base; const cuuint32_t* box; } maps[4] = {
      {&t->tb_h, Xh, box_b}, {&t->tb_l, Xl, box_b}, {&t->ty_h, Xh, box_y}, {&t->ty_l, Xl, box_y}};
  for (auto& mm : maps) {
    CUresult r = encode(mm.m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(mm.base),
                        dims, strides, mm.box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      delete t;
      return kls_fail(c, KLS_ERR_CUDA, "cuTensorMapEncodeTiled failed (TMEM-operand form)");
    }
  }
  t->splits = kls_tm_default_splits(c);
  cudaError_t e = tm_set_smem_limits();
  if (e != cudaSuccess) {
    delete t;
    return kls_cuda_fail(c, e, "cudaFuncSetAttribute (TMEM-operand form)");
  }
  *out = t;
  return KLS_OK;
}

void kls_tm_destroy(kls_mixed_tm* t) {
  if (!t) return;
  cudaFree(t->part);
  cudaFree(t->wt32);
  delete t;
}

int kls_tm_splits(const kls_mixed_tm* t) { return t->splits; }

void kls_tm_set_splits(const kls_ctx* c, kls_mixed_tm* t, int s) {
  t->splits = std::max(1, std::min(s, (int)(c->K_pad / TM_KB)));
}

void kls_tm_set_chunk(kls_mixed_tm* t, int stages) { t->chunk = std::max(1, stages); }

int kls_tm_contract(kls_ctx* c, kls_mixed_tm* t, int n, int* d_err, unsigned long long wait_ns,
                    int fault_skip) {
  const int tiles_a = c->Na_pad / TM_AB;
  const int nkb_total = (int)(c->K_pad / TM_KB);
  const int kbs = (nkb_total + t->splits - 1) / t->splits;
  const int splits = (nkb_total + kbs - 1) / kbs;          // no empty split
  const int n_tiles = n * tiles_a;
  const size_t need = (size_t)n_tiles * splits * c->Na_pad * 128;
  if (need > t->part_elems) {
    cudaFree(t->part);
    t->part = nullptr;
    t->part_elems = 0;
    KLS_CK(c, cudaMalloc(&t->part, need * sizeof(double)));
    t->part_elems = need;
  }
  const size_t nw = (size_t)n * c->K_pad * TM_WVAR;      // float2
  if (nw > t->wt32_elems) {
    cudaFree(t->wt32);
    t->wt32 = nullptr;
    t->wt32_elems = 0;
    KLS_CK(c, cudaMalloc(&t->wt32, nw * sizeof(float2)));
    t->wt32_elems = nw;
  }
  const unsigned wblocks = (unsigned)std::min<int64_t>((c->K_pad / 2 + 255) / 256, 2048);
  tm_weights32_kernel<<<dim3(wblocks, n), 256, 0, c->stream>>>(
      c->K_pad, c->d_wt, reinterpret_cast<float4*>(t->wt32));
  KLS_LAUNCHED(c);
  TmParams P{};
  P.Npad = c->Na_pad;
  P.tiles_a = tiles_a;
  P.n_tiles = n_tiles;
  P.splits = splits;
  P.kb_per_split = kbs;
  P.nkb_total = nkb_total;
  P.K_pad = c->K_pad;
  P.wait_ns = wait_ns;
  P.fault_skip = fault_skip;
  P.chunk = t->chunk;
  const int pairs = (n_tiles + 1) / 2;
  dim3 grid((unsigned)(2 * pairs), (unsigned)splits);
  mixed_tm_kernel<<<grid, TM_THREADS, tm_smem(c->Na_pad), c->stream>>>(
      t->tb_h, t->tb_l, t->ty_h, t->ty_l, P, t->wt32, t->part, d_err);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

void kls_tm_describe(const kls_ctx* c, const kls_mixed_tm* t, unsigned long long wait_ns,
                     int batch, kls_tm_model* d) {
  d->tb_h = t->tb_h;
  d->tb_l = t->tb_l;
  d->ty_h = t->ty_h;
  d->ty_l = t->ty_l;
  d->Npad = c->Na_pad;
  d->tiles_a = c->Na_pad / TM_AB;
  d->n_tiles = batch * d->tiles_a;
  d->nkb_total = (int)(c->K_pad / TM_KB);
  d->kb_per_split = (d->nkb_total + t->splits - 1) / t->splits;
  d->splits = (d->nkb_total + d->kb_per_split - 1) / d->kb_per_split;
  d->chunk = t->chunk;
  d->K_pad = c->K_pad;
  d->wait_ns = wait_ns;
  d->wt32 = nullptr;
  d->part = nullptr;
  d->pad = 0;
}

int kls_tm_multi_launch(cudaStream_t st, const kls_mdesc* d_md, const kls_tm_model* d_tm,
                        const int2* d_pairs, int n_pairs, const int4* d_items, int n_items,
                        int64_t max_K_pad, int max_Npad, int* d_err, const kls_tm_model* h_tm,
                        int n_models, bool per_model) {
  cudaError_t e;
  const int wblocks = (int)std::min<int64_t>((max_K_pad + 255) / 256, 1024);
  tm_multi_weights32_kernel<<<dim3(wblocks, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  if ((e = tm_set_smem_limits()) != cudaSuccess) return (int)e;
  if (per_model) {
    // one launch of the single-model kernel per model (tensor maps as
    // kernel parameters): the same body and parameters, hence the same bits
    for (int i = 0; i < n_models; ++i) {
      const kls_tm_model& d = h_tm[i];
      TmParams P{};
      P.Npad = d.Npad;
      P.tiles_a = d.tiles_a;
      P.n_tiles = d.n_tiles;
      P.splits = d.splits;
      P.kb_per_split = d.kb_per_split;
      P.nkb_total = d.nkb_total;
      P.K_pad = d.K_pad;
      P.wait_ns = d.wait_ns;
      P.fault_skip = 0;
      P.chunk = d.chunk;
      const dim3 grid((unsigned)(2 * ((d.n_tiles + 1) / 2)), (unsigned)d.splits);
      mixed_tm_kernel<<<grid, TM_THREADS, tm_smem(d.Npad), st>>>(d.tb_h, d.tb_l, d.ty_h, d.ty_l,
                                                                 P, d.wt32, d.part, d_err);
      if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    }
  } else {
    mixed_tm_multi_kernel<<<2 * n_items, TM_THREADS, tm_smem_max(), st>>>(d_tm, d_items,
                                                                               d_err);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  }
  tm_multi_reduce_kernel<<<dim3(256, n_pairs), 256, 0, st>>>(d_md, d_pairs);
  return (int)cudaGetLastError();
}

int kls_tm_reduce(kls_ctx* c, kls_mixed_tm* t, int n, bool export_M, const double2* Ma) {
  const int nkb_total = (int)(c->K_pad / TM_KB);
  const int kbs = (nkb_total + t->splits - 1) / t->splits;
  const int splits = (nkb_total + kbs - 1) / kbs;
  int blocks = std::min((c->Na * c->Na + 255) / 256, 1024);
  tm_reduce_kernel<<<dim3(blocks, n), 256, 0, c->stream>>>(
      c->Na, c->Na_pad, c->Na_pad / TM_AB, splits, c->cfg.G, c->d_N, t->part, c->d_A,
      export_M ? c->d_M : nullptr, Ma);
  KLS_LAUNCHED(c);
  return KLS_OK;
}

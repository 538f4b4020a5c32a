// PTX helpers shared by the tcgen05 / TMA contraction kernels (sm_100a):
// mbarriers with bounded waits, UMMA shared-memory and instruction
// descriptors, tcgen05.mma (shared-memory and tensor-memory A operands, one
// CTA or a CTA pair), tcgen05.ld / st, TMA tensor and bulk copies.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace kls_tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// cluster-scope acquire: barriers that the peer CTA (or its commits) complete
__device__ __forceinline__ bool mbar_try_cl(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (limit_ns of %globaltimer): false when the CTA is aborting
// (*abort set by another role) or the wait ran out, in which case it sets
// *abort and records `code` in *err (first failure wins).  Never spins forever.
template <bool CLUSTER>
__device__ __forceinline__ bool mbar_wait_impl(uint32_t a, uint32_t parity, volatile int* abort,
                                               int* err, int code, unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if (CLUSTER ? mbar_try_cl(a, parity) : mbar_try(a, parity)) return true;
    if (abort && *abort) return false;
    if ((it & 63) == 0) {
      unsigned long long t = globaltimer();
      if (t0 == 0) t0 = t;
      else if (t - t0 > limit_ns) {
        if (abort) *abort = 1;
        atomicCAS(err, 0, code);
        return false;
      }
    }
  }
}
__device__ __forceinline__ bool mbar_wait_lim(uint32_t a, uint32_t parity, volatile int* abort,
                                              int* err, int code, unsigned long long limit_ns) {
  return mbar_wait_impl<false>(a, parity, abort, err, code, limit_ns);
}
__device__ __forceinline__ bool mbar_wait_cl_lim(uint32_t a, uint32_t parity,
                                                 volatile int* abort, int* err, int code,
                                                 unsigned long long limit_ns) {
  return mbar_wait_impl<true>(a, parity, abort, err, code, limit_ns);
}
// one lane of the (fully active) warp, the same on every call: the warp
// stays converged around the MMA issue, so its loop state is warp-uniform
__device__ __forceinline__ bool elect_one() {
  uint32_t pred;
  asm volatile(
      "{\n.reg .pred p;\nelect.sync _|p, 0xffffffff;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(pred));
  return pred != 0;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// K-major, 128-byte swizzle UMMA shared-memory descriptor (sm100 format):
// start >> 4 in [0,14), LBO >> 4 in [16,30) (unused here), SBO = 1024 B
// (8 rows of 128 B) >> 4 in [32,46), version 1 at [46,48), layout
// SWIZZLE_128B = 2 at [61,64).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// K-major, 64-byte swizzle: rows of 64 B, SBO = 512 B (8 rows), layout
// SWIZZLE_64B = 4 at [61,64).
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;
  return d;
}
// byte offset of the 16-byte chunk c (0..3) of row n in a K-major 64-byte
// swizzled tile (address bits [4,6) ^= bits [7,9))
__device__ __forceinline__ uint32_t sw64_off(int n, int c) {
  return (uint32_t)(n * 64 + ((c ^ ((n >> 1) & 3)) << 4));
}
// kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major,
// N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                     uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            int z, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"((uint64_t)src), "r"(bytes), "r"(mbar)
      : "memory");
}
#define TMEM_LD32(taddr, r)                                                                      \
  asm volatile(                                                                                  \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13," \
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"        \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),     \
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),              \
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),           \
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),           \
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),           \
        "=r"(r[31])                                                                              \
      : "r"(taddr))
#define TMEM_LD16(taddr, r)                                                                      \
  asm volatile(                                                                                  \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13," \
      "%14,%15}, [%16];"                                                                         \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),     \
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),              \
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])                                                    \
      : "r"(taddr))
// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w writes
// lanes 32 (w % 4) .. +31)
#define TMEM_ST16(taddr, r)                                                                      \
  asm volatile(                                                                                  \
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"   \
      "%13,%14,%15,%16};" ::"r"(taddr),                                                          \
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),   \
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),         \
      "r"(r[15])                                                                                 \
      : "memory")

#define TMEM_ST8(taddr, r)                                                                       \
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(  \
                   taddr),                                                                       \
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),      \
               "r"(r[7])                                                                         \
               : "memory")

__device__ __forceinline__ float bf_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }
// error-free split of two FP32 values into BF16 high parts (returned, a in
// the low half) and BF16 low parts (lo): x = hi + lo to ~2^-17 relative
__device__ __forceinline__ uint32_t pack_split(float a, float b, uint32_t& lo) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);          // .x = a (low half)
  float ha = __low2float(h), hb = __high2float(h);
  __nv_bfloat162 l = __floats2bfloat162_rn(a - ha, b - hb);
  lo = *reinterpret_cast<uint32_t*>(&l);
  return *reinterpret_cast<uint32_t*>(&h);
}
// packed FP32 pairs (sm_100 f32x2 arithmetic): the low word holds the first
// element; each lane computes exactly what two scalar operations would
__device__ __forceinline__ uint64_t f2_pack(float a, float b) {
  return ((uint64_t)__float_as_uint(b) << 32) | __float_as_uint(a);
}
__device__ __forceinline__ uint64_t f2_bf16x2(uint32_t v) {   // (bf_lo(v), bf_hi(v))
  return ((uint64_t)(v & 0xffff0000u) << 32) | (uint32_t)(v << 16);
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// pack_split of a packed pair: the same bits as pack_split(lo word, hi word)
__device__ __forceinline__ uint32_t pack_split2(uint64_t v, uint32_t& lo) {
  uint32_t h, l;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h)
      : "f"(__uint_as_float((uint32_t)(v >> 32))), "f"(__uint_as_float((uint32_t)v)));
  const uint64_t r = f2_sub(v, f2_bf16x2(h));          // exact residuals
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l)
      : "f"(__uint_as_float((uint32_t)(r >> 32))), "f"(__uint_as_float((uint32_t)r)));
  lo = l;
  return h;
}
// byte offset of the 16-byte chunk (row n, k-chunk c) in a K-major SW128 tile
__device__ __forceinline__ uint32_t sw128_off(int n, int c) {
  return (uint32_t)((n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4));
}

// ---- CTA pairs (cluster of 2, tcgen05 cta_group::2) ---------------------------
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
// the same arrive with the default (CTA-scope) release: enough where the
// signalled work is tensor-memory traffic that tcgen05.wait has completed and
// the tcgen05 thread-sync fences order around the barrier; it spares the
// cluster-scope fence on every stage
__device__ __forceinline__ void mbar_arrive_remote_cta(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void umma_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// pair MMA with the A operand in tensor memory (each CTA's 128 A rows at the
// same TMEM address in its own TMEM), B from shared memory
__device__ __forceinline__ void umma_pair_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t b,
                                             uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(b), "r"(idesc), "r"(acc));
}
// commit of the leader's MMAs to the barrier at this offset in both CTAs
__device__ __forceinline__ void umma_pair_commit(uint32_t mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(mbar),
      "h"((unsigned short)3)
      : "memory");
}
// TMA into this CTA's shared memory, completing on the leader's barrier
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t mbar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(mbar_cluster)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap* map, int x, int y,
                                                 int z, uint32_t mbar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(mbar_cluster)
      : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
__device__ __forceinline__ void tensormap_acquire(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((uint64_t)map)
               : "memory");
}

}  // namespace kls_tc

// dsax_ptx.cuh -- thin inline-PTX helpers for sm_100a: mbarriers with
// bounded waits, tcgen05 (TMEM alloc, UMMA issue/commit, TMEM loads) and the
// UMMA shared-memory / instruction descriptors.
//
// Every wait in this library is bounded: after `limit_ns` of %globaltimer
// time the waiting thread records an error code in the kernel's device error
// word, raises a CTA-wide abort flag and returns false, so a kernel never
// spins forever.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "dsax kernels target sm_100a only"
#endif

namespace dsax {



__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}

// kCluster: acquire at cluster scope (the phase was completed by another
// CTA of the cluster: a remote arrive or remote stores with complete_tx).
template <bool kCluster = false>
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  if (kCluster)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  return ok != 0;
}

// Bounded wait on `bar` reaching phase parity `parity`.  Returns false (and
// records `code` in *err, raises *abort) when the limit expires or another
// thread already aborted.
template <bool kCluster = false>
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  volatile int *abort, int *err,
                                                  int code, uint64_t limit_ns) {
  if (mbar_try_wait<kCluster>(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait<kCluster>(bar, parity)) return true;
    // the clock is read after the second failed try (so a short limit bites
    // even where each try suspends the thread for a while) and then every
    // 64 tries
    if (it == 1u || (it & 63u) == 0) {
      if (*abort) return false;
      if (globaltimer() - t0 > limit_ns) {
        atomicOr(err, code);
        *abort = 1;
        return false;
      }
    }
  }
}

// Bound on the waits that drain a CTA's own copies and MMAs in flight before
// it frees TMEM and exits, also after an abort: at least 250 ms, so that a
// short pipeline-wait limit never lets a CTA exit while its copies are still
// landing in shared memory or its MMAs still reading it.
__device__ __forceinline__ uint64_t drain_limit(uint64_t limit_ns) {
  return limit_ns > 250000000ull ? limit_ns : 250000000ull;
}

// Generic-proxy shared-memory writes -> visible to the async proxy
// (tensor-core operand reads).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------- tcgen05
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, kind::i8 (s8 x s8 -> s32).
__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// D[tmem] (+)= A * B^T, kind::f16 (bf16/f16 inputs, f32 accumulate).
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// D[tmem] (+)= A * B^T, kind::f8f6f4 (e4m3 inputs here, f32 accumulate).
__device__ __forceinline__ void umma_f8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` once all previously issued tcgen05.mma of this thread
// have completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 lanes x 32 bit, 16 consecutive columns per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------ descriptors
// UMMA shared-memory matrix descriptor for a K-major operand in the
// 128-byte-swizzle canonical layout: 8-row x 128-byte atoms (1024 B), atoms
// stacked along M/N at `sbo` bytes.  Fields: start>>4 [0,14), LBO>>4
// [16,30) (unused for swizzled K-major, set to 1), SBO>>4 [32,46),
// version=1 [46,48), base offset 0 [49,52), layout SWIZZLE_128B=2 [61,64).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// The same for a K-major SWIZZLE_64B tile (64-byte rows, 8-row atoms of
// 512 bytes, atom stride sbo); layout type 4.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)4u << 61;
  return d;
}

// Instruction descriptor: c_format [4,6) (1=F32, 2=S32), a_format [7,10),
// b_format [10,13), a/b major [15],[16] (0 = K-major), N>>3 [17,23),
// M>>4 [24,29).
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t cfmt, uint32_t afmt, uint32_t bfmt,
                                                  uint32_t M, uint32_t N) {
  return (cfmt << 4) | (afmt << 7) | (bfmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Byte offset of 16-byte chunk `chunk` of row `row` inside a K-major
// SWIZZLE_128B tile whose base is 1024-byte aligned (rows of 128 bytes).
__device__ __forceinline__ uint32_t sw128_offset(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + (((chunk ^ (row & 7u)) & 7u) << 4);
}

// Byte offset of 16-byte chunk `chunk` (0..3) of row `row` inside a K-major
// SWIZZLE_64B tile whose base is 512-byte aligned (rows of 64 bytes): the
// chunk index is XORed with bits 7-8 of the row's byte offset.
__device__ __forceinline__ uint32_t sw64_offset(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 512u + (row & 7u) * 64u + (((chunk ^ (row >> 1)) & 3u) << 4);
}

__device__ __forceinline__ void st_shared_v4(uint32_t saddr, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(saddr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}

}  // namespace dsax

namespace dsax {

// ------------------------------------------------------------ bulk copies
// Arms `bar` for `bytes` of transaction count (one arrival).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// Non-tensor bulk copy global -> this CTA's shared memory (no multicast);
// completion is signalled on `bar` as transaction bytes.
__device__ __forceinline__ void bulk_g2s(uint32_t dst_smem, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst_smem),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 32 lanes x 32 bit, 32 consecutive columns per thread.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

// ---------------------------------------------------------------- tcgen05, CTA pairs
// cta_group::2: the two CTAs of a 2-CTA cluster share one MMA of M = 256
// (A rows 0-127 and D lanes in the even CTA, 128-255 in the odd one; B
// columns 0..N/2-1 from the even CTA's shared memory, N/2..N-1 from the
// odd one's, both at the same shared-memory offsets).  Every tcgen05
// instruction of such a kernel uses cta_group::2.
__device__ __forceinline__ void tmem_alloc_pair(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// D[tmem] (+)= A * B^T over the pair, kind::f16; issued by the even CTA.
__device__ __forceinline__ void umma_f16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                              uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// The same, kind::f8f6f4 (E4M3 operands here).
__device__ __forceinline__ void umma_f8_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// One arrival on the mbarrier at `bar`'s offset in each CTA of `cta_mask`
// once all previously issued pair MMAs of this thread have completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t *bar, uint16_t cta_mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
      "[%0], %1;" ::"r"(smem_u32(bar)),
      "h"(cta_mask)
      : "memory");
}

// ------------------------------------------------------------ clusters
// Rank of this CTA in its cluster.
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster (release / acquire).
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The shared::cluster address of this CTA's shared variable at `p` in CTA
// `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map(const void *p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ uint32_t cluster_map_u32(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
// One arrival on an mbarrier of another CTA of the cluster (release).
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar)
               : "memory");
}
// One arrival on an mbarrier of a CTA of the cluster with the default
// semantics (release at CTA scope, as the CTA-pair pipelines of the CUDA
// templates use): the producer's shared-memory writes are made visible to
// the tensor-core (async) proxy by fence.proxy.async before it.
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}
// Bulk copy from this CTA's shared memory into another CTA's of the cluster
// (no multicast), counted as transaction bytes on that CTA's mbarrier.
__device__ __forceinline__ void bulk_s2s_cluster(uint32_t cluster_dst, uint32_t src, uint32_t bytes,
                                                 uint32_t cluster_bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          cluster_dst),
      "r"(src), "r"(bytes), "r"(cluster_bar)
      : "memory");
}

// 2-D tiled TMA load (no multicast) into this CTA's shared memory,
// completing on `bar` with the box's byte count (`map`: a CUtensorMap).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled TMA load (no multicast) into this CTA's shared memory,
// completing on `bar` with the box's byte count.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void *map, int x, int y, int z,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Named barrier over `nthreads` threads (ids 1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_bar(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// 8 packed 4-bit two's-complement values (nibble 2i = real, 2i+1 = imag of
// element i) -> four words, word i = bf16(real_i) | bf16(imag_i) << 16.
// v + 8 (= nibble ^ 8, 0..15) placed in the mantissa of bf16(128) gives
// bf16(136 + v) exactly; one packed bf16 subtraction of 136 leaves v.
__device__ __forceinline__ void nib8_to_bf16x8(uint32_t x, uint32_t (&o)[4]) {
  const uint32_t xx = x ^ 0x88888888u;
  const uint32_t lo = xx & 0x0F0F0F0Fu;             // real parts + 8, byte i
  const uint32_t hi = (xx >> 4) & 0x0F0F0F0Fu;      // imaginary parts + 8, byte i
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t sel = (uint32_t)i | ((uint32_t)i << 4) | ((4u + i) << 8) | ((4u + i) << 12);
    const uint32_t w = (__byte_perm(lo, hi, sel) & 0x00FF00FFu) | 0x43004300u;
    asm("sub.rn.bf16x2 %0, %1, %2;" : "=r"(o[i]) : "r"(w), "r"(0x43084308u));
  }
}

}  // namespace dsax

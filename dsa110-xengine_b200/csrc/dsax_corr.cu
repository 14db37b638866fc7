// dsax_corr.cu -- the X-engine correlator on sm_100a tensor cores.
//
// Replaces, in one kernel, the reference's CPU reorder/fluff
// (src/dsaX_reorder_raw.c:153-169, src/dsaX_reorder_raw.c.bak:184-258), the
// xGPU-stage promoter (src/dsaX_xgpu.cu:67-77) and xgpuCudaXengine
// (src/dsaX_xgpu.cu:318; FP32 SIMT in the un-vendored xGPU library).
//
// Arithmetic.  For one frequency f' (= 2*chan + time-in-packet) and the 128
// inputs a = 2*station + pol, the products are
//     V[a][b] = sum_t x_a(t) conj(x_b(t)),   re = ra rb + ia ib,
//                                            im = ia rb - ra ib.
// With K = 2 * packets (k = 2p + {0: re, 1: im}) and the int8 operands
//     A[a][2p..2p+1]     = ( ra,  ia)
//     Arot[b][2p..2p+1]  = (-ib,  rb)
// one UMMA  D[128 x 256] = A * [A ; Arot]^T  yields Re V in columns 0..127
// and Im V in columns 128..255 (s32, exact).  The B operand is the
// concatenation of A and Arot in shared memory, so A is staged once.
//
// Tiling.  One CTA per channel = two frequencies (t = 0, 1); each frequency
// owns 256 TMEM columns (all 512 used).  K is streamed in stages of 64
// packets (128 bytes of K per row = one 128-byte swizzle atom).
//   warps 0-7 : producers -- load the packed 4-bit samples, unpack the
//               nibbles in registers and write the swizzled K-major A / Arot
//               tiles (the unpack never touches HBM);
//               after the K loop they are the epilogue (TMEM -> triangle).
//   warp  8   : TMEM allocator and single-thread UMMA issuer.
// Every pipeline wait is bounded (dsax_ptx.cuh).
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_ptx.cuh"

namespace dsax {

namespace corr {
constexpr int kPktPerStage = 64;                 // K bytes per row per stage = 128
constexpr int kStages = 3;
constexpr int kTileBytes = 128 * 128;            // 128 rows x 128 B
constexpr int kFreqBytes = 2 * kTileBytes;       // A + Arot
constexpr int kStageBytes = 2 * kFreqBytes;      // two frequencies
constexpr int kProducerThreads = 256;
constexpr int kThreads = kProducerThreads + 32;  // + MMA warp
constexpr int kSmemBytes = kStages * kStageBytes + 1024;  // + alignment slack
constexpr uint32_t kIdesc = umma_idesc(/*S32*/ 2, /*s8*/ 1, /*s8*/ 1, 128, 256);
}  // namespace corr

// 2 packed samples (bytes s of wa and wb) -> int8 [re_a, im_a, re_b, im_b].
__device__ __forceinline__ uint32_t unpack_pair(uint32_t wa, uint32_t wb, uint32_t s) {
  uint32_t x = __byte_perm(wa, wb, s | ((s + 4u) << 4));  // byte0 = wa.s, byte1 = wb.s
  uint32_t y = (x & 0x000Fu) | ((x & 0x00F0u) << 4) | ((x & 0x0F00u) << 8) |
               ((x & 0xF000u) << 12);
  return __vsub4(y ^ 0x08080808u, 0x08080808u);  // sign-extend each nibble
}

// [re_a, im_a, re_b, im_b] -> [-im_a, re_a, -im_b, re_b]
__device__ __forceinline__ uint32_t rotate_pair(uint32_t r) {
  uint32_t sw = __byte_perm(r, 0u, 0x2301u);
  uint32_t ng = __vneg4(sw);
  return (ng & 0x00FF00FFu) | (sw & 0xFF00FF00u);
}

// Loads the 8 packets of one (antenna, packet-group) task and returns, for
// each of the 4 (time, pol) sample slots, the packed byte quadruple words:
// w[q] holds, for packet q, bytes [t0p0, t0p1, t1p0, t1p1].
template <int FMT>
__device__ __forceinline__ void load_task(const CorrArgs &a, int ch, int ant, int p0,
                                          uint32_t (&w)[8], uint32_t (&v)[8]) {
  if (FMT == FMT_CAPTURED) {
    // [pkt][nant_in][nchan][2 t][2 pol] packed; one 32-bit word per (pkt, ant).
    const bool ok_ant = ant < a.nant_in;
    const uint8_t *base = a.in + ((int64_t)ant * a.nchan + ch) * 4;
    const int64_t pstride = (int64_t)a.nant_in * a.nchan * 4;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int p = p0 + q;
      w[q] = (ok_ant && p < a.npkt) ? __ldg(reinterpret_cast<const uint32_t *>(base + p * pstride))
                                    : 0u;
    }
  } else if (FMT == FMT_REORDERED) {
    // [pkt][2*nchan][64][2 pol] packed (the massage() output).
    const int64_t pstride = (int64_t)2 * a.nchan * 64 * 2;
    const uint8_t *base = a.in + ((int64_t)(2 * ch) * 64 + ant) * 2;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int p = p0 + q;
      uint32_t lo = 0, hi = 0;
      if (p < a.npkt) {
        lo = __ldg(reinterpret_cast<const uint16_t *>(base + p * pstride));
        hi = __ldg(reinterpret_cast<const uint16_t *>(base + p * pstride + 128));
      }
      w[q] = lo | (hi << 16);
    }
  } else {
    // FMT_XGPU_INT8: [pkt][nfreq][64][2 pol][re, im] int8 (xGPU ComplexInput).
    const int64_t pstride = (int64_t)2 * a.nchan * 64 * 4;
    const uint8_t *base = a.in + ((int64_t)(2 * ch) * 64 + ant) * 4;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int p = p0 + q;
      w[q] = p < a.npkt ? __ldg(reinterpret_cast<const uint32_t *>(base + p * pstride)) : 0u;
      v[q] = p < a.npkt ? __ldg(reinterpret_cast<const uint32_t *>(base + p * pstride + 256)) : 0u;
    }
  }
}

template <int FMT>
__global__ void __launch_bounds__(corr::kThreads, 1) corr_kernel(CorrArgs a) {
  using namespace corr;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t accum_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int ch = blockIdx.x;  // channel -> frequencies 2ch, 2ch+1

  // 1024-byte aligned stage area (required by the 128B swizzle atoms).
  const uint32_t smem_base = (smem_u32(smem_raw) + 1023u) & ~1023u;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], kProducerThreads);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&accum_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == 8) {
    tmem_alloc(&tmem_base_sh, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if ((tmem & 0xFFFFu) != 0u) {  // 512 columns must start at column 0
    if (tid == 0) { atomicOr(a.err, DEV_ERR_TMEM); }
    abort_sh = 1;
  }

  const int nks = (a.npkt + kPktPerStage - 1) / kPktPerStage;

  if (warp < 8) {
    // ------------------------------------------------------------ producers
    // lane -> (ant_lo, jbit, ant_hi); warp -> (ant group, packet-group pair)
    const int ant = 16 * (warp & 3) + 4 * (lane >> 3) + (lane & 3);
    const int jbit = (lane >> 2) & 1;
    for (int ks = 0; ks < nks && !abort_sh; ++ks) {
      const int s = ks % kStages;
      const uint32_t ph = (uint32_t)(ks / kStages) & 1u;
      if (!mbar_wait_bounded(&empty_bar[s], ph ^ 1u, &abort_sh, a.err, DEV_ERR_WAIT_EMPTY,
                             a.wait_limit_ns))
        break;
      const uint32_t stage = smem_base + (uint32_t)s * kStageBytes;
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int pg = 2 * ((warp >> 2) * 2 + it) + jbit;  // packet group 0..7
        uint32_t w[8], v[8];
        load_task<FMT>(a, ch, ant, ks * kPktPerStage + 8 * pg, w, v);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
#pragma unroll
          for (int pol = 0; pol < 2; ++pol) {
            uint32_t c[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
              if (FMT == FMT_XGPU_INT8) {
                const uint32_t wa = t ? v[2 * h] : w[2 * h];
                const uint32_t wb = t ? v[2 * h + 1] : w[2 * h + 1];
                const uint32_t sel = pol ? 0x7632u : 0x5410u;  // bytes (2pol, 2pol+1) of wa, wb
                c[h] = __byte_perm(wa, wb, sel);
              } else {
                c[h] = unpack_pair(w[2 * h], w[2 * h + 1], (uint32_t)(2 * t + pol));
              }
            }
            const uint32_t row = (uint32_t)(2 * ant + pol);
            const uint32_t off = sw128_offset(row, (uint32_t)pg);
            const uint32_t tileA = stage + (uint32_t)t * kFreqBytes;
            st_shared_v4(tileA + off, c[0], c[1], c[2], c[3]);
            st_shared_v4(tileA + kTileBytes + off, rotate_pair(c[0]), rotate_pair(c[1]),
                         rotate_pair(c[2]), rotate_pair(c[3]));
          }
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(&full_bar[s]);
    }
  } else {
    // ------------------------------------------------------------ UMMA issuer
    // One thread waits and issues; the other 31 lanes idle until the end.
    if (lane == 0) {
      for (int ks = 0; ks < nks && !abort_sh; ++ks) {
        const int s = ks % kStages;
        const uint32_t ph = (uint32_t)(ks / kStages) & 1u;
        if (!mbar_wait_bounded(&full_bar[s], ph, &abort_sh, a.err, DEV_ERR_WAIT_FULL,
                               a.wait_limit_ns))
          break;
        tc_fence_after();
        const uint32_t stage = smem_base + (uint32_t)s * kStageBytes;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const uint32_t tileA = stage + (uint32_t)t * kFreqBytes;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {  // 4 x K=32 bytes per 128-byte atom
            const uint64_t d = umma_desc_sw128(tileA + 32u * kk, 1024u);
            umma_i8(tmem + (uint32_t)t * 256u, d, d, kIdesc, (ks | kk) != 0);
          }
        }
        umma_commit(&empty_bar[s]);
      }
      umma_commit(&accum_bar);  // fires when every issued UMMA is done
    }
    __syncwarp();
  }

  // ---------------------------------------------------------------- epilogue
  if (warp < 8) {
    bool ok = mbar_wait_bounded(&accum_bar, 0u, &abort_sh, a.err, DEV_ERR_WAIT_ACCUM,
                                a.wait_limit_ns);
    tc_fence_after();
    // tcgen05.ld is .sync.aligned: the whole warp takes the same branch.
    ok = __all_sync(0xffffffffu, ok && !abort_sh);
    if (ok) {
      const int q = warp & 3;         // TMEM lane quarter of this warp
      const int t = warp >> 2;        // frequency within the channel
      const int m = 32 * q + lane;    // row = 2*station + pol
      const int i = m >> 1, pi = m & 1;
      float *vis = a.vis + (int64_t)(2 * ch + t) * (2080 * 8);
      const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)t * 256u;
      const int ncb = 2 * q + 2;      // station chunks of 8 reaching this warp's diagonal
      for (int cb = 0; cb < ncb; ++cb) {
        uint32_t re[16], im[16];
        tmem_ld16(trow + 16u * cb, re);
        tmem_ld16(trow + 128u + 16u * cb, im);
        tmem_wait_ld();
        const int64_t tri = (int64_t)i * (i + 1) / 2;
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int j = 8 * cb + jj;
          if (j <= i) {
            float4 o = make_float4((float)(int32_t)re[2 * jj], (float)(int32_t)im[2 * jj],
                                   (float)(int32_t)re[2 * jj + 1], (float)(int32_t)im[2 * jj + 1]);
            float4 *dst = reinterpret_cast<float4 *>(vis + ((tri + j) * 4 + 2 * pi) * 2);
            if (a.accumulate) {
              float4 old = *dst;
              o.x += old.x; o.y += old.y; o.z += old.z; o.w += old.w;
            }
            *dst = o;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    // Never free TMEM under an in-flight UMMA: wait for the final commit
    // (bounded, and independent of the abort flag).
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&accum_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------
// Channel-major correlator.  Input [nchan][npkt][64 ant][4 B] (one contiguous
// stream per channel, written by reorder_cm_kernel).
//
// Arithmetic without negated operands: with R, I the int8 real and
// imaginary parts (rows = 2*station + pol, K = packets),
//     Re V = R R^T + I I^T,   C = I R^T,   Im V[a][b] = C[a][b] - C[b][a].
// Three M128 N128 UMMAs per K step (25 % less tensor work than one M128
// N256 product with a rotated copy), C transposed in the epilogue through
// shared memory.
//
// Stage = 128 packets.  The loader warp bulk-copies each packet's 256 B
// into a raw row of 272 B (the 16-byte pad makes the unpack reads bank-
// conflict free).  A thread unpacks 8 packets P = pg + 16 q of one antenna:
// K position k(P) = 8 (P mod 16) + P / 16 puts them in 8 consecutive bytes
// of the R and I rows (K order is a free permutation shared by A and B).
namespace corrcm {
constexpr int kPktPerStage = 128;
constexpr int kRawRow = 272;                     // bytes per packet row in shared memory
constexpr int kRawBytes = kPktPerStage * kRawRow;  // 34,816
constexpr int kRawStages = 2;
constexpr int kTile = 128 * 128;                 // 128 rows x 128 B of K
constexpr int kFreqBytes = 2 * kTile;            // R + I
constexpr int kStageBytes = 2 * kFreqBytes;      // two frequencies
constexpr int kOpStages = 2;
constexpr int kThreads = 320;                    // 8 unpack/epilogue warps + UMMA warp + loader warp
constexpr int kSmemBytes = 1024 + kOpStages * kStageBytes + kRawStages * kRawBytes;
constexpr uint32_t kIdesc = umma_idesc(/*S32*/ 2, /*s8*/ 1, /*s8*/ 1, 128, 128);
}  // namespace corrcm

// Sign-extend the low nibble of each byte: v | (bit3 ? 0xF0 : 0).
__device__ __forceinline__ uint32_t sext_nib4(uint32_t v) {
  return v | ((v & 0x08080808u) * 0x1Eu);
}

__global__ void __launch_bounds__(corrcm::kThreads, 1) corr_cm_kernel(CorrArgs a) {
  using namespace corrcm;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kOpStages];
  __shared__ __align__(8) uint64_t empty_bar[kOpStages];
  __shared__ __align__(8) uint64_t rfull_bar[kRawStages];
  __shared__ __align__(8) uint64_t rempty_bar[kRawStages];
  __shared__ __align__(8) uint64_t accum_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ch = blockIdx.x;
  const uint32_t sbase = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t raw_base = sbase + kOpStages * kStageBytes;
  uint8_t *const gbase = smem_raw + (sbase - smem_u32(smem_raw));   // generic view of sbase

  if (tid == 0) {
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&full_bar[s], 256);
      mbar_init(&empty_bar[s], 1);
    }
    for (int r = 0; r < kRawStages; ++r) {
      mbar_init(&rfull_bar[r], 1);
      mbar_init(&rempty_bar[r], 256);
    }
    mbar_init(&accum_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == 8) {
    tmem_alloc(&tmem_base_sh, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if ((tmem & 0xFFFFu) != 0u) {
    if (tid == 0) atomicOr(a.err, DEV_ERR_TMEM);
    abort_sh = 1;
  }
  const int nks = (a.npkt + kPktPerStage - 1) / kPktPerStage;
  const uint8_t *chan_src = a.in + (int64_t)ch * a.npkt * 256;

  if (warp < 8) {
    // ------------------------------------------------------------ unpack
    const int ant_lo = lane & 3, pg_lo = lane >> 2;
    for (int ks = 0; ks < nks && !abort_sh; ++ks) {
      const int s = ks % kOpStages, r = ks % kRawStages;
      if (!mbar_wait_bounded(&rfull_bar[r], (uint32_t)(ks / kRawStages) & 1u, &abort_sh, a.err,
                             DEV_ERR_WAIT_FULL, a.wait_limit_ns))
        break;
      if (!mbar_wait_bounded(&empty_bar[s], ((uint32_t)(ks / kOpStages) & 1u) ^ 1u, &abort_sh,
                             a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
        break;
      const uint32_t *rw = reinterpret_cast<const uint32_t *>(gbase + kOpStages * kStageBytes +
                                                              r * kRawBytes);
      const uint32_t stage = sbase + (uint32_t)s * kStageBytes;
      const int pvalid = a.npkt - ks * kPktPerStage;   // packets of this stage that exist
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int pg = pg_lo + 8 * (it & 1);
        const int ant = 4 * (2 * warp + (it >> 1)) + ant_lo;
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int P = pg + 16 * q;
          w[q] = P < pvalid ? rw[P * (kRawRow / 4) + ant] : 0u;
        }
        // 4x4 byte transposes: X[sl][h] = sample slot sl (= 2t + pol) of
        // packets q = 4h .. 4h+3
        uint32_t X[4][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t t0 = __byte_perm(w[4 * h], w[4 * h + 1], 0x5140u);
          const uint32_t t1 = __byte_perm(w[4 * h], w[4 * h + 1], 0x7362u);
          const uint32_t t2 = __byte_perm(w[4 * h + 2], w[4 * h + 3], 0x5140u);
          const uint32_t t3 = __byte_perm(w[4 * h + 2], w[4 * h + 3], 0x7362u);
          X[0][h] = __byte_perm(t0, t2, 0x5410u);
          X[1][h] = __byte_perm(t0, t2, 0x7632u);
          X[2][h] = __byte_perm(t1, t3, 0x5410u);
          X[3][h] = __byte_perm(t1, t3, 0x7632u);
        }
#pragma unroll
        for (int sl = 0; sl < 4; ++sl) {
          const int t = sl >> 1, pol = sl & 1;
          const uint32_t re0 = sext_nib4(X[sl][0] & 0x0F0F0F0Fu);
          const uint32_t re1 = sext_nib4(X[sl][1] & 0x0F0F0F0Fu);
          const uint32_t im0 = sext_nib4((X[sl][0] >> 4) & 0x0F0F0F0Fu);
          const uint32_t im1 = sext_nib4((X[sl][1] >> 4) & 0x0F0F0F0Fu);
          const uint32_t row = (uint32_t)(2 * ant + pol);
          const uint32_t off = sw128_offset(row, (uint32_t)(pg >> 1)) + 8u * (pg & 1);
          const uint32_t tR = stage + (uint32_t)t * kFreqBytes;
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(tR + off), "r"(re0), "r"(re1)
                       : "memory");
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(tR + kTile + off), "r"(im0),
                       "r"(im1)
                       : "memory");
        }
      }
      mbar_arrive(&rempty_bar[r]);
      fence_proxy_async_smem();
      mbar_arrive(&full_bar[s]);
    }
  } else if (warp == 9) {
    // ------------------------------------------------------------ bulk loader
    if (lane == 0) {
      for (int ks = 0; ks < nks && !abort_sh; ++ks) {
        const int r = ks % kRawStages;
        if (!mbar_wait_bounded(&rempty_bar[r], ((uint32_t)(ks / kRawStages) & 1u) ^ 1u, &abort_sh,
                               a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        const int npk = min(kPktPerStage, a.npkt - ks * kPktPerStage);
        mbar_arrive_expect_tx(&rfull_bar[r], (uint32_t)npk * 256u);
        const uint8_t *src = chan_src + (int64_t)ks * kPktPerStage * 256;
        const uint32_t dst = raw_base + (uint32_t)r * kRawBytes;
        for (int p = 0; p < npk; ++p)
          bulk_g2s(dst + (uint32_t)p * kRawRow, src + (int64_t)p * 256, 256u, &rfull_bar[r]);
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ UMMA issuer
    if (lane == 0) {
      for (int ks = 0; ks < nks && !abort_sh; ++ks) {
        const int s = ks % kOpStages;
        if (!mbar_wait_bounded(&full_bar[s], (uint32_t)(ks / kOpStages) & 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_FULL, a.wait_limit_ns))
          break;
        tc_fence_after();
        const uint32_t stage = sbase + (uint32_t)s * kStageBytes;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const uint32_t tR = stage + (uint32_t)t * kFreqBytes, tI = tR + kTile;
          const uint32_t dre = tmem + (uint32_t)t * 256u, dc = dre + 128u;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {   // 4 x K = 32 bytes per 128-byte row
            const uint64_t dR = umma_desc_sw128(tR + 32u * kk, 1024u);
            const uint64_t dI = umma_desc_sw128(tI + 32u * kk, 1024u);
            umma_i8(dre, dR, dR, kIdesc, (ks | kk) != 0);   // Re += R R^T
            umma_i8(dre, dI, dI, kIdesc, 1u);               // Re += I I^T
            umma_i8(dc, dI, dR, kIdesc, (ks | kk) != 0);    // C  += I R^T
          }
        }
        umma_commit(&empty_bar[s]);
      }
      umma_commit(&accum_bar);
    }
    __syncwarp();
  }

  // ---------------------------------------------------------------- epilogue
  if (warp < 8) {
    bool ok = mbar_wait_bounded(&accum_bar, 0u, &abort_sh, a.err, DEV_ERR_WAIT_ACCUM,
                                a.wait_limit_ns);
    tc_fence_after();
    ok = __all_sync(0xffffffffu, ok && !abort_sh);
    const int q = warp & 3, t = warp >> 2;
    const int m = 32 * q + lane;                   // row = 2 * station + pol
    const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)t * 256u;
    // C^T through shared memory (operand stage t is free now): row m of C
    // stored at word (b ^ (m & 31)) of a 512-byte row.
    uint32_t *Cs = reinterpret_cast<uint32_t *>(gbase + t * kStageBytes);
    if (ok) {
#pragma unroll
      for (int cb = 0; cb < 8; ++cb) {
        uint32_t cv[16];
        tmem_ld16(trow + 128u + 16u * cb, cv);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 16; ++e) Cs[m * 128 + ((16 * cb + e) ^ lane)] = cv[e];
      }
    }
    named_bar(1, 256);
    if (ok) {
      const int i = m >> 1, pi = m & 1;
      float *vis = a.vis + (int64_t)(2 * ch + t) * (2080 * 8);
      const int64_t tri = (int64_t)i * (i + 1) / 2;
      const int ncb = 2 * q + 2;
      for (int cb = 0; cb < ncb; ++cb) {
        uint32_t re[16], cr[16];
        tmem_ld16(trow + 16u * cb, re);
        tmem_ld16(trow + 128u + 16u * cb, cr);
        tmem_wait_ld();
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int j = 8 * cb + jj;
          if (j <= i) {
            const int b0 = 2 * j, b1 = 2 * j + 1;
            const int32_t ct0 = (int32_t)Cs[b0 * 128 + (m ^ (b0 & 31))];
            const int32_t ct1 = (int32_t)Cs[b1 * 128 + (m ^ (b1 & 31))];
            float4 o = make_float4((float)(int32_t)re[2 * jj], (float)((int32_t)cr[2 * jj] - ct0),
                                   (float)(int32_t)re[2 * jj + 1],
                                   (float)((int32_t)cr[2 * jj + 1] - ct1));
            float4 *dst = reinterpret_cast<float4 *>(vis + ((tri + j) * 4 + 2 * pi) * 2);
            if (a.accumulate) {
              const float4 old = *dst;
              o.x += old.x; o.y += old.y; o.z += old.z; o.w += old.w;
            }
            *dst = o;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&accum_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

int launch_correlate_chanmajor(const CorrArgs &a, cudaStream_t st) {
  static bool attr_done = false;
  if (!attr_done) {
    if (cudaFuncSetAttribute(corr_cm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             corrcm::kSmemBytes) != cudaSuccess)
      return -2;
    attr_done = true;
  }
  void *args[] = {(void *)&a};
  return cudaLaunchKernel((const void *)corr_cm_kernel, dim3(a.nchan), dim3(corrcm::kThreads), args,
                          corrcm::kSmemBytes, st) == cudaSuccess
             ? 0
             : -2;
}

int launch_correlate(const CorrArgs &a, int fmt, cudaStream_t st) {
  static bool attr_done[3] = {false, false, false};
  const void *fn = fmt == FMT_CAPTURED    ? (const void *)corr_kernel<FMT_CAPTURED>
                   : fmt == FMT_REORDERED ? (const void *)corr_kernel<FMT_REORDERED>
                                          : (const void *)corr_kernel<FMT_XGPU_INT8>;
  if (fmt < 0 || fmt > 2) return -1;
  if (!attr_done[fmt]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         corr::kSmemBytes);
    if (e != cudaSuccess) return -2;
    attr_done[fmt] = true;
  }
  dim3 grid(a.nchan), block(corr::kThreads);
  void *args[] = {(void *)&a};
  cudaError_t e = cudaLaunchKernel(fn, grid, block, args, corr::kSmemBytes, st);
  return e == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

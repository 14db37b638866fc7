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
// Same product as corr_kernel -- D[128 x 256] = A [A ; Arot]^T per 32-byte
// K step, Re in columns 0..127, Im in 128..255 -- with K laid out per 64-
// packet stage as [64 real parts | 64 imaginary parts]:
//     A row    = [ R  | I ]        Arot row = [ -I | R ]
// Packet P of the stage sits at K byte k(P) = 8 (P mod 8) + P / 8 (a free
// permutation: A and B share it), so the 16 packets P = 2c + e + 8q
// (e = 0, 1; q = 0..7) fill 16-byte chunk c of the real half and chunk
// c + 4 of the imaginary half.  Thread (antenna, c) reads those 16 words
// (lanes = consecutive antennas: conflict-free), transposes bytes, and
// sign-extends / negates nibbles with SWAR arithmetic.  Lanes 4..7 of each
// group of 8 store the two pols in the opposite order, so every 16-byte
// store instruction covers all eight bank groups of the 128-byte swizzle.
// One loader thread brings each 64-packet stage (16 KB, contiguous) in with
// a single bulk copy, four stages ahead.
namespace corrcm {
constexpr int kPktPerStage = 64;
constexpr int kRawBytes = kPktPerStage * 256;      // 16 KB
constexpr int kRawStages = 4;
constexpr int kTile = 128 * 128;                   // 128 rows x 128 B of K
constexpr int kFreqBytes = 2 * kTile;              // A + Arot
constexpr int kStageBytes = 2 * kFreqBytes;        // two frequencies
constexpr int kOpStages = 2;
constexpr int kThreads = 320;                      // 8 unpack/epilogue warps + UMMA warp + loader warp
constexpr int kSmemBytes = 1024 + kOpStages * kStageBytes + kRawStages * kRawBytes;
}  // namespace corrcm

// Low nibble of each byte (0..15) -> sign-extended int8: v | (bit3 ? 0xF0 : 0).
__device__ __forceinline__ uint32_t sext_nib4(uint32_t v) {
  return v | ((v & 0x08080808u) * 0x1Eu);
}

// Bytewise two's-complement negation (no carries between bytes); exact for
// bytes in [-8, 7].
__device__ __forceinline__ uint32_t neg_bytes(uint32_t x) {
  const uint32_t t = (~x & 0x7F7F7F7Fu) + 0x01010101u;
  return t ^ (~x & 0x80808080u);
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
  const uint8_t *raw_gen = smem_raw + (raw_base - smem_u32(smem_raw));   // generic view

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
    const int ant = lane + 32 * (warp & 1);
    const uint32_t c = (uint32_t)(warp >> 1);          // K chunk of the real half (0..3)
    const uint32_t flip = (uint32_t)(lane >> 2) & 1u;  // store pol 1 first
    for (int ks = 0; ks < nks && !abort_sh; ++ks) {
      const int s = ks % kOpStages, r = ks % kRawStages;
      if (!mbar_wait_bounded(&rfull_bar[r], (uint32_t)(ks / kRawStages) & 1u, &abort_sh, a.err,
                             DEV_ERR_WAIT_FULL, a.wait_limit_ns))
        break;
      if (!mbar_wait_bounded(&empty_bar[s], ((uint32_t)(ks / kOpStages) & 1u) ^ 1u, &abort_sh,
                             a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
        break;
      const uint32_t *rw = reinterpret_cast<const uint32_t *>(raw_gen + r * kRawBytes);
      const int pvalid = a.npkt - ks * kPktPerStage;   // packets of this stage that exist
      // w[e][q]: packet 2c + e + 8q, word = bytes [t0p0, t0p1, t1p0, t1p1]
      uint32_t w[2][8];
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int P = 2 * (int)c + e + 8 * q;
          w[e][q] = P < pvalid ? rw[P * 64 + ant] : 0u;
        }
      mbar_arrive(&rempty_bar[r]);   // raw stage consumed (generic-proxy reads only)
      // X[sl][e][h]: sample slot sl = 2t + pol of packets q = 4h .. 4h+3
      uint32_t X[4][2][2];
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t *v = &w[e][4 * h];
          const uint32_t t0 = __byte_perm(v[0], v[1], 0x5140u);
          const uint32_t t1 = __byte_perm(v[0], v[1], 0x7362u);
          const uint32_t t2 = __byte_perm(v[2], v[3], 0x5140u);
          const uint32_t t3 = __byte_perm(v[2], v[3], 0x7362u);
          X[0][e][h] = __byte_perm(t0, t2, 0x5410u);
          X[1][e][h] = __byte_perm(t0, t2, 0x7632u);
          X[2][e][h] = __byte_perm(t1, t3, 0x5410u);
          X[3][e][h] = __byte_perm(t1, t3, 0x7632u);
        }
      const uint32_t stage = sbase + (uint32_t)s * kStageBytes;
#pragma unroll
      for (int t = 0; t < 2; ++t) {
#pragma unroll
        for (int sp = 0; sp < 2; ++sp) {
          const uint32_t pol = (uint32_t)sp ^ flip;
          uint32_t re[4], im[4], ni[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {   // chunk word k = (e, h) = (k >> 1, k & 1)
            const uint32_t x0 = X[2 * t][k >> 1][k & 1], x1 = X[2 * t + 1][k >> 1][k & 1];
            const uint32_t x = pol ? x1 : x0;
            re[k] = sext_nib4(x & 0x0F0F0F0Fu);
            im[k] = sext_nib4((x >> 4) & 0x0F0F0F0Fu);
            ni[k] = neg_bytes(im[k]);
          }
          const uint32_t row = (uint32_t)(2 * ant) + pol;
          const uint32_t tA = stage + (uint32_t)t * kFreqBytes, tB = tA + kTile;
          const uint32_t o_re = sw128_offset(row, c), o_im = sw128_offset(row, c + 4u);
          st_shared_v4(tA + o_re, re[0], re[1], re[2], re[3]);
          st_shared_v4(tA + o_im, im[0], im[1], im[2], im[3]);
          st_shared_v4(tB + o_re, ni[0], ni[1], ni[2], ni[3]);
          st_shared_v4(tB + o_im, re[0], re[1], re[2], re[3]);
        }
      }
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
        const uint32_t bytes = (uint32_t)npk * 256u;
        mbar_arrive_expect_tx(&rfull_bar[r], bytes);
        bulk_g2s(raw_base + (uint32_t)r * kRawBytes, chan_src + (int64_t)ks * kPktPerStage * 256,
                 bytes, &rfull_bar[r]);
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
          const uint32_t tA = stage + (uint32_t)t * kFreqBytes;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {   // 4 x K = 32 bytes per 128-byte row
            const uint64_t d = umma_desc_sw128(tA + 32u * kk, 1024u);
            umma_i8(tmem + (uint32_t)t * 256u, d, d, corr::kIdesc, (ks | kk) != 0);
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
    if (ok) {
      const int q = warp & 3, t = warp >> 2;
      const int m = 32 * q + lane;
      const int i = m >> 1, pi = m & 1;
      float *vis = a.vis + (int64_t)(2 * ch + t) * (2080 * 8);
      const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)t * 256u;
      const int ncb = 2 * q + 2;
      const int64_t tri = (int64_t)i * (i + 1) / 2;
      for (int cb = 0; cb < ncb; ++cb) {
        uint32_t re[16], im[16];
        tmem_ld16(trow + 16u * cb, re);
        tmem_ld16(trow + 128u + 16u * cb, im);
        tmem_wait_ld();
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const int j = 8 * cb + jj;
          if (j <= i) {
            float4 o = make_float4((float)(int32_t)re[2 * jj], (float)(int32_t)im[2 * jj],
                                   (float)(int32_t)re[2 * jj + 1], (float)(int32_t)im[2 * jj + 1]);
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

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
#include <cuda.h>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_ptx.cuh"
#include "dsax_tmap.h"

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
      mbar_wait_bounded(&accum_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, drain_limit(a.wait_limit_ns));
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
// Per 64-packet stage and time slot t, two K-major SWIZZLE_64B operand
// tiles of 128 rows (2 ant + pol) x 64 bytes, R then I (8 KB each, so that
// [R; I] is one 256-row operand), with packet P at K byte 8 (P mod 8) + P / 8
// (a permutation shared by every operand).  Two MMA groups per slot:
//     R [R; I]^T   (N = 256, K = 64)  -> R R^T | R I^T   TMEM cols t*256 + [0, 256)
//     I I^T        (N = 128, K = 64)  += into cols t*256 + [0, 128)
// so cols [0, 128) hold Re = R R^T + I I^T and cols [128, 256) hold
// E = R I^T = C^T for C = I R^T; the epilogue forms Im = C - C^T from E and
// its transpose (through shared memory).  The tensor time equals one N = 128
// group per 32 bytes of K; the operand reads are 80 KB per stage (a single
// [R | I] tile with Re = A A^T and C = I R^T as four and two N = 128 MMAs
// read 96 KB).
// Thread (antenna, c) owns the 16 packets P = 2c + e + 8q (e = 0, 1;
// q = 0..7), i.e. 16-byte chunk c of the R and of the I tile.  Its 16 words come either
// straight from global memory (kBulk = false: lanes = consecutive
// antennas, coalesced, two stages ahead in registers) or from 16 KB stages
// that a loader warp brings in with one cp.async.bulk each, four ahead
// (kBulk = true; conflict-free shared reads).  It transposes bytes with
// prmt and sign-extends nibbles with carry-free bytewise adds.  Lanes 4..7 of each group of 8
// store the two pols in the opposite order, so every 16-byte store
// instruction covers all eight bank groups (the 64-byte swizzle spreads
// four consecutive antennas' chunks over four groups, the pol the other
// four).
// Persistent (FEED 0 / 1): one CTA per SM, each correlating channels
// blockIdx.x, + gridDim.x, ...; the raw and operand rings and their
// barrier phases run on across a CTA's channels, so the loader brings the
// next channel's first stages in while the unpack warps run this channel's
// epilogue, and TMEM, barriers and the pipeline are set up once per SM
// instead of once per channel.  The next channel's MMAs overwrite the
// accumulators only after every unpack warp has left the epilogue (named
// barrier, then its first stage's full barrier).
// Epilogue balance: the lower triangle in 16 x 16 antenna blocks (I, J) is
// written by TMEM lane quadrant I, except block (3, 0), which quadrant 0
// writes as the conjugates of its own rows, so that no warp writes more
// than three blocks (four before).
// NW = 16 (bulk-fed only) doubles the unpack warps: warps 8..15 repeat the
// mapping of warps 0..7 for time slot 1 while warps 0..7 take slot 0 (each
// raw word is read twice, each thread does half the byte work), and the
// epilogue splits every warp's column blocks between the two halves.
//
// Feeds (FEED): 0 direct loads and 1 one bulk copy per stage, both from the
// channel-major corner turn; 2 the captured block itself, with no corner
// turn.  FEED 2 runs in clusters of four CTAs, the four channels of one
// 16-byte row of the captured layout.  Per 64-packet stage, CTA r of the
// cluster loads one TMA box [16 packets][nant_in antennas][16 bytes]
// (packets 16r..16r+15 of the stage, all four channels; rows past the
// block read zero) into a landing slot.  Two transposer warps read the box
// into registers and write it back in place split by channel, [channel q]
// [16 packets][64 antennas][4 bytes] (antenna 63 zero), and one thread
// sends each 4 KB piece to channel q's CTA with one shared-to-shared bulk
// copy, counted as transaction bytes on that CTA's raw-full mbarrier.  Each
// CTA's raw stage thus receives 4 KB from each of the four CTAs in the same
// [64 packets][64 antennas][4 bytes] layout as the bulk feed, and the
// unpack, UMMA and epilogue are those of FEED 1.  A raw slot is re-armed,
// and the four sources told that it is free (remote mbarrier arrivals), once
// the unpack warps have read it; a source loads the next box into its
// landing slot only when every destination has consumed the slot's previous
// round, which also means its bulk copies out of that landing slot are done.
// Every HBM byte of the block is read once and crosses the SM-to-SM network
// at most once, in 4 KB copies; no multicast is used.  (Sixteen-byte remote
// stores with per-store transaction counts ran at about 4 GB/s per SM.)
namespace corrcm {
constexpr int kPktPerStage = 64;
constexpr int kTile = 128 * 128;                   // 128 rows x 128 B of K
constexpr int kStageBytes = 2 * kTile;             // two time slots
constexpr int kOpStages = 4;
constexpr int kRawBytes = kPktPerStage * 256;      // bulk-fed variant: one 16 KB stage
constexpr int kClusterCh = 4;                      // FEED 2: channels (CTAs) per cluster
constexpr int kLandPkts = kPktPerStage / kClusterCh;   // packets of a TMA box
constexpr int kLandBytes = kLandPkts * 64 * 16;    // a landing slot (box <= 64 antennas)
static_assert(kLandBytes == kClusterCh * kLandPkts * 64 * 4, "landing slot holds the split box");
// raw stages: 4 for the bulk feed; 3 for FEED 2, which also keeps one
// landing slot per raw stage
template <int FEED> constexpr int raw_stages() { return FEED == 2 ? 3 : 4; }
// NW unpack/epilogue warps + UMMA warp (+ bulk loader warp for FEED 1; TMA
// warp, raw-slot manager warp and two transposer warps for FEED 2)
template <int FEED, int NW> constexpr int threads() {
  return 32 * NW + 32 + (FEED == 1 ? 32 : FEED == 2 ? 128 : 0);
}
template <int FEED> constexpr int smem_bytes() {
  return 1024 + kOpStages * kStageBytes + (FEED >= 1 ? raw_stages<FEED>() * kRawBytes : 0) +
         (FEED == 2 ? raw_stages<FEED>() * kLandBytes : 0);
}
constexpr uint32_t kIdescN128 = umma_idesc(/*S32*/ 2, /*s8*/ 1, /*s8*/ 1, 128, 128);
constexpr uint32_t kIdescN256 = umma_idesc(/*S32*/ 2, /*s8*/ 1, /*s8*/ 1, 128, 256);
constexpr uint32_t kHalfTile = 128 * 64;           // one 64-byte-row tile (R or I)
static_assert(kOpStages * kStageBytes >= 2 * 128 * 128 * 4, "C^T scratch reuses the stages");
}  // namespace corrcm

// Low / high nibble of each byte (4-bit two's complement) -> int8, bytewise
// without carries: x = nibble ^ 8 = v + 8 in [0, 15]; (x + 0x78) ^ 0x80 = v.
__device__ __forceinline__ uint32_t sext_lo4(uint32_t w) {
  return (((w & 0x0F0F0F0Fu) ^ 0x08080808u) + 0x78787878u) ^ 0x80808080u;
}
__device__ __forceinline__ uint32_t sext_hi4(uint32_t w) {
  return ((((w >> 4) & 0x0F0F0F0Fu) ^ 0x08080808u) + 0x78787878u) ^ 0x80808080u;
}

template <int FEED, int NW>
__global__ void __launch_bounds__(corrcm::threads<FEED, NW>(), 1)
    corr_cm_kernel(const __grid_constant__ CUtensorMap tmap, CorrArgs a) {
  using namespace corrcm;
  constexpr bool kBulk = FEED >= 1;   // unpack from raw stages in shared memory
  constexpr bool kCl = FEED == 2;
  constexpr int kRawStages = raw_stages<FEED>();
  static_assert(NW == 8 || (NW == 16 && kBulk), "8 unpack warps, or 16 when stage-fed");
  constexpr int kUnpackThreads = 32 * NW;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kOpStages];
  __shared__ __align__(8) uint64_t empty_bar[kOpStages];
  __shared__ __align__(8) uint64_t rfull_bar[kRawStages];
  __shared__ __align__(8) uint64_t rempty_bar[kRawStages];
  __shared__ __align__(8) uint64_t accum_bar;            // a channel's accumulators complete
  __shared__ __align__(8) uint64_t final_bar;            // every MMA of the CTA complete
  __shared__ __align__(8) uint64_t land_full[kRawStages]; // FEED 2: TMA box landed
  __shared__ __align__(8) uint64_t dest_free[kRawStages]; // FEED 2: slot consumed in all 4 CTAs
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ch = blockIdx.x;   // FEED 2: the CTA's channel
  // FEED 0 / 1: channels blockIdx.x, + gridDim.x, ... (a grid of fewer CTAs
  // than channels loops; the rings and barrier phases run on across the
  // channels, stage G = ci * nks + ks of channel ci); FEED 2: one channel
  const int nchc = kCl ? 1 : (a.nchan - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const uint32_t crank = kCl ? cluster_ctarank() : 0u;     // channel within the cluster's four
  const int nks = (a.npkt + kPktPerStage - 1) / kPktPerStage;
  const uint32_t sbase = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *const gbase = smem_raw + (sbase - smem_u32(smem_raw));   // generic view of sbase

  if (tid == 0) {
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&full_bar[s], kUnpackThreads);
      mbar_init(&empty_bar[s], 1);
    }
    for (int r = 0; r < kRawStages; ++r) {
      mbar_init(&rfull_bar[r], 1);
      mbar_init(&rempty_bar[r], kUnpackThreads);
    }
    mbar_init(&accum_bar, 1);
    mbar_init(&final_bar, 1);
    if (kCl) {
      for (int r = 0; r < kRawStages; ++r) {
        mbar_init(&land_full[r], 1);
        mbar_init(&dest_free[r], kClusterCh);
        // the first round of raw stages is armed here; the slot manager
        // re-arms each slot after the unpack has read it
        if (r < nks) mbar_arrive_expect_tx(&rfull_bar[r], kRawBytes);
      }
    }
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == NW) {
    tmem_alloc(&tmem_base_sh, 512);
    tmem_relinquish();
  }
  const uint32_t raw_base = sbase + kOpStages * kStageBytes;   // kBulk only
  tc_fence_before();
  __syncthreads();
  if (kCl) cluster_barrier();   // every CTA's barriers exist before any remote access
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if ((tmem & 0xFFFFu) != 0u) {
    if (tid == 0) atomicOr(a.err, DEV_ERR_TMEM);
    abort_sh = 1;
  }

  if (warp < NW) {
    // ------------------------------------------------------------ unpack
    const int ant = lane + 32 * (warp & 1);
    const uint32_t c = (uint32_t)((warp >> 1) & 3);    // 16-byte chunk of each half (0..3)
    const int tsel = warp >> 3;                        // NW = 16: the one time slot
    const uint32_t flip = (uint32_t)(lane >> 2) & 1u;  // store pol 1 first
    // tile offsets of this thread's chunks, store order sp = 0, 1 (pol = sp ^ flip)
    uint32_t o_re[2], o_im[2];
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) {
      const uint32_t row = (uint32_t)(2 * ant) + ((uint32_t)sp ^ flip);
      o_re[sp] = sw64_offset(row, c);
      o_im[sp] = kHalfTile + sw64_offset(row, c);
    }
    int gs0 = 0;                                       // stages of the earlier channels
    const uint32_t *chan_src = nullptr;                // FEED 0: the channel's stream
    // w[e][q]: packet 2c + e + 8q of the stage, word = bytes [t0p0, t0p1, t1p0, t1p1]
    auto load = [&](int ks, uint32_t (&w)[2][8]) {
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int p = ks * kPktPerStage + 2 * (int)c + e + 8 * q;
          w[e][q] = (ks < nks && p < a.npkt) ? __ldg(chan_src + (int64_t)p * 64 + ant) : 0u;
        }
    };
    auto unpack_store = [&](int ks, const uint32_t (&w)[2][8]) -> bool {
      const int G = gs0 + ks;
      const int s = G % kOpStages;
      if (!mbar_wait_bounded(&empty_bar[s], ((uint32_t)(G / kOpStages) & 1u) ^ 1u, &abort_sh,
                             a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
        return false;
      // X[sl][e][h]: sample slot sl = 2t + pol of packets q = 4h .. 4h+3
      // (NW = 16: only the slots of time slot tsel, at sl = 0, 1)
      uint32_t X[4][2][2];
      const uint32_t sel_t = tsel ? 0x7362u : 0x5140u;
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t *v = &w[e][4 * h];
          if (NW == 16) {
            const uint32_t ta = __byte_perm(v[0], v[1], sel_t);
            const uint32_t tb = __byte_perm(v[2], v[3], sel_t);
            X[0][e][h] = __byte_perm(ta, tb, 0x5410u);
            X[1][e][h] = __byte_perm(ta, tb, 0x7632u);
          } else {
            const uint32_t t0 = __byte_perm(v[0], v[1], 0x5140u);
            const uint32_t t1 = __byte_perm(v[0], v[1], 0x7362u);
            const uint32_t t2 = __byte_perm(v[2], v[3], 0x5140u);
            const uint32_t t3 = __byte_perm(v[2], v[3], 0x7362u);
            X[0][e][h] = __byte_perm(t0, t2, 0x5410u);
            X[1][e][h] = __byte_perm(t0, t2, 0x7632u);
            X[2][e][h] = __byte_perm(t1, t3, 0x5410u);
            X[3][e][h] = __byte_perm(t1, t3, 0x7632u);
          }
        }
      const uint32_t stage = sbase + (uint32_t)s * kStageBytes;
#pragma unroll
      for (int tt = 0; tt < (NW == 16 ? 1 : 2); ++tt) {
        const int t = NW == 16 ? tsel : tt;   // time slot (tile)
        const int xs = 2 * tt;                // its slots in X
#pragma unroll
        for (int sp = 0; sp < 2; ++sp) {
          const uint32_t pol = (uint32_t)sp ^ flip;
          uint32_t re[4], im[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {   // chunk word k = (e, h) = (k >> 1, k & 1)
            const uint32_t x0 = X[xs][k >> 1][k & 1], x1 = X[xs + 1][k >> 1][k & 1];
            const uint32_t x = pol ? x1 : x0;
            re[k] = sext_lo4(x);
            im[k] = sext_hi4(x);
          }
          const uint32_t tile = stage + (uint32_t)t * kTile;
          st_shared_v4(tile + o_re[sp], re[0], re[1], re[2], re[3]);
          st_shared_v4(tile + o_im[sp], im[0], im[1], im[2], im[3]);
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(&full_bar[s]);
      return true;
    };
    const uint32_t *rw_base = reinterpret_cast<const uint32_t *>(gbase + kOpStages * kStageBytes);
    // the words of raw stage ks -> w, then the stage goes back to the loader
    auto fetch = [&](int ks, uint32_t (&w)[2][8]) -> bool {
      const int G = gs0 + ks;
      const int r = G % kRawStages;
      if (!mbar_wait_bounded<kCl>(&rfull_bar[r], (uint32_t)(G / kRawStages) & 1u, &abort_sh,
                                  a.err, DEV_ERR_WAIT_FULL, a.wait_limit_ns))
        return false;
      const uint32_t *rw = rw_base + r * (kRawBytes / 4);
      const int pvalid = a.npkt - ks * kPktPerStage;
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int P = 2 * (int)c + e + 8 * q;
          w[e][q] = P < pvalid ? rw[P * 64 + ant] : 0u;
        }
      // The next bulk copy (async proxy) overwrites this stage: order these
      // generic-proxy reads before it, or under load the copy can land
      // first (a write-after-read race across proxies).
      fence_proxy_async_smem();
      mbar_arrive(&rempty_bar[r]);
      return true;
    };
#pragma unroll 1
    for (int ci = 0; ci < nchc; ++ci) {
      const int ch = (int)blockIdx.x + ci * (kCl ? 0 : (int)gridDim.x);
      gs0 = ci * nks;
      chan_src = reinterpret_cast<const uint32_t *>(a.in + (int64_t)ch * a.npkt * 256);
      if (kBulk) {
        // one stage of words in registers ahead of the stage being unpacked,
        // so the shared-memory loads overlap the previous stage's unpack
        uint32_t wa[2][8], wb[2][8];
        if (nks > 0 && fetch(0, wa)) {
          for (int ks = 0; ks < nks && !abort_sh; ks += 2) {
            if (ks + 1 < nks && !fetch(ks + 1, wb)) break;
            if (!unpack_store(ks, wa)) break;
            if (ks + 1 >= nks) break;
            if (ks + 2 < nks && !fetch(ks + 2, wa)) break;
            if (!unpack_store(ks + 1, wb)) break;
          }
        }
      } else {
        // two stages of loads in flight ahead of the stage being unpacked
        uint32_t wa[2][8], wb[2][8], wc[2][8];
        load(0, wa);
        load(1, wb);
        for (int ks = 0; ks < nks && !abort_sh; ks += 3) {
          load(ks + 2, wc);
          if (!unpack_store(ks, wa)) break;
          if (ks + 1 >= nks) break;
          load(ks + 3, wa);
          if (!unpack_store(ks + 1, wb)) break;
          if (ks + 2 >= nks) break;
          load(ks + 4, wb);
          if (!unpack_store(ks + 2, wc)) break;
        }
      }
      // ------------------------------------------------------------ epilogue
      bool ok = mbar_wait_bounded(&accum_bar, (uint32_t)ci & 1u, &abort_sh, a.err, DEV_ERR_WAIT_ACCUM,
                                  a.wait_limit_ns);
      tc_fence_after();
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      // TMEM lane quadrant q (warp % 4), time slot t; with NW = 16 the two
      // warps of each (q, t) take alternate column blocks (hh)
      constexpr int kCbStep = NW / 8;
      const int q = warp & 3, t = (warp >> 2) & 1, hh = warp >> 3;
      const int m = 32 * q + lane;                   // row = 2 * antenna + pol
      const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)t * 256u;
      // C^T through shared memory (every MMA has completed, so the operand
      // stages are free): row m of C at word (col ^ (m & 31)) of a 512-byte row.
      uint32_t *Cs = reinterpret_cast<uint32_t *>(gbase + t * (128 * 128 * 4));
      if (ok) {
#pragma unroll
        for (int cb = hh; cb < 8; cb += kCbStep) {
          uint32_t cv[16];
          tmem_ld16(trow + 128u + 16u * cb, cv);
          tmem_wait_ld();
#pragma unroll
          for (int e = 0; e < 16; ++e) Cs[m * 128 + ((16 * cb + e) ^ lane)] = cv[e];
        }
      }
      named_bar(1, kUnpackThreads);
      if (ok) {
        const int i = m >> 1, pi = m & 1;
        float *vis = a.vis + (int64_t)(2 * ch + t) * (2080 * 8);
        const int64_t tri = (int64_t)i * (i + 1) / 2;
        const int ncb = 2 * q + 2;
        // The triangle in 16 x 16 antenna blocks (I, J), I >= J: quadrant q
        // writes row block q, except that block (3, 0) goes to quadrant 0
        // as the conjugates of its own rows (V_ij = conj V_ji), so that no
        // warp does more than three blocks (48 column steps instead of 64
        // for quadrant 3).
        for (int cb = (q == 3 ? 2 : 0) + hh; cb < ncb; cb += kCbStep) {
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
              // cr = E[m][.] = C[.][m], ct = C[m][.]: Im = C[m][.] - C[.][m]
              float4 o = make_float4((float)(int32_t)re[2 * jj], (float)(ct0 - (int32_t)cr[2 * jj]),
                                     (float)(int32_t)re[2 * jj + 1],
                                     (float)(ct1 - (int32_t)cr[2 * jj + 1]));
              float4 *dst = reinterpret_cast<float4 *>(vis + ((tri + j) * 4 + 2 * pi) * 2);
              if (a.accumulate) {
                const float4 old = *dst;
                o.x += old.x; o.y += old.y; o.z += old.z; o.w += old.w;
              }
              *dst = o;
            }
          }
        }
        if (q == 0) {
          // block (3, 0) from rows m' = 2j + pj, j < 16: output (i, j) for
          // i = 48..63 is V_ij = conj V_ji, Re from Re[m'][2i + pi], Im =
          // E[m'][n] - E[n][m'] (n = 2i + pi); the two pols of j (lanes
          // 2j, 2j + 1) swap one value so that each writes one 16-byte pair
          const int j = m >> 1, pj = m & 1;
          for (int ib = hh; ib < 2; ib += kCbStep) {
            uint32_t re[16], er[16];
            tmem_ld16(trow + 96u + 16u * ib, re);
            tmem_ld16(trow + 128u + 96u + 16u * ib, er);
            tmem_wait_ld();
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
              const int ic = 48 + 8 * ib + ii;   // output row antenna i
              const int n0 = 2 * ic, n1 = 2 * ic + 1;
              const int32_t en0 = (int32_t)Cs[n0 * 128 + (m ^ (n0 & 31))];   // E[n0][m']
              const int32_t en1 = (int32_t)Cs[n1 * 128 + (m ^ (n1 & 31))];
              const float r0 = (float)(int32_t)re[2 * ii], i0 = (float)((int32_t)er[2 * ii] - en0);
              const float r1 = (float)(int32_t)re[2 * ii + 1],
                          i1 = (float)((int32_t)er[2 * ii + 1] - en1);
              // pj = 0 keeps pi = 0 and sends pi = 1; pj = 1 the reverse
              const float sr = __shfl_xor_sync(0xffffffffu, pj ? r0 : r1, 1);
              const float si = __shfl_xor_sync(0xffffffffu, pj ? i0 : i1, 1);
              float4 o = pj ? make_float4(sr, si, r1, i1) : make_float4(r0, i0, sr, si);
              const int64_t trc = (int64_t)ic * (ic + 1) / 2;
              float4 *dst = reinterpret_cast<float4 *>(vis + ((trc + j) * 4 + 2 * pj) * 2);
              if (a.accumulate) {
                const float4 old = *dst;
                o.x += old.x; o.y += old.y; o.z += old.z; o.w += old.w;
              }
              *dst = o;
            }
          }
        }
      }
      // every warp is done with this channel's accumulators and with the
      // C^T scratch (the operand stages) before the next channel's stages
      // are written and its MMAs issued
      if (ci + 1 < nchc) {
        tc_fence_before();
        named_bar(1, kUnpackThreads);
      }
    }
  } else if (kCl && warp == NW + 1) {
    // ------------------------------------------------------------ TMA loader (FEED 2)
    // Landing slot r is reloaded for stage ks only after all four CTAs have
    // consumed stage ks - R, i.e. after the bulk copies out of it landed.
    if (lane == 0) {
      const uint32_t land_bytes = (uint32_t)(kLandPkts * a.nant_in * 16);
      const uint32_t land_base = raw_base + kRawStages * kRawBytes;
      const int x0 = 4 * (ch - (int)crank);   // byte offset of the cluster's four channels
      int ks = 0;
      for (; ks < nks && !abort_sh; ++ks) {
        const int r = ks % kRawStages;
        if (ks >= kRawStages &&
            !mbar_wait_bounded<true>(&dest_free[r], (uint32_t)(ks / kRawStages - 1) & 1u, &abort_sh,
                                     a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        mbar_arrive_expect_tx(&land_full[r], land_bytes);
        tma_load_3d(land_base + (uint32_t)r * kLandBytes, &tmap, x0, 0,
                    ks * kPktPerStage + kLandPkts * (int)crank, &land_full[r]);
      }
      // boxes still landing after an abort: wait for them before exit
      volatile int no_abort = 0;
      for (int k2 = ks - kRawStages; k2 < ks; ++k2)
        if (k2 >= 0)
          mbar_wait_bounded(&land_full[k2 % kRawStages], (uint32_t)(k2 / kRawStages) & 1u,
                            &no_abort, a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  } else if (kCl && warp == NW + 2) {
    // ------------------------------------------------------------ raw-slot manager (FEED 2)
    if (lane == 0) {
      int ks = 0;
      for (; ks < nks && !abort_sh; ++ks) {
        const int r = ks % kRawStages;
        if (!mbar_wait_bounded(&rempty_bar[r], (uint32_t)(ks / kRawStages) & 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        if (ks + kRawStages < nks) {   // arm the slot for stage ks + R, then free it everywhere
          mbar_arrive_expect_tx(&rfull_bar[r], kRawBytes);
          for (uint32_t q = 0; q < (uint32_t)kClusterCh; ++q)
            mbar_arrive_remote(cluster_map(&dest_free[r], q));
        }
      }
      // stages armed but not seen consumed (only after an abort): wait until
      // the stores the other CTAs may still have in flight to this CTA land
      volatile int no_abort = 0;
      for (int k2 = ks; k2 < nks && k2 < ks + kRawStages; ++k2)
        mbar_wait_bounded<true>(&rfull_bar[k2 % kRawStages], (uint32_t)(k2 / kRawStages) & 1u,
                                &no_abort, a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  } else if (kCl && warp > NW + 2) {
    // ------------------------------------------------------------ transposers (FEED 2)
    // Thread tt holds antenna quad aq of packets pl0 + 4i.  It reads the
    // quad's four 16-byte rows (all four channels of one antenna each) in an
    // order rotated by aq, so that a warp's reads, and its 16-byte writes of
    // consecutive quads, hit distinct banks; the rotation is undone in
    // registers.  All 64 threads read before any writes (the split box
    // reuses the landing slot).
    const int tt = tid - 32 * (NW + 3);                    // 0..63
    const int aq = tt & 15, pl0 = tt >> 4;
    const int NA = a.nant_in;
    const uint32_t land_base = raw_base + kRawStages * kRawBytes;
    const uint8_t *gland = gbase + kOpStages * kStageBytes + kRawStages * kRawBytes;
    for (int ks = 0; ks < nks && !abort_sh; ++ks) {
      const int r = ks % kRawStages;
      if (!mbar_wait_bounded(&land_full[r], (uint32_t)(ks / kRawStages) & 1u, &abort_sh, a.err,
                             DEV_ERR_WAIT_FULL, a.wait_limit_ns))
        break;
      const uint8_t *land = gland + r * kLandBytes;
      uint4 v[4][4];   // [item i][slot e]: antenna 4 aq + ((e + aq) & 3) of packet pl0 + 4i
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int pl = pl0 + 4 * i;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int ant = 4 * aq + ((e + aq) & 3);
          v[i][e] = ant < NA ? *reinterpret_cast<const uint4 *>(land + (pl * NA + ant) * 16)
                             : make_uint4(0u, 0u, 0u, 0u);
        }
      }
      named_bar(2, 64);   // the whole box is in registers
      const uint32_t slot = land_base + (uint32_t)r * kLandBytes;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        // undo the rotation: t[s] = antenna 4 aq + s
        uint4 t0 = v[i][0], t1 = v[i][1], t2 = v[i][2], t3 = v[i][3];
        if (aq & 1) {
          const uint4 x = t3; t3 = t2; t2 = t1; t1 = t0; t0 = x;
        }
        if (aq & 2) {
          uint4 x = t0; t0 = t2; t2 = x;
          x = t1; t1 = t3; t3 = x;
        }
        const uint32_t off = (uint32_t)(((pl0 + 4 * i) * 64 + 4 * aq) * 4);
        st_shared_v4(slot + 0u * 4096u + off, t0.x, t1.x, t2.x, t3.x);
        st_shared_v4(slot + 1u * 4096u + off, t0.y, t1.y, t2.y, t3.y);
        st_shared_v4(slot + 2u * 4096u + off, t0.z, t1.z, t2.z, t3.z);
        st_shared_v4(slot + 3u * 4096u + off, t0.w, t1.w, t2.w, t3.w);
      }
      fence_proxy_async_smem();   // the bulk copies (async proxy) read these writes
      named_bar(2, 64);
      if (tt == 0) {
        // channel q's 4 KB -> packets 16 crank .. +15 of CTA q's raw slot r
        const uint32_t dst = raw_base + (uint32_t)r * kRawBytes + crank * 4096u;
#pragma unroll
        for (uint32_t q = 0; q < (uint32_t)kClusterCh; ++q)
          bulk_s2s_cluster(cluster_map_u32(dst, q), slot + q * 4096u, 4096u,
                           cluster_map(&rfull_bar[r], q));
      }
    }
  } else if (FEED == 1 && warp == NW + 1) {
    // ------------------------------------------------------------ bulk loader
    if (lane == 0) {
      // the stages of all the CTA's channels in order: the next channel's
      // first stages load while this one's epilogue runs
      int G = 0;
      for (; G < nchc * nks && !abort_sh; ++G) {
        const int ci = G / nks, ks = G - ci * nks;
        const int chg = (int)blockIdx.x + ci * (int)gridDim.x;
        const int r = G % kRawStages;
        if (!mbar_wait_bounded(&rempty_bar[r], ((uint32_t)(G / kRawStages) & 1u) ^ 1u, &abort_sh,
                               a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        const int npk = min(kPktPerStage, a.npkt - ks * kPktPerStage);
        const uint32_t bytes = (uint32_t)npk * 256u;
        mbar_arrive_expect_tx(&rfull_bar[r], bytes);
        bulk_g2s(raw_base + (uint32_t)r * kRawBytes,
                 a.in + (int64_t)chg * a.npkt * 256 + (int64_t)ks * kPktPerStage * 256, bytes,
                 &rfull_bar[r]);
      }
      // copies still landing after an abort (their stages are never
      // consumed): wait for the last one issued on each raw stage before the
      // CTA exits; each stage has at most one copy outstanding
      volatile int no_abort = 0;
      for (int k2 = G - kRawStages; k2 < G; ++k2)
        if (k2 >= 0)
          mbar_wait_bounded(&rfull_bar[k2 % kRawStages], (uint32_t)(k2 / kRawStages) & 1u,
                            &no_abort, a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  } else if (warp == NW) {
    // ------------------------------------------------------------ UMMA issuer
    if (lane == 0) {
      bool go = true;
      for (int ci = 0; ci < nchc && go; ++ci) {
      for (int ks = 0; ks < nks; ++ks) {
        const int G = ci * nks + ks;
        const int s = G % kOpStages;
        if (abort_sh ||
            !mbar_wait_bounded(&full_bar[s], (uint32_t)(G / kOpStages) & 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_FULL, a.wait_limit_ns)) {
          go = false;
          break;
        }
        // (channel ci's first stage was written after the epilogue of
        // channel ci - 1 read its accumulators, which these MMAs overwrite)
        tc_fence_after();
        const uint32_t stage = sbase + (uint32_t)s * kStageBytes;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const uint32_t tr = stage + (uint32_t)t * kTile, ti = tr + kHalfTile;
          const uint32_t dre = tmem + (uint32_t)t * 256u;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {   // R [R; I]^T: K = 64 bytes = 2 x 32
            const uint64_t d = umma_desc_sw64(tr + 32u * kk, 512u);
            umma_i8(dre, d, d, kIdescN256, (ks | kk) != 0);
          }
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {   // += I I^T into the first 128 columns
            const uint64_t d = umma_desc_sw64(ti + 32u * kk, 512u);
            umma_i8(dre, d, d, kIdescN128, 1u);
          }
        }
        umma_commit(&empty_bar[s]);
      }
      if (go) umma_commit(&accum_bar);   // channel ci's accumulators are complete
      }
      umma_commit(&final_bar);           // every MMA issued here is complete
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  // no CTA leaves while another may still address its shared memory
  if (kCl) cluster_barrier();
  if (warp == NW) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// FEED 2: the captured block [npkt][nant_in][nchan][4 B] as a 3-D uint8
// tensor (bytes of a packet-antenna row, antennas, packets); boxes of 16
// bytes x nant_in x 16 packets, zero fill past the last packet.
static int encode_captured_map(CUtensorMap *map, const CorrArgs &a) {
  EncodeTiledFn fn = tensor_map_encoder();
  if (!fn) return -1;
  const cuuint64_t dims[3] = {(cuuint64_t)a.nchan * 4, (cuuint64_t)a.nant_in, (cuuint64_t)a.npkt};
  const cuuint64_t strides[2] = {(cuuint64_t)a.nchan * 4, (cuuint64_t)a.nchan * 4 * a.nant_in};
  const cuuint32_t box[3] = {16u, (cuuint32_t)a.nant_in, (cuuint32_t)corrcm::kLandPkts};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t *>(a.in), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

template <int FEED, int NW>
static int launch_cm(const CorrArgs &a, cudaStream_t st) {
  static SmemAttrOnce attr;
  constexpr int smem = corrcm::smem_bytes<FEED>();
  if (smem_attr_once(attr, corr_cm_kernel<FEED, NW>, smem) != cudaSuccess) return -2;
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  if (FEED == 2 && encode_captured_map(&tmap, a) != 0) return -2;
  cudaLaunchConfig_t cfg = {};
  // FEED 0 / 1: persistent, one CTA per SM (the 512 TMEM columns), each
  // looping over channels blockIdx.x, + gridDim.x, ...; FEED 2: one CTA
  // per channel (clusters of four channels)
  unsigned grid = (unsigned)a.nchan;
  if (FEED != 2) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return -2;
    // as few CTAs as give every CTA the largest share (384 channels: 128
    // CTAs of three; the other 20 SMs are free for the next block's corner
    // turn in dsax_correlate_many, 1 % faster than 148 CTAs of two or three)
    if (nsm > 0 && (unsigned)nsm < grid) {
      const int per = (a.nchan + nsm - 1) / nsm;
      grid = (unsigned)((a.nchan + per - 1) / per);
    }
  }
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(corrcm::threads<FEED, NW>(), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = FEED == 2 ? (unsigned)corrcm::kClusterCh : 1u;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, corr_cm_kernel<FEED, NW>, tmap, a) == cudaSuccess ? 0 : -2;
}

int launch_correlate_chanmajor(const CorrArgs &a, cudaStream_t st, int corr_path) {
  switch (corr_path) {
    case 3: return launch_cm<0, 8>(a, st);

    case 5:
    case 7: return launch_cm<1, 16>(a, st);
    default: return launch_cm<1, 8>(a, st);
  }
}

bool captured_cluster_ok(const CorrArgs &a) {
  return a.nchan % corrcm::kClusterCh == 0 && a.nant_in >= 1 && a.nant_in <= 64 &&
         (reinterpret_cast<uintptr_t>(a.in) & 15u) == 0 && tensor_map_encoder() != nullptr;
}

int launch_correlate_captured_cluster(const CorrArgs &a, cudaStream_t st, int unpack_warps) {
  if (!captured_cluster_ok(a)) return -1;
  return unpack_warps == 16 ? launch_cm<2, 16>(a, st) : launch_cm<2, 8>(a, st);
}

int launch_correlate(const CorrArgs &a, int fmt, cudaStream_t st) {
  static SmemAttrOnce attr[3];
  const void *fn = fmt == FMT_CAPTURED    ? (const void *)corr_kernel<FMT_CAPTURED>
                   : fmt == FMT_REORDERED ? (const void *)corr_kernel<FMT_REORDERED>
                                          : (const void *)corr_kernel<FMT_XGPU_INT8>;
  if (fmt < 0 || fmt > 2) return -1;
  if (smem_attr_once(attr[fmt], fn, corr::kSmemBytes) != cudaSuccess) return -2;
  dim3 grid(a.nchan), block(corr::kThreads);
  void *args[] = {(void *)&a};
  cudaError_t e = cudaLaunchKernel(fn, grid, block, args, corr::kSmemBytes, st);
  return e == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

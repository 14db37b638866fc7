// dsax_lflag_tma.cu -- the learned flagger's 64-channel 3x3 layers on
// sm_100a tensor cores, fed by TMA from zero-padded activations.
//
// Activations live on the padded grid [B][H+2][W+2][64] (BF16, NHWC) whose
// border pixels are zero.  On that grid the 3x3 neighbourhood of a run of
// 128 consecutive pixels p0 .. p0+127 is, for tap (dy, dx), the run starting
// at p0 + dy (W+2) + dx.  Per kernel row dy one TMA load (tensor map over
// [npp][64] BF16, 128-byte swizzle) brings the 130-pixel band starting at
// p0 + dy (W+2) - 1; the three taps dx = -1, 0, 1 are the 128-row windows
// starting 0, 1 and 2 rows into it, each the K-major A operand of
// tcgen05.mma kind::f16 (M = 128 pixels, N = Cout, K = 64 channels).  The
// 128-byte swizzle follows the shared-memory address, so a window may start
// at any 128-byte row with the usual descriptor.  Three loads and 36 MMAs
// per tile, no per-pixel gather, each activation row fetched about three
// times.  Loads that start before the first or run past the last padded
// pixel read zeros (TMA out-of-bounds fill).  Tiles cover the
// padded grid; the epilogue writes interior pixels only, so the border stays
// zero.  A layer with fewer input channels (32) keeps them in the first
// channels of the 64 and gets zero weights for the rest.
//   warps 0-7 : epilogue: TMEM -> + bias -> ReLU -> padded BF16 activations,
//               or the nine per-tap projections onto the last layer's weights.
//               Warps q and q + 4 share TMEM lanes 32q .. 32q + 31 and split
//               the output channels (activations) or the taps (projections).
//   warp  8   : TMA producer (one elected thread)
//   warp  9   : TMEM allocation, weight image (bulk copy, resident), UMMA issue
// Persistent CTAs walk the tiles; two TMEM accumulators let the epilogue of
// tile i overlap the MMAs of tile i+1.  Every wait is bounded.
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_lflag.h"
#include "dsax_ptx.cuh"
#include "dsax_tmap.h"

namespace dsax {

namespace lftma {
constexpr int kThreads = 320;
constexpr int kBandRows = 130;                    // 128 pixels + one on each side
constexpr int kBandBytes = kBandRows * 128;       // one band: 130 pixels x 64 BF16
constexpr int kABytes = 17 * 1024;                // stage: the band, rounded to 1 KB
constexpr int kTaps = 9;
constexpr int kBands = 3;
constexpr int kC = 64;                            // channels per padded pixel
template <int COUT> constexpr int stages() {
  return (200 * 1024 - kTaps * COUT * 128) / kABytes < 8 ? (200 * 1024 - kTaps * COUT * 128) / kABytes
                                                          : 8;
}
}  // namespace lftma

struct LfTmaArgs {
  const uint8_t *wimg;   // [9 taps][cout rows x 128 B], 128-byte swizzle
  const float *bias;     // [cout]
  const float *w4;       // projection only: last layer's weights [9][cout] (tap-major)
  uint16_t *out;         // non-projection: padded BF16 [npp][64]
  float *z9;             // projection only: [9][npx] (unpadded pixel order)
  int *err;
  int B, H, W;
  uint64_t wait_limit_ns;
};

// n / d for 0 <= n < 2^24 (exact in FP32) with inv = 1 / d: the FP32
// estimate is within one of the quotient; one integer correction fixes it.
__device__ __forceinline__ int div_small(int n, int d, float inv) {
  int q = __float2int_rz((float)n * inv);
  const int r = n - q * d;
  return q + (r >= d) - (r < 0);
}

__device__ __forceinline__ uint32_t tma_pack_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// CIN: the real input channels of the 64-channel grid rows (32 for layer 2,
// whose upper 32 channels carry zero weights): the MMAs cover K = CIN per
// tap, so layer 2 issues half of layer 3's.
template <int COUT, bool PROJ, int CIN>
__global__ void __launch_bounds__(lftma::kThreads, 1)
    lf_conv_tma_kernel(const __grid_constant__ CUtensorMap tin, LfTmaArgs a) {
  using namespace lftma;
  constexpr int WBYTES = kTaps * COUT * 128;
  constexpr uint32_t IDESC = umma_idesc(/*F32*/ 1, /*BF16*/ 1, /*BF16*/ 1, 128, COUT);
  constexpr uint32_t TCOLS = 2 * COUT;
  constexpr int kStages = stages<COUT>();
  static_assert(COUT == 64, "64 output channels");
  static_assert(CIN == 32 || CIN == 64, "32 or 64 real input channels");
  constexpr int KK = CIN / 16;   // 16-channel K steps per tap

  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar[2];
  __shared__ __align__(8) uint64_t tempty_bar[2];
  __shared__ __align__(8) uint64_t w_bar;
  __shared__ __align__(8) uint64_t final_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ __align__(16) float s_bias[COUT];
  __shared__ __align__(16) float s_w4[PROJ ? kTaps * COUT : 4];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  for (int i = tid; i < COUT; i += blockDim.x) s_bias[i] = a.bias[i];
  if (PROJ)
    for (int i = tid; i < kTaps * COUT; i += blockDim.x) s_w4[i] = a.w4[i];
  const uint32_t wsm = base;
  const uint32_t asm_base = base + WBYTES;

  const int Hp = a.H + 2, Wp = a.W + 2;
  const int npp = a.B * Hp * Wp;
  const int ntiles = (npp + 127) / 128;
  const int nmine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 256);
    }
    mbar_init(&w_bar, 1);
    mbar_init(&final_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == 9) {
    tmem_alloc(&tmem_base_sh, TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 8) {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3, half = warp >> 2;
    const int m = 32 * q + lane;
    const bool small = npp < (1 << 24);
    const float iWp = 1.0f / (float)Wp, iHp = 1.0f / (float)Hp;
    // activations: this warp's 32 channels; projections: all 64, taps 0-4 or 5-8
    constexpr int kCols = PROJ ? COUT : COUT / 2;
    const int c0 = PROJ ? 0 : half * kCols;
    for (int i = 0; i < nmine; ++i) {
      const int bf = i & 1;
      bool ok = mbar_wait_bounded(&tfull_bar[bf], (uint32_t)(i >> 1) & 1u, &abort_sh, a.err,
                                  DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
      tc_fence_after();
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      float v[kCols];
      if (ok) {
        const uint32_t taddr =
            tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(bf * COUT) + (uint32_t)c0;
#pragma unroll
        for (int c = 0; c < kCols / 32; ++c) {
          uint32_t r[32];
          tmem_ld32(taddr + 32u * c, r);
          tmem_wait_ld();
#pragma unroll
          for (int e = 0; e < 32; ++e) v[32 * c + e] = __uint_as_float(r[e]);
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty_bar[bf]);
      const int pp = ((int)blockIdx.x + i * (int)gridDim.x) * 128 + m;
      if (!ok || pp >= npp) continue;
      const int r = small ? div_small(pp, Wp, iWp) : pp / Wp;
      const int wq = pp - r * Wp;
      const int b = small ? div_small(r, Hp, iHp) : r / Hp;
      const int hq = r - b * Hp;
      if (wq < 1 || wq > a.W || hq < 1 || hq > a.H) continue;
#pragma unroll
      for (int c = 0; c < kCols; c += 4) {
        const float4 bb = *reinterpret_cast<const float4 *>(s_bias + c0 + c);
        v[c] = fmaxf(v[c] + bb.x, 0.0f);
        v[c + 1] = fmaxf(v[c + 1] + bb.y, 0.0f);
        v[c + 2] = fmaxf(v[c + 2] + bb.z, 0.0f);
        v[c + 3] = fmaxf(v[c + 3] + bb.w, 0.0f);
      }
      if (PROJ) {
        const int64_t npx = (int64_t)a.B * a.H * a.W;
        const int64_t p = ((int64_t)b * a.H + (hq - 1)) * a.W + (wq - 1);
        const int t0 = half ? 5 : 0, t1 = half ? kTaps : 5;
#pragma unroll
        for (int tap = 0; tap < kTaps; ++tap) {
          if (tap < t0 || tap >= t1) continue;
          float z0 = 0.0f, z1 = 0.0f;   // two chains
#pragma unroll
          for (int c = 0; c < COUT; c += 4) {
            const float4 ww = *reinterpret_cast<const float4 *>(s_w4 + tap * COUT + c);
            z0 = fmaf(ww.x, v[c], z0);
            z1 = fmaf(ww.y, v[c + 1], z1);
            z0 = fmaf(ww.z, v[c + 2], z0);
            z1 = fmaf(ww.w, v[c + 3], z1);
          }
          a.z9[tap * npx + p] = z0 + z1;
        }
      } else {
        uint4 *dst = reinterpret_cast<uint4 *>(a.out + (int64_t)pp * kC + c0);
#pragma unroll
        for (int c = 0; c < kCols / 8; ++c)
          dst[c] = make_uint4(tma_pack_bf16x2(v[8 * c], v[8 * c + 1]),
                              tma_pack_bf16x2(v[8 * c + 2], v[8 * c + 3]),
                              tma_pack_bf16x2(v[8 * c + 4], v[8 * c + 5]),
                              tma_pack_bf16x2(v[8 * c + 6], v[8 * c + 7]));
      }
    }
  } else if (warp == 8) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tin)) : "memory");
      const int G = nmine * kBands;
      int g = 0;
      for (; g < G && !abort_sh; ++g) {
        const int s = g % kStages;
        if (!mbar_wait_bounded(&empty_bar[s], ((uint32_t)(g / kStages) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        const int i = g / kBands, band = g - i * kBands;   // kernel row dy = band - 1
        const int row = ((int)blockIdx.x + i * (int)gridDim.x) * 128 + (band - 1) * Wp - 1;
        mbar_arrive_expect_tx(&full_bar[s], (uint32_t)kBandBytes);
        tma_load_2d(asm_base + (uint32_t)s * kABytes, &tin, 0, row, &full_bar[s]);
      }
      // loads still landing after an abort: wait (bounded) before exiting
      volatile int no_abort = 0;
      for (int g2 = g - kStages; g2 < g; ++g2)
        if (g2 >= 0)
          mbar_wait_bounded(&full_bar[g2 % kStages], (uint32_t)(g2 / kStages) & 1u, &no_abort,
                            a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ weights + UMMA
    if (lane == 0) {
      mbar_arrive_expect_tx(&w_bar, (uint32_t)WBYTES);
      for (int o = 0; o < WBYTES; o += 8192)
        bulk_g2s(wsm + (uint32_t)o, a.wimg + o, (uint32_t)min(8192, WBYTES - o), &w_bar);
      const uint64_t adesc0 = umma_desc_sw128(asm_base, 1024u);
      const uint64_t bdesc0 = umma_desc_sw128(wsm, 1024u);
      bool ok = mbar_wait_bounded(&w_bar, 0u, &abort_sh, a.err, DEV_ERR_WAIT_FULL, a.wait_limit_ns);
      if (!ok) {   // the weight copies may still be landing
        volatile int no_abort = 0;
        mbar_wait_bounded(&w_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
      }
      for (int i = 0; i < nmine && ok && !abort_sh; ++i) {
        const int bf = i & 1;
        if (!mbar_wait_bounded(&tempty_bar[bf], ((uint32_t)(i >> 1) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        // Descriptors: base + compile-time offsets (the 14-bit address field
        // cannot overflow below 256 KB), so each MMA costs one add and the
        // issue.
        const uint32_t dcol = tmem + (uint32_t)(bf * COUT);
#pragma unroll
        for (int band = 0; band < kBands; ++band) {
          const int g = i * kBands + band, s = g % kStages;
          if (!mbar_wait_bounded(&full_bar[s], (uint32_t)(g / kStages) & 1u, &abort_sh, a.err,
                                 DEV_ERR_WAIT_FULL, a.wait_limit_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ab = adesc0 + (uint64_t)(((uint32_t)s * kABytes) >> 4);
#pragma unroll
          for (int dx = 0; dx < 3; ++dx)   // tap (band, dx): window starting dx rows in
#pragma unroll
            for (int kk = 0; kk < KK; ++kk)   // K = CIN bf16 = KK x 16
              umma_f16(dcol, ab + (uint64_t)((128 * dx + 32 * kk) >> 4),
                       bdesc0 + (uint64_t)(((3 * band + dx) * COUT * 128 + 32 * kk) >> 4), IDESC,
                       (band | dx | kk) != 0);
          umma_commit(&empty_bar[s]);
        }
        if (!ok) break;
        umma_commit(&tfull_bar[bf]);
      }
      umma_commit(&final_bar);
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 9) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, TCOLS);
  }
}

// Layer weights W[co][tap][ci] (FP32, cin real input channels) -> the B
// operand image of the padded layers: tap t is K block t, row n, element ci
// (< 64) at the 128-byte-swizzled offset; zero for ci >= cin.
__global__ void lf_tma_wimg_kernel(const float *w, uint8_t *img, int cin, int cout) {
  const int n_el = lftma::kTaps * 64 * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
    const int n = i / (lftma::kTaps * 64), k = i % (lftma::kTaps * 64);
    const int tap = k / 64, ci = k % 64;
    const float v = ci < cin ? w[((int64_t)n * lftma::kTaps + tap) * cin + ci] : 0.0f;
    uint32_t bits;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(bits) : "f"(0.0f), "f"(v));
    *reinterpret_cast<uint16_t *>(img + (int64_t)tap * cout * 128 +
                                  sw128_offset((uint32_t)n, (uint32_t)(ci / 8)) + 2 * (ci % 8)) =
        (uint16_t)(bits & 0xFFFFu);
  }
}

// Zeroes the border pixels of a padded grid of `chunks` 16-byte chunks per
// pixel (8 for 64 BF16 channels, 1 for the 8 BF16 features).
__global__ void lf_pad_border_kernel(uint16_t *act, int B, int H, int W, int chunks) {
  const int Hp = H + 2, Wp = W + 2;
  const int per = 2 * Wp + 2 * H;   // border pixels per image
  const int64_t n = (int64_t)B * per * chunks;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int chunk = (int)(i % chunks);
    const int64_t q = i / chunks;
    const int b = (int)(q / per), k = (int)(q % per);
    int hq, wq;
    if (k < Wp) { hq = 0; wq = k; }
    else if (k < 2 * Wp) { hq = Hp - 1; wq = k - Wp; }
    else { const int k2 = k - 2 * Wp; hq = 1 + (k2 >> 1); wq = (k2 & 1) ? Wp - 1 : 0; }
    const int64_t pp = ((int64_t)b * Hp + hq) * Wp + wq;
    reinterpret_cast<uint4 *>(act)[pp * chunks + chunk] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// ---------------------------------------------------------------------------
// First layer (8 -> 32 channels) from the zero-bordered feature grid
// [B][H+2][W+2][8] BF16.  A tap is 16 bytes, too narrow for a swizzled box,
// so per tile three unswizzled TMA boxes of 130 pixels x 16 B (one per
// kernel row) land in a band slot, and four builder warps copy each pixel's
// nine taps into the K-major 128-byte-swizzled A tile (K = 72 in two 64-wide
// blocks, k = 8 tap + ci; the rest of the second block stays zero), then
// 5 MMAs of N = 32 (K 64 + 16).  The epilogue writes channels 0-31 of the interior
// pixels of the 64-channel grid the next layer reads (channels 32-63 are
// zero there).
//   warps 0-3 : A-tile builders      warps 4-7 : epilogue
//   warp  8   : TMA producer         warp  9   : TMEM, weights, UMMA issue
namespace lf1 {
constexpr int kThreads = 320;
constexpr int kBandPix = 130;
constexpr int kBandBytes = kBandPix * 16;           // 2,080
constexpr int kBandStride = 2176;                   // 128-byte aligned band offset
constexpr int kSlotStride = 6656;                   // 128-byte aligned slot
constexpr int kSlots = 8;
constexpr int kABytes = 2 * 16384;                  // two K blocks of 128 x 128 B
constexpr int kAStages = 4;
constexpr int kCout = 32;
constexpr int kWBytes = 2 * kCout * 128;            // B operand: two K blocks
constexpr int kSmemBytes = 1024 + kWBytes + kAStages * kABytes + kSlots * kSlotStride;
static_assert(kSmemBytes <= 227 * 1024, "shared memory budget");
}  // namespace lf1

struct Lf1Args {
  const uint8_t *wimg;   // [2 K blocks][32 rows x 128 B], 128-byte swizzle
  const float *bias;     // [32]
  uint16_t *out;         // padded BF16 [npp][64]: channels 0-31 written
  int *err;
  int B, H, W;
  uint64_t wait_limit_ns;
};

__global__ void __launch_bounds__(lf1::kThreads, 1)
    lf_conv1_tma_kernel(const __grid_constant__ CUtensorMap tfeat, Lf1Args a) {
  using namespace lf1;
  constexpr uint32_t IDESC = umma_idesc(/*F32*/ 1, /*BF16*/ 1, /*BF16*/ 1, 128, kCout);
  constexpr uint32_t TCOLS = 2 * kCout;   // 64
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bfull_bar[kSlots];
  __shared__ __align__(8) uint64_t bempty_bar[kSlots];
  __shared__ __align__(8) uint64_t afull_bar[kAStages];
  __shared__ __align__(8) uint64_t aempty_bar[kAStages];
  __shared__ __align__(8) uint64_t tfull_bar[2];
  __shared__ __align__(8) uint64_t tempty_bar[2];
  __shared__ __align__(8) uint64_t w_bar;
  __shared__ __align__(8) uint64_t final_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ __align__(16) float s_bias[kCout];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *const gbase = smem_raw + (base - smem_u32(smem_raw));
  const uint32_t wsm = base;
  const uint32_t a_base = base + kWBytes;                    // 1024-aligned (kWBytes = 8 KB)
  const uint32_t b_base = a_base + kAStages * kABytes;
  for (int i = tid; i < kCout; i += blockDim.x) s_bias[i] = a.bias[i];
  // chunks 1-7 of every A stage's second K block are never written again
  for (int i = tid; i < kAStages * 128 * 7; i += blockDim.x) {
    const int st = i / (128 * 7), r = (i / 7) % 128, ch = 1 + i % 7;
    *reinterpret_cast<uint4 *>(gbase + kWBytes + st * kABytes + 16384 + sw128_offset(r, ch)) =
        make_uint4(0u, 0u, 0u, 0u);
  }
  fence_proxy_async_smem();

  const int Hp = a.H + 2, Wp = a.W + 2;
  const int npp = a.B * Hp * Wp;
  const int ntiles = (npp + 127) / 128;
  const int nmine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  if (tid == 0) {
    for (int r = 0; r < kSlots; ++r) {
      mbar_init(&bfull_bar[r], 1);
      mbar_init(&bempty_bar[r], 128);
    }
    for (int s2 = 0; s2 < kAStages; ++s2) {
      mbar_init(&afull_bar[s2], 128);
      mbar_init(&aempty_bar[s2], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 128);
    }
    mbar_init(&w_bar, 1);
    mbar_init(&final_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == 9) {
    tmem_alloc(&tmem_base_sh, TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 4) {
    // ------------------------------------------------------------ A builders
    const int m = tid;
    for (int i = 0; i < nmine && !abort_sh; ++i) {
      const int r = i % kSlots, s2 = i % kAStages;
      if (!mbar_wait_bounded(&bfull_bar[r], (uint32_t)(i / kSlots) & 1u, &abort_sh, a.err,
                             DEV_ERR_WAIT_FULL, a.wait_limit_ns))
        break;
      uint4 t[9];
      const uint8_t *slot = gbase + kWBytes + kAStages * kABytes + r * kSlotStride;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap)
        t[tap] = *reinterpret_cast<const uint4 *>(slot + (tap / 3) * kBandStride + (m + tap % 3) * 16);
      // the next TMA load (async proxy) overwrites this slot: order the reads
      fence_proxy_async_smem();
      mbar_arrive(&bempty_bar[r]);
      if (!mbar_wait_bounded(&aempty_bar[s2], ((uint32_t)(i / kAStages) & 1u) ^ 1u, &abort_sh, a.err,
                             DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
        break;
      uint8_t *as = gbase + kWBytes + s2 * kABytes;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap)
        *reinterpret_cast<uint4 *>(as + (tap / 8) * 16384 + sw128_offset((uint32_t)m, (uint32_t)(tap % 8))) =
            t[tap];
      fence_proxy_async_smem();
      mbar_arrive(&afull_bar[s2]);
    }
  } else if (warp < 8) {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int m = 32 * q + lane;
    const bool small = npp < (1 << 24);
    const float iWp = 1.0f / (float)Wp, iHp = 1.0f / (float)Hp;
    for (int i = 0; i < nmine; ++i) {
      const int bf = i & 1;
      bool ok = mbar_wait_bounded(&tfull_bar[bf], (uint32_t)(i >> 1) & 1u, &abort_sh, a.err,
                                  DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
      tc_fence_after();
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      float v[kCout];
      if (ok) {
        uint32_t rr[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(bf * kCout), rr);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; ++e) v[e] = __uint_as_float(rr[e]);
      }
      tc_fence_before();
      mbar_arrive(&tempty_bar[bf]);
      const int pp = ((int)blockIdx.x + i * (int)gridDim.x) * 128 + m;
      if (!ok || pp >= npp) continue;
      const int r = small ? div_small(pp, Wp, iWp) : pp / Wp;
      const int wq = pp - r * Wp;
      const int b = small ? div_small(r, Hp, iHp) : r / Hp;
      const int hq = r - b * Hp;
      if (wq < 1 || wq > a.W || hq < 1 || hq > a.H) continue;
#pragma unroll
      for (int c = 0; c < kCout; ++c) v[c] = fmaxf(v[c] + s_bias[c], 0.0f);
      uint4 *dst = reinterpret_cast<uint4 *>(a.out + (int64_t)pp * lftma::kC);
#pragma unroll
      for (int c = 0; c < kCout / 8; ++c)
        dst[c] = make_uint4(tma_pack_bf16x2(v[8 * c], v[8 * c + 1]),
                            tma_pack_bf16x2(v[8 * c + 2], v[8 * c + 3]),
                            tma_pack_bf16x2(v[8 * c + 4], v[8 * c + 5]),
                            tma_pack_bf16x2(v[8 * c + 6], v[8 * c + 7]));
    }
  } else if (warp == 8) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tfeat)) : "memory");
      int i = 0;
      for (; i < nmine && !abort_sh; ++i) {
        const int r = i % kSlots;
        if (!mbar_wait_bounded(&bempty_bar[r], ((uint32_t)(i / kSlots) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        const int p0 = ((int)blockIdx.x + i * (int)gridDim.x) * 128;
        mbar_arrive_expect_tx(&bfull_bar[r], (uint32_t)(3 * kBandBytes));
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
          tma_load_2d(b_base + (uint32_t)(r * kSlotStride + dy * kBandStride), &tfeat, 0,
                      p0 + (dy - 1) * Wp - 1, &bfull_bar[r]);
      }
      // loads still landing after an abort: wait (bounded) before exiting
      volatile int no_abort = 0;
      for (int i2 = i - kSlots; i2 < i; ++i2)
        if (i2 >= 0)
          mbar_wait_bounded(&bfull_bar[i2 % kSlots], (uint32_t)(i2 / kSlots) & 1u, &no_abort, a.err,
                            DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ weights + UMMA
    if (lane == 0) {
      mbar_arrive_expect_tx(&w_bar, (uint32_t)kWBytes);
      bulk_g2s(wsm, a.wimg, (uint32_t)kWBytes, &w_bar);
      const uint64_t adesc0 = umma_desc_sw128(a_base, 1024u);
      const uint64_t bdesc0 = umma_desc_sw128(wsm, 1024u);
      bool ok = mbar_wait_bounded(&w_bar, 0u, &abort_sh, a.err, DEV_ERR_WAIT_FULL, a.wait_limit_ns);
      if (!ok) {   // the weight copy may still be landing
        volatile int no_abort = 0;
        mbar_wait_bounded(&w_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_FULL, drain_limit(a.wait_limit_ns));
      }
      for (int i = 0; i < nmine && ok && !abort_sh; ++i) {
        const int bf = i & 1, s2 = i % kAStages;
        if (!mbar_wait_bounded(&tempty_bar[bf], ((uint32_t)(i >> 1) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        if (!mbar_wait_bounded(&afull_bar[s2], (uint32_t)(i / kAStages) & 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_FULL, a.wait_limit_ns))
          break;
        tc_fence_after();
        const uint64_t ab = adesc0 + (uint64_t)(((uint32_t)s2 * kABytes) >> 4);
        const uint32_t dcol = tmem + (uint32_t)(bf * kCout);
        // K = 72: block 0 holds taps 0-7, block 1 tap 8 in its first 16
        // K elements (the rest is zero and not issued)
#pragma unroll
        for (int kb = 0; kb < 2; ++kb)
#pragma unroll
          for (int kk = 0; kk < (kb == 0 ? 4 : 1); ++kk)
            umma_f16(dcol, ab + (uint64_t)((kb * 16384 + 32 * kk) >> 4),
                     bdesc0 + (uint64_t)((kb * kCout * 128 + 32 * kk) >> 4), IDESC, (kb | kk) != 0);
        umma_commit(&aempty_bar[s2]);
        umma_commit(&tfull_bar[bf]);
      }
      umma_commit(&final_bar);
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 9) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, TCOLS);
  }
}

namespace {

// Tensor map over a padded grid [npp][ch] BF16 with 130-pixel boxes: ch =
// 64 (128-byte rows, 128-byte swizzle) or 8 (16-byte rows, no swizzle);
// zero fill out of bounds.
int encode_grid_map(CUtensorMap *map, const uint16_t *grid, int64_t npp, int ch) {
  EncodeTiledFn fn = tensor_map_encoder();
  if (!fn || npp < 1 || npp > (int64_t)0x7fffffff || (ch != 64 && ch != 8)) return -1;
  const cuuint64_t dims[2] = {(cuuint64_t)ch, (cuuint64_t)npp};
  const cuuint64_t strides[1] = {(cuuint64_t)ch * 2};
  const cuuint32_t box[2] = {(cuuint32_t)ch, (cuuint32_t)lftma::kBandRows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t *>(grid), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        ch == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

template <int COUT, bool PROJ, int CIN>
int conv_tma_launch(const CUtensorMap &map, const LfTmaArgs &a, int num_sms, cudaStream_t st) {
  constexpr int smem = 1024 + lftma::kTaps * COUT * 128 + lftma::stages<COUT>() * lftma::kABytes;
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, lf_conv_tma_kernel<COUT, PROJ, CIN>, smem) != cudaSuccess) return -2;
  const int64_t npp = (int64_t)a.B * (a.H + 2) * (a.W + 2);
  const int ntiles = (int)((npp + 127) / 128);
  const int grid = ntiles < num_sms ? ntiles : num_sms;
  if (grid < 1) return 0;
  lf_conv_tma_kernel<COUT, PROJ, CIN><<<grid, lftma::kThreads, smem, st>>>(map, a);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

size_t lf_pad_bytes(int B, int H, int W) {
  return (size_t)B * (H + 2) * (W + 2) * lftma::kC * 2;
}

size_t lf_tma_wimg_bytes() { return (size_t)2 * lftma::kTaps * 64 * 128; }

int lf_tma_prepare(const LfNet &net, uint8_t *wimg, cudaStream_t st) {
  lf_tma_wimg_kernel<<<64, 256, 0, st>>>(net.w[1], wimg, kLfCin[1], kLfCout[1]);
  lf_tma_wimg_kernel<<<64, 256, 0, st>>>(net.w[2], wimg + lftma::kTaps * 64 * 128, kLfCin[2],
                                         kLfCout[2]);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int lf_pad_borders(uint16_t *grid, int B, int H, int W, int chunks, cudaStream_t st) {
  lf_pad_border_kernel<<<256, 256, 0, st>>>(grid, B, H, W, chunks);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

size_t lf_feat_pad_bytes(int B, int H, int W) { return (size_t)B * (H + 2) * (W + 2) * 16; }

// Layer 1 (8 -> 32) from the padded feature grid featp into channels 0-31 of
// the padded grid act1p.
int lf_tma_layer1(const LfNet &net, const uint8_t *wimg, const uint16_t *featp, uint16_t *act1p,
                  int B, int H, int W, int num_sms, int *err, uint64_t wait_limit_ns,
                  cudaStream_t st) {
  static_assert(kLfCin[0] == 8 && kLfCout[0] == lf1::kCout, "layer 1 is 8 -> 32");
  const int64_t npp = (int64_t)B * (H + 2) * (W + 2);
  CUtensorMap mf;
  if (encode_grid_map(&mf, featp, npp, 8) != 0) return -1;
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, lf_conv1_tma_kernel, lf1::kSmemBytes) != cudaSuccess) return -2;
  Lf1Args a{};
  a.wimg = wimg; a.bias = net.b[0]; a.out = act1p; a.err = err;
  a.B = B; a.H = H; a.W = W; a.wait_limit_ns = wait_limit_ns;
  const int ntiles = (int)((npp + 127) / 128);
  const int grid = ntiles < num_sms ? ntiles : num_sms;
  if (grid < 1) return 0;
  lf_conv1_tma_kernel<<<grid, lf1::kThreads, lf1::kSmemBytes, st>>>(mf, a);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Layers 2 and 3 of the net (32 -> 64, 64 -> 64 + the projection onto the
// last layer), from the padded layer-1 activations act1p to z9.
int lf_tma_layers23(const LfNet &net, const uint8_t *wimg, const uint16_t *act1p, uint16_t *act2p,
                    float *z9, int B, int H, int W, int num_sms, int *err, uint64_t wait_limit_ns,
                    cudaStream_t st) {
  static_assert(kLfCin[1] == 32 && kLfCout[1] == 64 && kLfCin[2] == 64 && kLfCout[2] == 64,
                "padded layers are written for 32 -> 64 -> 64");
  const int64_t npp = (int64_t)B * (H + 2) * (W + 2);
  CUtensorMap m1, m2;
  if (encode_grid_map(&m1, act1p, npp, 64) != 0 || encode_grid_map(&m2, act2p, npp, 64) != 0) return -1;
  LfTmaArgs a{};
  a.err = err;
  a.B = B; a.H = H; a.W = W;
  a.wait_limit_ns = wait_limit_ns;
  a.wimg = wimg; a.bias = net.b[1]; a.out = act2p;
  int e = conv_tma_launch<64, false, kLfCin[1]>(m1, a, num_sms, st);
  a.wimg = wimg + lftma::kTaps * 64 * 128; a.bias = net.b[2]; a.out = nullptr;
  a.w4 = net.w[3]; a.z9 = z9;
  e |= conv_tma_launch<64, true, kLfCin[2]>(m2, a, num_sms, st);
  return e;
}

}  // namespace dsax

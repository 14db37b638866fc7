// dsax_lflag_tc.cu -- learned-flagger inference on sm_100a tensor cores:
// the first 3x3 layer (8 -> 32 channels), the 64 -> 1 tap sum and the mask;
// the 64-channel layers are TMA-fed (dsax_lflag_tma.cu).
//
// The first layer is an implicit GEMM: D[128 pixels x Cout] = A B^T with
// A row m = the pixel's 3x3 neighbourhood, K = 9 taps x Cin (k = tap * Cin
// + ci, tap = 3 ky + kx, zero outside the image), and B = the layer's
// weights W[co][tap][ci] in the same K order.  BF16 operands, FP32
// accumulation in TMEM (tcgen05.mma kind::f16, M=128, N=Cout).  With 8
// input channels a tap is 16 bytes, too narrow for a swizzled TMA box, so
//   warps 0-3 : producers.  Thread m gathers pixel m's eight 16-byte K
//               chunks of a 64-wide K block straight into the 128-byte-
//               swizzled A stage with cp.async (zero fill at the image
//               border); it keeps all but two of the stages in flight and
//               marks a stage full once its own copies have landed.
//   warps 4-7 : epilogue: TMEM -> + bias -> ReLU -> BF16 activations, written
//               into the zero-bordered 64-channel grid the next layer reads
//               (pad_out), or, for a projection layer, the 9 per-tap
//               projections onto the last layer's weights.
//   warp  8   : TMEM allocation, weight image load (bulk copy, resident),
//               single-thread UMMA issue.
// Persistent CTAs walk 128-pixel tiles; TMEM holds two accumulators so the
// epilogue of tile i overlaps the MMAs of tile i+1.  Every wait is bounded.
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_lflag.h"
#include "dsax_ptx.cuh"

namespace dsax {

namespace lftc {
constexpr int kThreads = 288;
constexpr int kABytes = 128 * 128;      // A stage: 128 pixels x 64 bf16 (one K block)
// As many A stages as fit beside the resident weight image (<= 200 KB of
// shared memory); the producers keep all but two of them in flight.
template <int CIN, int COUT> constexpr int stages() {
  return (200 * 1024 - ((9 * CIN + 63) / 64) * COUT * 128) / kABytes < 12
             ? (200 * 1024 - ((9 * CIN + 63) / 64) * COUT * 128) / kABytes
             : 12;
}
}  // namespace lftc

struct LfTcArgs {
  const uint16_t *in;   // BF16 activations [npx][cin] (NHWC)
  const uint8_t *wimg;  // weight image [kb][cout rows x 128 B], 128-byte swizzle
  const float *bias;    // [cout]
  const float *w4;      // projection only: last layer's weights [9][cout] (tap-major)
  uint16_t *out;        // BF16 [npx][cout]
  float *z9;            // projection only: [9][npx]
  int *err;
  int B, H, W;
  uint64_t wait_limit_ns;
  int pad_out;          // 1: write the padded grid [B][H+2][W+2][64] (channels >= COUT zero)
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

template <int CIN, int COUT, bool PROJ>
__global__ void __launch_bounds__(lftc::kThreads, 1) lf_conv_tc_kernel(LfTcArgs a) {
  using namespace lftc;
  constexpr int KB = (9 * CIN + 63) / 64;
  constexpr int WBYTES = KB * COUT * 128;
  constexpr uint32_t IDESC = umma_idesc(/*F32*/ 1, /*BF16*/ 1, /*BF16*/ 1, 128, COUT);
  constexpr uint32_t TCOLS = 2 * COUT;   // 64 or 128: a power of two >= 32
  constexpr int kStages = stages<CIN, COUT>();
  constexpr int kAhead = kStages - 2;      // cp.async groups in flight per producer thread
  static_assert(CIN % 8 == 0 && (COUT == 32 || COUT == 64), "layer shape");

  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar[2];
  __shared__ __align__(8) uint64_t tempty_bar[2];
  __shared__ __align__(8) uint64_t w_bar;
  __shared__ __align__(8) uint64_t final_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  // epilogue constants: bias, and the last layer's weights for the projection
  __shared__ __align__(16) float s_bias[COUT];
  __shared__ __align__(16) float s_w4[PROJ ? 9 * COUT : 4];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  for (int i = tid; i < COUT; i += blockDim.x) s_bias[i] = a.bias[i];
  if (PROJ)
    for (int i = tid; i < 9 * COUT; i += blockDim.x) s_w4[i] = a.w4[i];
  const uint32_t wsm = base;
  const uint32_t asm_base = base + WBYTES;

  const int npx = a.B * a.H * a.W;
  const int ntiles = (npx + 127) / 128;
  const int nmine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 128);
      mbar_init(&empty_bar[s], 1);
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
  if (warp == 8) {
    tmem_alloc(&tmem_base_sh, TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 4) {
    // ------------------------------------------------------------ producers
    const int m = tid;
    const int G = nmine * KB;
    int b = 0, h = 0, w = 0;
    bool pv = false;
    for (int g = 0; g < G + kAhead; ++g) {
      if (g < G && !abort_sh) {
        const int s = g % kStages;
        const int i = g / KB, kb = g - i * KB;
        if (kb == 0) {
          const int p = ((int)blockIdx.x + i * (int)gridDim.x) * 128 + m;
          pv = p < npx;
          const int pp = pv ? p : 0;
          w = pp % a.W;
          h = (pp / a.W) % a.H;
          b = pp / (a.W * a.H);
        }
        if (mbar_wait_bounded(&empty_bar[s], ((uint32_t)(g / kStages) & 1u) ^ 1u, &abort_sh, a.err,
                              DEV_ERR_WAIT_EMPTY, a.wait_limit_ns)) {
          const uint32_t dst = asm_base + (uint32_t)s * kABytes;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int k0 = 64 * kb + 8 * j;
            const int tap = k0 / CIN, ci0 = k0 - (k0 / CIN) * CIN;
            const int hh = h + tap / 3 - 1, ww = w + tap % 3 - 1;
            const bool ok = pv && k0 < 9 * CIN && hh >= 0 && hh < a.H && ww >= 0 && ww < a.W;
            const uint16_t *src = ok ? a.in + ((int64_t)(b * a.H + hh) * a.W + ww) * CIN + ci0 : a.in;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                             dst + sw128_offset((uint32_t)m, (uint32_t)j)),
                         "l"(src), "r"(ok ? 16 : 0)
                         : "memory");
          }
        }
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
      if (g >= kAhead && g - kAhead < G) {
        asm volatile("cp.async.wait_group %0;" ::"n"(kAhead) : "memory");
        fence_proxy_async_smem();
        mbar_arrive(&full_bar[(g - kAhead) % kStages]);
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp < 8) {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int m = 32 * q + lane;
    for (int i = 0; i < nmine; ++i) {
      const int bf = i & 1;
      bool ok = mbar_wait_bounded(&tfull_bar[bf], (uint32_t)(i >> 1) & 1u, &abort_sh, a.err,
                                  DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
      tc_fence_after();
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      float v[COUT];
      if (ok) {
        const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(bf * COUT);
#pragma unroll
        for (int c = 0; c < COUT / 32; ++c) {
          uint32_t r[32];
          tmem_ld32(taddr + 32u * c, r);
          tmem_wait_ld();
#pragma unroll
          for (int e = 0; e < 32; ++e) v[32 * c + e] = __uint_as_float(r[e]);
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty_bar[bf]);
      const int p = ((int)blockIdx.x + i * (int)gridDim.x) * 128 + m;
      if (!ok || p >= npx) continue;
#pragma unroll
      for (int c = 0; c < COUT; c += 4) {
        const float4 bb = *reinterpret_cast<const float4 *>(s_bias + c);
        v[c] = fmaxf(v[c] + bb.x, 0.0f);
        v[c + 1] = fmaxf(v[c + 1] + bb.y, 0.0f);
        v[c + 2] = fmaxf(v[c + 2] + bb.z, 0.0f);
        v[c + 3] = fmaxf(v[c + 3] + bb.w, 0.0f);
      }
      if (PROJ) {
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
          float z0 = 0.0f, z1 = 0.0f;   // two chains
#pragma unroll
          for (int c = 0; c < COUT; c += 4) {
            const float4 ww = *reinterpret_cast<const float4 *>(s_w4 + tap * COUT + c);
            z0 = fmaf(ww.x, v[c], z0);
            z1 = fmaf(ww.y, v[c + 1], z1);
            z0 = fmaf(ww.z, v[c + 2], z0);
            z1 = fmaf(ww.w, v[c + 3], z1);
          }
          a.z9[(int64_t)tap * npx + p] = z0 + z1;
        }
      } else {
        uint4 *dst;
        if (a.pad_out) {   // padded grid: pixel (b, h + 1, w + 1) of [B][H+2][W+2][64]
          const int w = p % a.W, h = (p / a.W) % a.H, b = p / (a.W * a.H);
          dst = reinterpret_cast<uint4 *>(a.out + (((int64_t)b * (a.H + 2) + h + 1) * (a.W + 2) + w + 1) * 64);
#pragma unroll
          for (int c = COUT / 8; c < 8; ++c) dst[c] = make_uint4(0u, 0u, 0u, 0u);
        } else {
          dst = reinterpret_cast<uint4 *>(a.out + (int64_t)p * COUT);
        }
#pragma unroll
        for (int c = 0; c < COUT / 8; ++c)
          dst[c] = make_uint4(pack_bf16x2(v[8 * c], v[8 * c + 1]), pack_bf16x2(v[8 * c + 2], v[8 * c + 3]),
                              pack_bf16x2(v[8 * c + 4], v[8 * c + 5]),
                              pack_bf16x2(v[8 * c + 6], v[8 * c + 7]));
      }
    }
  } else {
    // ------------------------------------------------------------ weights + UMMA
    if (lane == 0) {
      mbar_arrive_expect_tx(&w_bar, (uint32_t)WBYTES);
      for (int o = 0; o < WBYTES; o += 8192)
        bulk_g2s(wsm + (uint32_t)o, a.wimg + o, (uint32_t)min(8192, WBYTES - o), &w_bar);
      bool ok = mbar_wait_bounded(&w_bar, 0u, &abort_sh, a.err, DEV_ERR_WAIT_FULL, a.wait_limit_ns);
      for (int i = 0; i < nmine && ok && !abort_sh; ++i) {
        const int bf = i & 1;
        if (!mbar_wait_bounded(&tempty_bar[bf], ((uint32_t)(i >> 1) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        for (int kb = 0; kb < KB; ++kb) {
          const int g = i * KB + kb, s = g % kStages;
          if (!mbar_wait_bounded(&full_bar[s], (uint32_t)(g / kStages) & 1u, &abort_sh, a.err,
                                 DEV_ERR_WAIT_FULL, a.wait_limit_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t as = asm_base + (uint32_t)s * kABytes;
          const uint32_t bs = wsm + (uint32_t)kb * (COUT * 128);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {   // K = 64 bf16 = 4 x 16
            const uint64_t ad = umma_desc_sw128(as + 32u * kk, 1024u);
            const uint64_t bd = umma_desc_sw128(bs + 32u * kk, 1024u);
            umma_f16(tmem + (uint32_t)(bf * COUT), ad, bd, IDESC, (kb | kk) != 0);
          }
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
  if (warp == 8) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM, a.wait_limit_ns);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, TCOLS);
  }
}

// Layer weights W[co][tap][ci] (FP32) -> the B operand image: K block kb,
// row n, bytes of element k = 64 kb + e at the 128-byte-swizzled offset;
// zero beyond 9 * cin.
__global__ void lf_tc_wimg_kernel(const float *w, uint8_t *img, int cin, int cout, int nkb) {
  const int n_el = nkb * 64 * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
    const int n = i / (nkb * 64), k = i % (nkb * 64);
    const float v = k < 9 * cin ? w[((int64_t)n * 9 + k / cin) * cin + k % cin] : 0.0f;
    const int kb = k / 64, e = k % 64;
    uint32_t bits;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(bits) : "f"(0.0f), "f"(v));
    *reinterpret_cast<uint16_t *>(img + (int64_t)kb * cout * 128 +
                                  sw128_offset((uint32_t)n, (uint32_t)(e / 8)) + 2 * (e % 8)) =
        (uint16_t)(bits & 0xFFFFu);
  }
}

// Last layer (Cout = 1): logit[p] = b + sum over taps of z9[tap][p + shift],
// zero outside the image; then the mask (inside the guard band, logit >
// threshold, or a permanently flagged channel).
__global__ void lf_tapsum_kernel(const float *z9, const float *b4, float *logit, uint8_t *mask,
                                 int B, int H, int W, int guard, float thresh, LfPerm perm) {
  const int npx = B * H * W;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += gridDim.x * blockDim.x) {
    const int w = p % W, h = (p / W) % H, b = p / (W * H);
    float z = __ldg(b4);
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int hh = h + tap / 3 - 1, ww = w + tap % 3 - 1;
      if (hh >= 0 && hh < H && ww >= 0 && ww < W)
        z += z9[(int64_t)tap * npx + ((int64_t)b * H + hh) * W + ww];
    }
    if (logit) logit[p] = z;
    bool pm = false;
    for (int k = 0; k < perm.n; ++k) pm |= perm.ch[k] == w;
    mask[p] = (w >= guard && w < W - guard && (z > thresh || pm)) ? 1 : 0;
  }
}

namespace {

template <int CIN, int COUT, bool PROJ>
int conv_tc_launch(const LfTcArgs &a, int num_sms, cudaStream_t st) {
  constexpr int KB = (9 * CIN + 63) / 64;
  constexpr int smem = 1024 + KB * COUT * 128 + lftc::stages<CIN, COUT>() * lftc::kABytes;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(lf_conv_tc_kernel<CIN, COUT, PROJ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return -2;
    attr = true;
  }
  const int npx = a.B * a.H * a.W;
  const int ntiles = (npx + 127) / 128;
  const int grid = ntiles < num_sms ? ntiles : num_sms;
  if (grid < 1) return 0;
  lf_conv_tc_kernel<CIN, COUT, PROJ><<<grid, lftc::kThreads, smem, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

// Weight images: layer 0 in the gather layout (K = 9 taps x 8 channels in
// 64-wide blocks), then layers 1 and 2 in the padded-grid layout
// (dsax_lflag_tma.cu).
static size_t lf_l0_wimg_bytes() { return (size_t)((9 * kLfCin[0] + 63) / 64) * kLfCout[0] * 128; }

size_t lf_tc_wimg_bytes() { return lf_l0_wimg_bytes() + lf_tma_wimg_bytes(); }

int lf_tc_prepare(const LfNet &net, uint8_t *wimg, cudaStream_t st) {
  lf_tc_wimg_kernel<<<64, 256, 0, st>>>(net.w[0], wimg, kLfCin[0], kLfCout[0],
                                        (9 * kLfCin[0] + 63) / 64);
  if (cudaGetLastError() != cudaSuccess) return -2;
  return lf_tma_prepare(net, wimg + lf_l0_wimg_bytes(), st);
}

// Forward pass: layer 1 (8 -> 32, per-pixel gather) into the padded grid
// act1p, layers 2 and 3 TMA-fed from the padded grids (dsax_lflag_tma.cu),
// then the 64 -> 1 tap sum and the mask.
int lf_tc_forward(const LfNet &net, const LfTcBuffers &bufs, int B, int H, int W, int guard,
                  const LfPerm &perm, int num_sms, int *err, uint64_t wait_limit_ns,
                  cudaStream_t st) {
  static_assert(kLfCin[0] == 8 && kLfCout[0] == 32 && kLfCin[3] == 64 && kLfCout[3] == 1,
                "tensor-core path is written for the 8-32-64-64-1 net");
  LfTcArgs a{};
  a.B = B; a.H = H; a.W = W; a.err = err; a.wait_limit_ns = wait_limit_ns;
  a.in = bufs.feat_bf16; a.wimg = bufs.wimg; a.bias = net.b[0]; a.out = bufs.act1p;
  a.pad_out = 1;
  int e = lf_pad_borders(bufs.act1p, B, H, W, st);
  e |= lf_pad_borders(bufs.act2p, B, H, W, st);
  e |= conv_tc_launch<8, 32, false>(a, num_sms, st);
  e |= lf_tma_layers23(net, bufs.wimg + lf_l0_wimg_bytes(), bufs.act1p, bufs.act2p, bufs.z9, B, H, W,
                       num_sms, err, wait_limit_ns, st);
  lf_tapsum_kernel<<<1024, 256, 0, st>>>(bufs.z9, net.b[3], bufs.logit, bufs.mask, B, H, W, guard,
                                         0.0f, perm);
  if (cudaGetLastError() != cudaSuccess) e = -2;
  return e;
}

}  // namespace dsax

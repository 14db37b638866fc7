// dsax_lflag_tc.cu -- learned-flagger inference on sm_100a tensor cores:
// the weight images, the forward pass over the three TMA-fed tcgen05 layers
// (dsax_lflag_tma.cu), the 64 -> 1 tap sum and the mask.
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_lflag.h"
#include "dsax_ptx.cuh"

namespace dsax {

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

// Forward pass over the zero-bordered grids: layer 1 (8 -> 32) from the
// feature grid into act1p, layers 2 and 3 from act1p / act2p to the tap
// projections (dsax_lflag_tma.cu), then the 64 -> 1 tap sum and the mask.
int lf_tc_forward(const LfNet &net, const LfTcBuffers &bufs, int B, int H, int W, int guard,
                  const LfPerm &perm, bool zero_borders, int num_sms, int *err,
                  uint64_t wait_limit_ns, cudaStream_t st) {
  static_assert(kLfCin[3] == 64 && kLfCout[3] == 1, "64 -> 1 last layer");
  int e = 0;
  if (zero_borders) {   // the grids' borders, once per geometry
    e |= lf_pad_borders(bufs.featp, B, H, W, 1, st);
    e |= lf_pad_borders(bufs.act1p, B, H, W, 8, st);
    e |= lf_pad_borders(bufs.act2p, B, H, W, 8, st);
  }
  e |= lf_tma_layer1(net, bufs.wimg, bufs.featp, bufs.act1p, B, H, W, num_sms, err, wait_limit_ns, st);
  e |= lf_tma_layers23(net, bufs.wimg + lf_l0_wimg_bytes(), bufs.act1p, bufs.act2p, bufs.z9, B, H, W,
                       num_sms, err, wait_limit_ns, st);
  lf_tapsum_kernel<<<1024, 256, 0, st>>>(bufs.z9, net.b[3], bufs.logit, bufs.mask, B, H, W, guard,
                                         0.0f, perm);
  if (cudaGetLastError() != cudaSuccess) e = -2;
  return e;
}

}  // namespace dsax

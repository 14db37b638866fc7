// dsax_lflag.cu -- the learned RFI flagger: a 4-layer 3x3 conv net
// (8 -> 32 -> 64 -> 64 -> 1 channels, ReLU, 58,337 parameters) over a
// downsampled Stokes-I spectrogram, trained on the plain flagger's masks.
// No reference counterpart: the reference flags only with the statistics
// of src/gpu_flagger.cu, which stay the label source, judge and fallback.
//
// Kernels (NHWC activations, FP32):
//   (features: the plain flagger's staged statistics pass plus
//    lf_stat_features_kernel, both in dsax_flag.cu)
//   lf_labels_kernel   : plain-flagger masks -> pixel labels on the H x C grid
//   conv3x3_kernel     : out = conv(in, w) + b (+ReLU); with flipped and
//                        transposed weights it is also the data gradient,
//                        the ReLU mask of the layer fused into its input load
//   conv3x3_wgrad_kernel + lf_reduce_kernel : weight/bias gradients,
//                        per-chunk partials reduced in a fixed order
//   lf_bce_kernel      : weighted BCE-with-logits loss and d/dlogits
//   lf_adam_kernel     : Adam update of the FP32 master weights
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_lflag.h"

namespace dsax {

__device__ __forceinline__ float slog(float v) { return copysignf(log1pf(fabsf(v)), v); }

// pixel label = chan flag, or (any ts flag in the tds samples and inside the
// guard band)
__global__ void lf_labels_kernel(const uint8_t *chanmask, const uint8_t *tsmask, uint8_t *L,
                                 int B, int T, int C, int tds, int guard) {
  const int H = T / tds;
  const int64_t n = (int64_t)B * H * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t bh = i / C;
    const int h = (int)(bh % H), b = (int)(bh / H);
    uint8_t v = chanmask[b * C + c];
    if (!v && c >= guard && c < C - guard) {
      const uint8_t *ts = tsmask + (int64_t)b * T + (int64_t)h * tds;
      for (int k = 0; k < tds; ++k) v |= ts[k];
    }
    L[i] = v ? 1 : 0;
  }
}

// ---------------------------------------------------------------- conv3x3
// out[b][y][x][co] = bias[co] + sum_{ky,kx,ci} wt[ky*3+kx][ci][co] *
//                    in'[b][y+ky-1][x+kx-1][ci]     (zero padding)
// in' = in * (gate > 0) when gate != null (ReLU backward of the layer below).
// Thread = 4 consecutive x pixels of one row x CO_T output channels.
template <int CIN, int COUT, int CO_T, bool RELU>
__global__ void __launch_bounds__(256) conv3x3_kernel(const float *__restrict__ in,
                                                      const float *__restrict__ gate,
                                                      const float *__restrict__ wt,
                                                      const float *__restrict__ bias,
                                                      float *__restrict__ out, int B, int H, int W) {
  constexpr int TH = 4;                          // rows per CTA
  extern __shared__ float tile[];                // [TH+2][W+2][CIN]
  const int nrt = (H + TH - 1) / TH;
  const int b = blockIdx.x / nrt, y0 = (blockIdx.x % nrt) * TH;
  const int WP = W + 2;
  for (int i = threadIdx.x; i < (TH + 2) * WP * CIN; i += blockDim.x) {
    const int ci = i % CIN, xx = (i / CIN) % WP, yy = i / (CIN * WP);
    const int gy = y0 + yy - 1, gx = xx - 1;
    float v = 0.f;
    if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
      const int64_t gi = (((int64_t)b * H + gy) * W + gx) * CIN + ci;
      v = in[gi];
      if (gate && !(gate[gi] > 0.f)) v = 0.f;
    }
    tile[i] = v;
  }
  __syncthreads();
  const int ngx = W / 4;                          // pixel groups per row
  const int nunits = TH * ngx * (COUT / CO_T);
  for (int u = threadIdx.x; u < nunits; u += blockDim.x) {
    const int cog = u / (TH * ngx);
    const int rem = u % (TH * ngx);
    const int ty = rem / ngx, gx4 = (rem % ngx) * 4;
    if (y0 + ty >= H) continue;
    float acc[4][CO_T];
#pragma unroll
    for (int j = 0; j < CO_T; ++j) {
      const float bb = bias ? bias[cog * CO_T + j] : 0.f;
#pragma unroll
      for (int p = 0; p < 4; ++p) acc[p][j] = bb;
    }
    for (int ky = 0; ky < 3; ++ky)
      for (int kx = 0; kx < 3; ++kx) {
        const float *trow = tile + ((ty + ky) * WP + gx4 + kx) * CIN;
        const float *wrow = wt + (int64_t)(ky * 3 + kx) * CIN * COUT + cog * CO_T;
#pragma unroll 4
        for (int ci = 0; ci < CIN; ++ci) {
          float wv[CO_T];
#pragma unroll
          for (int j = 0; j < CO_T; ++j) wv[j] = __ldg(wrow + (int64_t)ci * COUT + j);
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const float v = trow[p * CIN + ci];
#pragma unroll
            for (int j = 0; j < CO_T; ++j) acc[p][j] = fmaf(v, wv[j], acc[p][j]);
          }
        }
      }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      float *o = out + (((int64_t)b * H + y0 + ty) * W + gx4 + p) * COUT + cog * CO_T;
#pragma unroll
      for (int j = 0; j < CO_T; ++j) o[j] = RELU ? fmaxf(acc[p][j], 0.f) : acc[p][j];
    }
  }
}

// Weight gradient partials: for a chunk of RPC pixel rows, thread r in
// [0, 9*CIN] (r == 9*CIN is the bias) accumulates, for CO_T output
// channels, sum over the chunk's pixels of dz[co] * patch[r].
template <int CIN, int CO_T>
__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(const float *__restrict__ in,
                                                            const float *__restrict__ dz,
                                                            const float *__restrict__ gate,
                                                            int cout, float *part, int B, int H,
                                                            int W, int rpc) {
  extern __shared__ float wsh[];                 // tile [rpc+2][W+2][CIN] then dz [rpc*W][CO_T]
  const int nrc = (H + rpc - 1) / rpc;
  const int chunk = blockIdx.x;                  // (b, row chunk)
  const int cog = blockIdx.y;
  const int b = chunk / nrc, y0 = (chunk % nrc) * rpc;
  const int WP = W + 2;
  float *tile = wsh;
  float *dzs = wsh + (rpc + 2) * WP * CIN;
  for (int i = threadIdx.x; i < (rpc + 2) * WP * CIN; i += blockDim.x) {
    const int ci = i % CIN, xx = (i / CIN) % WP, yy = i / (CIN * WP);
    const int gy = y0 + yy - 1, gx = xx - 1;
    tile[i] = (gy >= 0 && gy < H && gx >= 0 && gx < W)
                  ? in[(((int64_t)b * H + gy) * W + gx) * CIN + ci]
                  : 0.f;
  }
  for (int i = threadIdx.x; i < rpc * W * CO_T; i += blockDim.x) {
    const int j = i % CO_T, px = i / CO_T;
    const int yy = px / W, xx = px % W;
    float d = 0.f;
    if (y0 + yy < H) {
      const int64_t gi = (((int64_t)b * H + y0 + yy) * W + xx) * cout + cog * CO_T + j;
      d = dz[gi];
      if (gate && !(gate[gi] > 0.f)) d = 0.f;
    }
    dzs[i] = d;
  }
  __syncthreads();
  const int nr = 9 * CIN + 1;
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    float acc[CO_T];
#pragma unroll
    for (int j = 0; j < CO_T; ++j) acc[j] = 0.f;
    const int tap = r / CIN, ci = r % CIN, ky = tap / 3, kx = tap % 3;
    const bool isb = r == 9 * CIN;
    for (int yy = 0; yy < rpc; ++yy)
      for (int xx = 0; xx < W; ++xx) {
        const float v = isb ? 1.f : tile[((yy + ky) * WP + xx + kx) * CIN + ci];
        const float *d = dzs + (yy * W + xx) * CO_T;
#pragma unroll
        for (int j = 0; j < CO_T; ++j) acc[j] = fmaf(v, d[j], acc[j]);
      }
    float *pp = part + (int64_t)chunk * nr * cout + (int64_t)r * cout + cog * CO_T;
#pragma unroll
    for (int j = 0; j < CO_T; ++j) pp[j] = acc[j];
  }
}

// Sums the per-chunk partials [nchunk][9*CIN+1][COUT] in chunk order and
// writes the gradients in the parameter layout W[co][ky][kx][ci], b[co].
__global__ void lf_reduce_kernel(const float *part, int nchunk, int cin, int cout, float *gw,
                                 float *gb) {
  const int nr = 9 * cin + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nr * cout; i += gridDim.x * blockDim.x) {
    const int r = i / cout, co = i % cout;
    float s = 0.f;
    for (int k = 0; k < nchunk; ++k) s += part[((int64_t)k * nr + r) * cout + co];
    if (r == 9 * cin) gb[co] = s;
    else {
      const int tap = r / cin, ci = r % cin;
      gw[((int64_t)co * 9 + tap) * cin + ci] = s;
    }
  }
}

// W[co][tap][ci] -> forward layout wt[tap][ci][co]; flip=1 builds the data-
// gradient layout wt[tap'][co][ci] with tap' = 8 - tap.
__global__ void lf_wlayout_kernel(const float *w, float *wt, int cin, int cout, int flip) {
  const int n = 9 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i / (9 * cin), tap = (i / cin) % 9, ci = i % cin;
    if (!flip) wt[((int64_t)tap * cin + ci) * cout + co] = w[i];
    else wt[((int64_t)(8 - tap) * cout + co) * cin + ci] = w[i];
  }
}

// Weighted BCE-with-logits over valid pixels (guard band excluded), mean;
// writes dlogits and accumulates the loss sum and the valid count.
__global__ void lf_bce_kernel(const float *z, const uint8_t *L, float *dz, double *loss_acc,
                              int B, int H, int W, int guard, float pos_weight, float inv_n) {
  const int64_t n = (int64_t)B * H * W;
  double local = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % W);
    const bool valid = c >= guard && c < W - guard;
    const float zi = z[i], y = L[i] ? 1.f : 0.f;
    const float wgt = valid ? (y > 0.f ? pos_weight : 1.f) : 0.f;
    const float sp = fmaxf(zi, 0.f) + log1pf(expf(-fabsf(zi)));
    local += (double)(wgt * (sp - y * zi));
    const float sig = 1.f / (1.f + expf(-zi));
    dz[i] = wgt * (sig - y) * inv_n;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_acc, local);
}

__global__ void lf_adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr,
                               float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// sigmoid(z) > 0.5  <=>  z > 0; guard band never flagged.
// Pixel mask from the logits; the permanently flagged channels of the
// plain flagger's configuration (inside the guard band) are always set.
__global__ void lf_mask_kernel(const float *z, uint8_t *mask, int64_t n, int W, int guard,
                               float thresh_logit, LfPerm perm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % W);
    const bool inside = c >= guard && c < W - guard;
    bool pm = false;
    for (int k = 0; k < perm.n; ++k) pm |= perm.ch[k] == c;
    mask[i] = (inside && (z[i] > thresh_logit || pm)) ? 1 : 0;
  }
}

// ---------------------------------------------------------------- launchers
namespace {

template <int CIN, int COUT, int CO_T, bool RELU>
int conv_launch(const float *in, const float *gate, const float *wt, const float *bias, float *out,
                int B, int H, int W, cudaStream_t st) {
  const size_t sh = (size_t)6 * (W + 2) * CIN * sizeof(float);
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, conv3x3_kernel<CIN, COUT, CO_T, RELU>, 200 * 1024) != cudaSuccess)
    return -2;
  const int grid = B * ((H + 3) / 4);
  conv3x3_kernel<CIN, COUT, CO_T, RELU><<<grid, 256, sh, st>>>(in, gate, wt, bias, out, B, H, W);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <int CIN, int CO_T>
int wgrad_launch(const float *in, const float *dz, const float *gate, int cout, float *part, int B,
                 int H, int W, int rpc, cudaStream_t st) {
  const size_t sh = ((size_t)(rpc + 2) * (W + 2) * CIN + (size_t)rpc * W * CO_T) * sizeof(float);
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, conv3x3_wgrad_kernel<CIN, CO_T>, 200 * 1024) != cudaSuccess) return -2;
  dim3 grid(B * ((H + rpc - 1) / rpc), cout / CO_T);
  conv3x3_wgrad_kernel<CIN, CO_T><<<grid, 256, sh, st>>>(in, dz, gate, cout, part, B, H, W, rpc);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace


int lf_labels(const uint8_t *cm, const uint8_t *tm, uint8_t *L, int B, int T, int C, int tds,
              int guard, cudaStream_t st) {
  lf_labels_kernel<<<1024, 256, 0, st>>>(cm, tm, L, B, T, C, tds, guard);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Forward through the 4 layers: acts[0] = features, acts[1..3] post-ReLU,
// acts[4] = logits.  wt[l] are forward-layout weights.
int lf_forward(const LfNet &net, float *const acts[5], int B, int H, int W, cudaStream_t st) {
  int rc = 0;
  rc |= conv_launch<8, 32, 16, true>(acts[0], nullptr, net.wt[0], net.b[0], acts[1], B, H, W, st);
  rc |= conv_launch<32, 64, 16, true>(acts[1], nullptr, net.wt[1], net.b[1], acts[2], B, H, W, st);
  rc |= conv_launch<64, 64, 16, true>(acts[2], nullptr, net.wt[2], net.b[2], acts[3], B, H, W, st);
  rc |= conv_launch<64, 1, 1, false>(acts[3], nullptr, net.wt[3], net.b[3], acts[4], B, H, W, st);
  return rc;
}

int lf_prepare_weights(const LfNet &net, cudaStream_t st) {
  static const int cin[4] = {8, 32, 64, 64}, cout[4] = {32, 64, 64, 1};
  for (int l = 0; l < 4; ++l) {
    lf_wlayout_kernel<<<64, 256, 0, st>>>(net.w[l], net.wt[l], cin[l], cout[l], 0);
    lf_wlayout_kernel<<<64, 256, 0, st>>>(net.w[l], net.wf[l], cin[l], cout[l], 1);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Backward from dlogits d4 [B][H][W][1]: fills net.gw / net.gb.  The ReLU
// masks are applied as gates (acts[l] > 0) inside the kernels that read the
// gradients.  d_a / d_b: scratch of B*H*W*64 floats each; part: partials.
int lf_backward(const LfNet &net, float *const acts[5], float *d4, float *d_a, float *d_b,
                float *part, int B, int H, int W, cudaStream_t st) {
  const int rpc = 4;
  const int nchunk = B * ((H + rpc - 1) / rpc);
  int rc = 0;
  // layer 4 (64 -> 1, no ReLU)
  rc |= wgrad_launch<64, 1>(acts[3], d4, nullptr, 1, part, B, H, W, rpc, st);
  lf_reduce_kernel<<<64, 256, 0, st>>>(part, nchunk, 64, 1, net.gw[3], net.gb[3]);
  rc |= conv_launch<1, 64, 16, false>(d4, nullptr, net.wf[3], nullptr, d_a, B, H, W, st);
  // layer 3 (64 -> 64): dz3 = d_a * (acts[3] > 0)
  rc |= wgrad_launch<64, 16>(acts[2], d_a, acts[3], 64, part, B, H, W, rpc, st);
  lf_reduce_kernel<<<256, 256, 0, st>>>(part, nchunk, 64, 64, net.gw[2], net.gb[2]);
  rc |= conv_launch<64, 64, 16, false>(d_a, acts[3], net.wf[2], nullptr, d_b, B, H, W, st);
  // layer 2 (32 -> 64): dz2 = d_b * (acts[2] > 0)
  rc |= wgrad_launch<32, 16>(acts[1], d_b, acts[2], 64, part, B, H, W, rpc, st);
  lf_reduce_kernel<<<256, 256, 0, st>>>(part, nchunk, 32, 64, net.gw[1], net.gb[1]);
  rc |= conv_launch<64, 32, 16, false>(d_b, acts[2], net.wf[1], nullptr, d_a, B, H, W, st);
  // layer 1 (8 -> 32): dz1 = d_a * (acts[1] > 0)
  rc |= wgrad_launch<8, 16>(acts[0], d_a, acts[1], 32, part, B, H, W, rpc, st);
  lf_reduce_kernel<<<64, 256, 0, st>>>(part, nchunk, 8, 32, net.gw[0], net.gb[0]);
  return rc ? -2 : (cudaGetLastError() == cudaSuccess ? 0 : -2);
}

size_t lf_part_floats(int B, int H) {
  const int rpc = 4;
  return (size_t)B * ((H + rpc - 1) / rpc) * (9 * 64 + 1) * 64;
}

int lf_bce(const float *z, const uint8_t *L, float *dz, double *loss_acc, int B, int H, int W,
           int guard, float pos_weight, float inv_n, cudaStream_t st) {
  lf_bce_kernel<<<512, 256, 0, st>>>(z, L, dz, loss_acc, B, H, W, guard, pos_weight, inv_n);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int lf_adam(LfNet &net, float lr, cudaStream_t st) {
  net.step += 1;
  net.version += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)net.step), c2 = 1.f - powf(b2, (float)net.step);
  lf_adam_kernel<<<128, 256, 0, st>>>(net.params, net.grads, net.m, net.v, lf_nparams(), lr, b1, b2,
                                      1e-8f, c1, c2);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int lf_mask(const float *z, uint8_t *mask, int64_t n, int W, int guard, float thresh_logit,
            const LfPerm &perm, cudaStream_t st) {
  lf_mask_kernel<<<1024, 256, 0, st>>>(z, mask, n, W, guard, thresh_logit, perm);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

// dsax_lflag.h -- learned-flagger network state and kernel launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dsax {

constexpr int kLfLayers = 4;
constexpr int kLfCin[kLfLayers] = {8, 32, 64, 64};
constexpr int kLfCout[kLfLayers] = {32, 64, 64, 1};

// Offsets of layer l's weights / bias in the flat parameter vector:
// for each layer W[co][3][3][ci] then b[co].
inline int lf_w_offset(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += kLfCout[k] * 9 * kLfCin[k] + kLfCout[k];
  return o;
}
inline int lf_b_offset(int l) { return lf_w_offset(l) + kLfCout[l] * 9 * kLfCin[l]; }
inline int lf_nparams() { return lf_w_offset(kLfLayers); }

struct LfNet {
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;  // flat, FP32
  float *w[kLfLayers] = {}, *b[kLfLayers] = {};      // views into params
  float *gw[kLfLayers] = {}, *gb[kLfLayers] = {};    // views into grads
  float *wt[kLfLayers] = {}, *wf[kLfLayers] = {};    // forward / data-gradient layouts
  int step = 0;
  unsigned version = 0;   // bumped whenever the parameters change
};

// Permanently flagged channels of the plain flagger's configuration.
struct LfPerm {
  int n = 0;
  int ch[8] = {};
};

int lf_labels(const uint8_t *cm, const uint8_t *tm, uint8_t *L, int B, int T, int C, int tds,
              int guard, cudaStream_t st);
int lf_prepare_weights(const LfNet &net, cudaStream_t st);
int lf_forward(const LfNet &net, float *const acts[5], int B, int H, int W, cudaStream_t st);
int lf_backward(const LfNet &net, float *const acts[5], float *d4, float *d_a, float *d_b,
                float *part, int B, int H, int W, cudaStream_t st);
int lf_bce(const float *z, const uint8_t *L, float *dz, double *loss_acc, int B, int H, int W,
           int guard, float pos_weight, float inv_n, cudaStream_t st);
int lf_adam(LfNet &net, float lr, cudaStream_t st);
int lf_mask(const float *z, uint8_t *mask, int64_t n, int W, int guard, float thresh_logit,
            const LfPerm &perm, cudaStream_t st);
size_t lf_part_floats(int B, int H);   // partial-gradient scratch size

// Tensor-core inference (dsax_lflag_tc.cu).
struct LfTcBuffers {
  uint16_t *featp = nullptr;            // padded grid [B][H+2][W+2][8] BF16 features
  uint16_t *act1p = nullptr;            // padded grid [B][H+2][W+2][64] BF16 (layer-1 output)
  uint16_t *act2p = nullptr;            // padded grid [B][H+2][W+2][64] BF16 (layer-2 output)
  float *z9 = nullptr;                  // [9][npx] last-layer tap projections
  float *logit = nullptr;               // [npx] (may be null)
  uint8_t *mask = nullptr;              // [npx]
  const uint8_t *wimg = nullptr;        // weight images of layers 0..2 (lf_tc_wimg_bytes)
};
size_t lf_tc_wimg_bytes();
// Padded-grid layers (dsax_lflag_tma.cu).
size_t lf_pad_bytes(int B, int H, int W);   // one padded activation grid
size_t lf_tma_wimg_bytes();
int lf_tma_prepare(const LfNet &net, uint8_t *wimg, cudaStream_t st);
size_t lf_feat_pad_bytes(int B, int H, int W);   // the padded feature grid
int lf_pad_borders(uint16_t *grid, int B, int H, int W, int chunks, cudaStream_t st);
int lf_tma_layer1(const LfNet &net, const uint8_t *wimg, const uint16_t *featp, uint16_t *act1p,
                  int B, int H, int W, int num_sms, int *err, uint64_t wait_limit_ns,
                  cudaStream_t st);
int lf_tma_layers23(const LfNet &net, const uint8_t *wimg, const uint16_t *act1p, uint16_t *act2p,
                    float *z9, int B, int H, int W, int num_sms, int *err, uint64_t wait_limit_ns,
                    cudaStream_t st);
int lf_tc_prepare(const LfNet &net, uint8_t *wimg, cudaStream_t st);
int lf_tc_forward(const LfNet &net, const LfTcBuffers &bufs, int B, int H, int W, int guard,
                  const LfPerm &perm, bool zero_borders, int num_sms, int *err,
                  uint64_t wait_limit_ns, cudaStream_t st);

}  // namespace dsax

// dsax_ctx.h -- the context object behind the opaque dsax_ctx handle.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_lflag.h"

namespace dsax {

// Slots of dsax_ctx::aux.
enum {
  AUX_WIMG_BF16 = 0,  // beamformer weight operand image (BF16)
  AUX_WIMG_FP8 = 1,   // beamformer weight operand image (FP8 E4M3)
  AUX_BEAM_U8 = 2,    // host-mode staging: Stokes-I uint8
  AUX_BEAM_F32 = 3,   // host-mode staging: FP32 power
  AUX_FLAG_STATS = 4, // flagger statistics + counts
  AUX_FLAG_X = 5,     // host-mode staging: filterbank + oldspec
  AUX_FLAG_MASK = 6,  // host-mode staging: masks
  AUX_REORDERED = 7,  // corner-turned block for the two-pass correlator path
  AUX_REORDER_OUT = 8,  // host-mode staging for dsax_reorder output
  AUX_LF_STATE = 9,     // learned flagger: params, grads, Adam m, v
  AUX_LF_WLAYOUT = 10,  // learned flagger: forward / data-gradient weight layouts
  AUX_LF_SCRATCH = 11,  // learned flagger: activations, gradients, partials
  AUX_BATCH_SCRATCH = 12,  // batch: corner-turned block, beam filterbank, flag statistics
  AUX_TUNE = 13,           // autotuner: synthetic block + visibilities
  AUX_LF_TCW = 14,         // learned flagger: BF16 weight images of the tensor-core path
  AUX_PIPE = 15,           // correlate_many: double-buffered inputs, corner turns, visibilities
  AUX_AGC = 16,            // beamformer AGC: bandpass history, scales, per-beam power
  AUX_EXTRACT = 17,        // correlate_extract: device visibilities, input, product
  AUX_LF_PAD = 18,         // learned flagger: two zero-bordered activation grids
  AUX_COUNT = 20
};

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

class DeviceGuard {
 public:
  explicit DeviceGuard(int dev);
  ~DeviceGuard();

 private:
  int prev_ = -1;
};

int set_error(dsax_ctx *c, int code, const char *fmt, ...);
int cuda_check(dsax_ctx *c, cudaError_t e, const char *what);
int ensure_buffer(dsax_ctx *c, DevBuf &b, size_t nbytes, const char *what);
int check_device_error(dsax_ctx *c);
void release_batch_plan(dsax_ctx *c);
bool aligned16(const void *p);

}  // namespace dsax

struct dsax_ctx {
  dsax_config cfg{};
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int *d_err = nullptr;   // device error word written by bounded waits
  int *h_err = nullptr;   // pinned readback slot
  dsax::DevBuf in_buf;    // host-mode staging: input block
  dsax::DevBuf vis_buf;   // host-mode staging: visibilities
  dsax::DevBuf aux[dsax::AUX_COUNT];   // per-stage buffers, indexed by dsax::AUX_*
  int agc_on = 0;         // beamformer uses (and updates) the AGC bandpass state
  float fp8_pscale = 1.0f;   // 2^-2E: FP8 operands carry 2^E in every product
  int fp8_shift = 0;         // FP8 data get a nonzero per-antenna exponent
  size_t fp8_img_bytes = 0;  // FP8 weight image; the 64 exponent bytes follow it
  int weights_ready = 0;
  int weights_nchan = 0;      // channels covered by the weight image
  void *batch_plan = nullptr; // captured batch graph (dsax_batch.cu)
  // correlate_many pipeline: side streams (copy in, corner turn, copy out)
  // and per-buffer events, created on first use
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t pev[9] = {};
  // dsax_run_batch: the beamform + flag chain's stream and its fork/join
  // events, created on first use
  cudaStream_t bstream = nullptr;
  cudaEvent_t bev[2] = {};
  dsax::LfNet lf_storage;
  unsigned lf_wimg_version = ~0u;   // parameter version the inference weight images hold
  int lf_pad_geom[3] = {0, 0, 0};   // (B, H, W) whose grid borders are zero
  dsax::LfNet *lf = &lf_storage;
  char errmsg[512] = {0};

  void release_all() {
    in_buf.release();
    vis_buf.release();
    for (auto &b : aux) b.release();
  }
};

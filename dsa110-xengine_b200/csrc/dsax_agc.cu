// dsax_agc.cu -- the beamformer's automatic gain control (bandpass) on the
// GPU: from each block's per-beam power, the per-beam uint8 scale used for
// the next block.
//
// Restates the host logic of src/dsaX_beamformer.cu: badder (:79-112) and
// calc_allbp (:482-494) give the block's total power per beam; the history
// of the last NBP = 8 blocks (:1022-1024); ret_med_bp (:506-513) for the
// first NBP blocks (every beam gets the median over beams, the first
// block's median is frozen as medbp); ret_many_bp (:515-530) afterwards
// (mean over the history, beams more than 10 % off medbp reset to medbp);
// with AGC off the frozen median is used throughout (:1055-1056); finally
// bp = 2.5 * 128 / (bp / (48 * nints)) (:1057-1062).  The first block's
// scale is 0 (the reference writes zeros for it, :1035-1036).
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

namespace dsax {

namespace {

// Device state: header, then history [NBP][nbeam], scale [nbeam], power [nbeam].
struct AgcHdr {
  int started;   // 0 before the first block, then 1, 2 once the history is in use
  int bpctr;     // blocks seen
  int agc;       // 1: adaptive; 0: the first block's median throughout
  int nbeam;
  float medbp;
  float pad[3];
};

constexpr int kAgcThreads = 512;

size_t up256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

size_t agc_state_bytes(int nbeam) {
  return up256(sizeof(AgcHdr)) + up256(sizeof(float) * (size_t)(kAgcNbp + 2) * nbeam);
}

float *agc_scale_ptr(void *state, int nbeam) {
  return reinterpret_cast<float *>(static_cast<uint8_t *>(state) + up256(sizeof(AgcHdr))) +
         (size_t)kAgcNbp * nbeam;
}

float *agc_power_ptr(void *state, int nbeam) { return agc_scale_ptr(state, nbeam) + nbeam; }

// Value at sorted position k of v[0..n) (rank counting, ties by index).
__device__ float block_select(const float *v, int n, int k, float *slot) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = v[i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const float y = v[j];
      r += (y < x) || (y == x && j < i);
    }
    if (r == k) *slot = x;
  }
  __syncthreads();
  const float s = *slot;
  __syncthreads();
  return s;
}

__global__ void __launch_bounds__(kAgcThreads) agc_update_kernel(AgcHdr *h, float *hist,
                                                                 float *scale, float *power,
                                                                 int nbeam, int ngrp, int nints) {
  extern __shared__ float bp[];   // [nbeam]
  __shared__ float slot;
  const int started = h->started, bpctr = h->bpctr, agc = h->agc;
  float *row = hist + (size_t)(bpctr % kAgcNbp) * nbeam;
  for (int b = threadIdx.x; b < nbeam; b += blockDim.x) {
    bp[b] = power[b];
    row[b] = power[b];
    power[b] = 0.0f;   // accumulation of the next block starts from zero
  }
  __syncthreads();
  float medbp = h->medbp;
  bool from_history = false;
  if (started == 0 || bpctr < kAgcNbp) {
    // ret_med_bp: every beam gets 0.5 (sorted[n/2 - 1] + sorted[n/2])
    const float lo = block_select(bp, nbeam, nbeam / 2 - 1, &slot);
    const float hi = block_select(bp, nbeam, nbeam / 2, &slot);
    const float med = 0.5f * (lo + hi);
    if (started == 0) medbp = med;
    for (int b = threadIdx.x; b < nbeam; b += blockDim.x) bp[b] = med;
  } else {
    from_history = true;
    for (int b = threadIdx.x; b < nbeam; b += blockDim.x) {
      float s = 0.0f;
      for (int j = 0; j < kAgcNbp; ++j) s += hist[(size_t)j * nbeam + b];
      float v = (float)((double)s / (double)kAgcNbp);
      if (fabs((double)(v - medbp)) / (double)medbp > 0.1) v = medbp;
      bp[b] = v;
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbeam; b += blockDim.x) {
    float v = agc ? bp[b] : medbp;
    if (v != 0.0f) {
      v = (float)((double)v / ((double)ngrp * nints));   // mean power per (channel group, int)
      v = (float)(2.5 * 128.0 / (double)v);
    }
    scale[b] = v;
  }
  if (threadIdx.x == 0) {
    h->medbp = medbp;
    h->started = started == 0 ? 1 : (from_history ? 2 : started);
    h->bpctr = bpctr + 1;
  }
}

int launch_agc_update(void *state, int nbeam, int ngrp, int nints, cudaStream_t st) {
  AgcHdr *h = static_cast<AgcHdr *>(state);
  float *hist = reinterpret_cast<float *>(static_cast<uint8_t *>(state) + up256(sizeof(AgcHdr)));
  agc_update_kernel<<<1, kAgcThreads, sizeof(float) * nbeam, st>>>(
      h, hist, agc_scale_ptr(state, nbeam), agc_power_ptr(state, nbeam), nbeam, ngrp, nints);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

__global__ void agc_reset_kernel(AgcHdr *h, int agc, int nbeam, float *rest, int nrest) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    h->started = 0;
    h->bpctr = 0;
    h->agc = agc;
    h->nbeam = nbeam;
    h->medbp = 0.0f;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrest; i += gridDim.x * blockDim.x)
    rest[i] = 0.0f;
}

}  // namespace dsax

using namespace dsax;

extern "C" int dsax_agc_enable(dsax_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 2) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  if (mode == 0) {
    c->agc_on = 0;
    return DSAX_OK;
  }
  const int nbeam = c->cfg.nbeam;
  if (nbeam < 2 || nbeam > 4096) return set_error(c, DSAX_ERR_ARG, "AGC needs 2..4096 beams");
  int rc = ensure_buffer(c, c->aux[AUX_AGC], agc_state_bytes(nbeam), "AGC state");
  if (rc != DSAX_OK) return rc;
  AgcHdr *h = static_cast<AgcHdr *>(c->aux[AUX_AGC].ptr);
  float *rest = reinterpret_cast<float *>(static_cast<uint8_t *>(c->aux[AUX_AGC].ptr) +
                                          up256(sizeof(AgcHdr)));
  agc_reset_kernel<<<16, 256, 0, c->stream>>>(h, mode == 1 ? 1 : 0, nbeam, rest,
                                             (kAgcNbp + 2) * nbeam);
  if (cudaGetLastError() != cudaSuccess) return cuda_check(c, cudaGetLastError(), "AGC reset");
  c->agc_on = 1;
  return DSAX_OK;
}

extern "C" int dsax_agc_state(dsax_ctx *c, float *scale, int *started, int *blocks) {
  if (!c || !c->agc_on) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const int nbeam = c->cfg.nbeam;
  AgcHdr h{};
  cudaError_t e = cudaMemcpyAsync(&h, c->aux[AUX_AGC].ptr, sizeof(h), cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess && scale)
    e = cudaMemcpyAsync(scale, agc_scale_ptr(c->aux[AUX_AGC].ptr, nbeam), sizeof(float) * nbeam,
                        cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "AGC state readback");
  int rc = dsax_sync(c);
  if (rc != DSAX_OK) return rc;
  if (started) *started = h.started;
  if (blocks) *blocks = h.bpctr;
  return DSAX_OK;
}

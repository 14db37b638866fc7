// dsax_tune.cu -- autotuner: times the interchangeable kernel variants of
// a stage on the context's own geometry and device, keeps the fastest in
// the context, and reports every timing.  Candidates for the captured-block
// correlator (corr_path): (1) one fused kernel on the captured layout,
// (2) corner turn to the REORDER layout + row-load correlator, (3) corner
// turn to channel-major streams + correlator fed by direct coalesced loads,
// (4) the same correlator fed by one bulk copy per 64-packet stage and
// unpacked by 8 warps, (5) as 4 with 16 unpack warps, (6) no corner turn:
// the captured block read directly by clusters of four channel CTAs, (7) as
// 6 with 16 unpack warps.  Candidates for the beamformer: (1) one CTA per
// 64-beam tile (bf_path 1), (2-5) CTA pairs sharing a cta_group::2 MMA
// (bf_path 2) with stage parameters bf_variant 1-4 (TMEM loads in flight
// per epilogue wait x raw staging slots).
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace {

__global__ void fill_pattern(uint8_t *p, size_t n, uint32_t seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    p[i] = (uint8_t)h;
  }
}

}  // namespace

extern "C" int dsax_autotune(dsax_ctx *c, int reps, float *times_ms, int ntimes, int *best_path) {
  if (!c || reps < 1) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nvis = dsax_vis_bytes(&c->cfg);
  int rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_TUNE], nin + nvis + 256, "autotune block")) != DSAX_OK)
    return rc;
  uint8_t *blk = static_cast<uint8_t *>(c->aux[AUX_TUNE].ptr);
  float *vis = reinterpret_cast<float *>(blk + ((nin + 255) & ~(size_t)255));
  fill_pattern<<<1024, 256, 0, c->stream>>>(blk, nin, 12345u);
  const int saved = c->cfg.corr_path;
  constexpr int kNumPaths = 7;
  const int paths[kNumPaths] = {1, 2, 3, 4, 5, 6, 7};
  float best = 1e30f;
  int bestp = 4;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int k = 0; k < kNumPaths; ++k) {
    c->cfg.corr_path = paths[k];
    for (int w = 0; w < 2; ++w)
      if ((rc = dsax_correlate_fmt(c, DSAX_FMT_CAPTURED, blk, vis, DSAX_MEM_DEVICE, 0)) != DSAX_OK)
        break;
    if (rc != DSAX_OK) break;
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps; ++r)
      if ((rc = dsax_correlate_fmt(c, DSAX_FMT_CAPTURED, blk, vis, DSAX_MEM_DEVICE, 0)) != DSAX_OK)
        break;
    cudaEventRecord(e1, c->stream);
    if (rc != DSAX_OK) break;
    if ((rc = dsax_sync(c)) != DSAX_OK) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if (times_ms && k < ntimes) times_ms[k] = ms;
    if (ms < best) { best = ms; bestp = paths[k]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != DSAX_OK) {
    c->cfg.corr_path = saved;
    return rc;
  }
  c->cfg.corr_path = bestp;
  if (best_path) *best_path = bestp;
  return DSAX_OK;
}

extern "C" int dsax_autotune_beamformer(dsax_ctx *c, int reps, float *times_ms, int ntimes,
                                        int *best_path) {
  if (!c || reps < 1) return DSAX_ERR_ARG;
  if (!c->weights_ready) return set_error(c, DSAX_ERR_ARG, "dsax_set_weights not called");
  DeviceGuard g(c->device);
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nout = dsax_beam_bytes(&c->cfg);
  int rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_TUNE], nin + nout + 256, "autotune block")) != DSAX_OK)
    return rc;
  uint8_t *blk = static_cast<uint8_t *>(c->aux[AUX_TUNE].ptr);
  uint8_t *beams = blk + ((nin + 255) & ~(size_t)255);
  fill_pattern<<<1024, 256, 0, c->stream>>>(blk, nin, 54321u);
  const int saved = c->cfg.bf_path, saved_v = c->cfg.bf_variant;
  constexpr int kNumCand = 5;
  const int paths[kNumCand] = {1, 2, 2, 2, 2};
  const int variants[kNumCand] = {0, 1, 2, 3, 4};
  float best = 1e30f;
  int bestk = 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int k = 0; k < kNumCand; ++k) {
    c->cfg.bf_path = paths[k];
    c->cfg.bf_variant = variants[k];
    for (int w = 0; w < 2; ++w)
      if ((rc = dsax_beamform(c, blk, beams, nullptr, DSAX_MEM_DEVICE)) != DSAX_OK) break;
    if (rc != DSAX_OK) break;
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps; ++r)
      if ((rc = dsax_beamform(c, blk, beams, nullptr, DSAX_MEM_DEVICE)) != DSAX_OK) break;
    cudaEventRecord(e1, c->stream);
    if (rc != DSAX_OK) break;
    if ((rc = dsax_sync(c)) != DSAX_OK) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if (times_ms && k < ntimes) times_ms[k] = ms;
    if (ms < best) { best = ms; bestk = k; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != DSAX_OK) {
    c->cfg.bf_path = saved;
    c->cfg.bf_variant = saved_v;
    return rc;
  }
  c->cfg.bf_path = paths[bestk];
  c->cfg.bf_variant = variants[bestk];
  if (best_path) *best_path = bestk + 1;
  return DSAX_OK;
}

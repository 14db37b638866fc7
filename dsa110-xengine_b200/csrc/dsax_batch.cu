// dsax_batch.cu -- many blocks in one submission: corner turn, correlate,
// beamform and flag each block of a batch (subband widths may differ per
// block), optionally captured once into a CUDA graph and replayed.  The
// correlation chain (HBM-bound corner turn, then the correlator) runs on the
// context stream and the beamform + flag chain (tensor-bound) on a second
// stream, forked from and joined back to the context stream, so that the
// two chains may overlap where one leaves SMs idle (both mostly fill the
// GPU, so the measured gain is within noise); each chain keeps its own
// scratch, so blocks within a chain stay in order.
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace {

struct BatchPlan {
  std::vector<dsax_block_desc> blocks;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// Enqueues one block's stages: correlation on sc, beamform + flag on sb.
int enqueue_block(dsax_ctx *c, const dsax_block_desc &d, uint8_t *scratch, float *fb,
                  float *fstats, cudaStream_t sc, cudaStream_t sb) {
  const dsax_config &cf = c->cfg;
  const int npkt = cf.npkt, nchan = d.nchan, ngrp = nchan / 8, ppo = cf.bf_pkt_per_out;
  const int nout = npkt / ppo;
  if (d.vis) {
    CorrArgs a{};
    a.in = static_cast<const uint8_t *>(d.blk);
    a.vis = d.vis;
    a.err = c->d_err;
    a.npkt = npkt;
    a.nant_in = cf.nant_in;
    a.nchan = nchan;
    a.wait_limit_ns = cf.wait_limit_ns;
    if (corr_path_fused(cf.corr_path) && captured_cluster_ok(a)) {
      // the correlator reads the captured block directly (no corner turn)
      if (launch_correlate_captured_cluster(a, sc, corr_path_unpack_warps(cf.corr_path)) != 0)
        return -2;
    } else {
      if (launch_reorder_chanmajor(static_cast<const uint8_t *>(d.blk), scratch, npkt, cf.nant_in,
                                   nchan, sc) != 0)
        return -2;
      a.in = scratch;
      a.nant_in = 64;
      if (launch_correlate_chanmajor(a, sc, cf.corr_path) != 0) return -2;
    }
  }
  if (d.beams || d.chanmask) {
    BfArgs b{};
    b.in = static_cast<const uint8_t *>(d.blk);
    b.wimg = static_cast<const uint8_t *>(c->aux[AUX_WIMG_BF16].ptr);
    b.out_u8 = d.beams;
    b.out_fb = d.chanmask ? fb : nullptr;
    b.err = c->d_err;
    b.npkt = npkt;
    b.nant_in = cf.nant_in;
    b.nchan = nchan;
    b.nbeam = cf.nbeam;
    b.ppo = ppo;
    b.scale = cf.bf_scale;
    b.path = cf.bf_path;
    b.variant = cf.bf_variant;
    b.wait_limit_ns = cf.wait_limit_ns;
    if (launch_beamform(b, c->num_sms, sb) != 0) return -2;
  }
  if (d.chanmask) {
    dsax_flag_params p;
    dsax_default_flag_params(&p, cf.nbeam, nout, ngrp);
    p.tbin = nout >= 64 ? 16 : (nout >= 16 ? nout / 4 : 1);
    p.filt = p.filt > ngrp - 2 * p.guard ? ngrp - 2 * p.guard : p.filt;
    FlagArgs f{};
    f.err = c->d_err;
    f.wait_limit_ns = cf.wait_limit_ns;
    f.x = fb;
    f.nbeam = cf.nbeam; f.ntime = nout; f.nchan = ngrp;
    f.guard = p.guard; f.filt = p.filt; f.tbin = p.tbin; f.fbin = p.fbin;
    f.ts_base = p.ts_base; f.tsflag = d.tsmask ? 1 : 0; f.parity = 0;
    f.thresh = p.thresh; f.var_add = p.var_add; f.ts_thresh = p.ts_thresh;
    const size_t nbc = (size_t)cf.nbeam * ngrp;
    f.spec = fstats; f.var = fstats + nbc; f.maxs = fstats + 2 * nbc; f.pp = fstats + 3 * nbc;
    f.ts = fstats + 4 * nbc;
    f.counts = reinterpret_cast<int *>(fstats + 4 * nbc + (size_t)cf.nbeam * nout);
    f.chanmask = d.chanmask;
    f.tsmask = d.tsmask ? d.tsmask : reinterpret_cast<uint8_t *>(f.counts + 2);
    f.ctr = reinterpret_cast<int *>(fstats + 4 * nbc + 2 * (size_t)cf.nbeam * nout + 64);
    // the flag counters accumulate with atomics: clear them per block (inside
    // the graph too, so every replay starts from zero)
    if (cudaMemsetAsync(f.counts, 0, 2 * sizeof(int), sb) != cudaSuccess) return -2;
    if (launch_flag(f, sb) != 0) return -2;
  }
  return 0;
}

}  // namespace

extern "C" {

int dsax_run_batch(dsax_ctx *c, const dsax_block_desc *blocks, int nblk, int use_graph) {
  if (!c || !blocks || nblk < 1) return DSAX_ERR_ARG;
  const dsax_config &cf = c->cfg;
  int maxch = 0;
  bool need_bf = false;
  for (int i = 0; i < nblk; ++i) {
    const dsax_block_desc &d = blocks[i];
    if (!d.blk || d.nchan < 8 || d.nchan % 8 || d.nchan / 8 > 128 ||
        !aligned16(d.blk) || (d.vis && !aligned16(d.vis)))
      return set_error(c, DSAX_ERR_ARG, "block %d: bad pointer or nchan (multiple of 8, <= 1024)", i);
    if (d.nchan > maxch) maxch = d.nchan;
    need_bf |= d.beams != nullptr || d.chanmask != nullptr;
  }
  if (need_bf && !c->weights_ready)
    return set_error(c, DSAX_ERR_ARG, "dsax_set_weights not called");
  if (need_bf && c->weights_nchan < maxch)
    return set_error(c, DSAX_ERR_ARG, "weights cover %d channels, batch needs %d", c->weights_nchan,
                     maxch);
  DeviceGuard g(c->device);
  const int nout = cf.npkt / cf.bf_pkt_per_out;
  const size_t nscr = (size_t)maxch * cf.npkt * 256;
  const size_t nfb = (size_t)cf.nbeam * nout * (maxch / 8);
  const size_t nfs = 4 * (size_t)cf.nbeam * (maxch / 8) + (size_t)cf.nbeam * nout + 64 +
                     (size_t)cf.nbeam * nout + flag_ctr_ints(cf.nbeam);
  int rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_BATCH_SCRATCH], nscr + 4 * (nfb + nfs), "batch scratch")) !=
      DSAX_OK)
    return rc;
  uint8_t *scratch = static_cast<uint8_t *>(c->aux[AUX_BATCH_SCRATCH].ptr);
  float *fb = reinterpret_cast<float *>(scratch + nscr);
  float *fs = fb + nfb;

  BatchPlan *plan = static_cast<BatchPlan *>(c->batch_plan);
  bool same = plan && (int)plan->blocks.size() == nblk &&
              memcmp(plan->blocks.data(), blocks, sizeof(dsax_block_desc) * nblk) == 0;
  if (use_graph && same && plan->exec) {
    cudaError_t e = cudaGraphLaunch(plan->exec, c->stream);
    return e == cudaSuccess ? DSAX_OK : cuda_check(c, e, "graph launch");
  }
  if (!c->bstream) {
    cudaError_t e0 = cudaStreamCreateWithFlags(&c->bstream, cudaStreamNonBlocking);
    for (auto &ev : c->bev)
      if (e0 == cudaSuccess && !ev) e0 = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e0 != cudaSuccess) return cuda_check(c, e0, "batch stream");
  }
  // fork the beamform chain off the context stream, run both chains, join
  auto enqueue_all = [&]() -> int {
    if (cudaEventRecord(c->bev[0], c->stream) != cudaSuccess ||
        cudaStreamWaitEvent(c->bstream, c->bev[0], 0) != cudaSuccess)
      return -2;
    for (int i = 0; i < nblk; ++i)
      if (enqueue_block(c, blocks[i], scratch, fb, fs, c->stream, c->bstream) != 0) return -2;
    if (cudaEventRecord(c->bev[1], c->bstream) != cudaSuccess ||
        cudaStreamWaitEvent(c->stream, c->bev[1], 0) != cudaSuccess)
      return -2;
    return 0;
  };
  if (!use_graph) {
    if (enqueue_all() != 0) return cuda_check(c, cudaGetLastError(), "batch launch");
    return DSAX_OK;
  }
  // (re)capture
  if (plan) {
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    delete plan;
  }
  plan = new BatchPlan();
  c->batch_plan = plan;
  plan->blocks.assign(blocks, blocks + nblk);
  cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_check(c, e, "begin capture");
  const int lrc = enqueue_all();
  e = cudaStreamEndCapture(c->stream, &plan->graph);
  if (lrc || e != cudaSuccess) return cuda_check(c, e != cudaSuccess ? e : cudaErrorUnknown, "capture");
  e = cudaGraphInstantiate(&plan->exec, plan->graph, 0);
  if (e != cudaSuccess) return cuda_check(c, e, "graph instantiate");
  e = cudaGraphLaunch(plan->exec, c->stream);
  return e == cudaSuccess ? DSAX_OK : cuda_check(c, e, "graph launch");
}

}  // extern "C"

namespace dsax {
void release_batch_plan(dsax_ctx *c) {
  BatchPlan *plan = static_cast<BatchPlan *>(c->batch_plan);
  if (!plan) return;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  delete plan;
  c->batch_plan = nullptr;
}
}  // namespace dsax

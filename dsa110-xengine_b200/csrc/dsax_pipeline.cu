// dsax_pipeline.cu -- many captured blocks through the correlator with the
// stages of consecutive blocks overlapped on separate streams.
//
// The reference processes one psrdada block at a time: dsaX_xgpu waits for
// each block's H2D copy, promote, xgpuCudaXengine and matrix copy-out
// before it reads the next (src/dsaX_xgpu.cu:300-357).  Here block i+1's
// corner turn (HBM-bound) runs on a side stream while block i is correlated
// (bound by the unpack warps, with HBM bandwidth to spare), and in host mode
// the PCIe copies in and out overlap both.  The fused paths (corr_path 6,
// 7) have no corner turn: only the copies overlap the correlations.  Buffers are double-buffered and
// every reuse waits on the event of the stage that last read the buffer.
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace {

enum { S_H2D = 0, S_REO = 1, S_D2H = 2 };
enum { E_START = 0, E_H2D = 1, E_REO = 3, E_CORR = 5, E_D2H = 7 };   // [2] each from 1

int ensure_pipeline(dsax_ctx *c) {
  for (auto &st : c->side)
    if (!st && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      return cuda_check(c, cudaGetLastError(), "pipeline stream");
  for (auto &ev : c->pev)
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
      return cuda_check(c, cudaGetLastError(), "pipeline event");
  return DSAX_OK;
}

}  // namespace

extern "C" int dsax_correlate_many(dsax_ctx *c, const void *const *blocks, void *const *vis,
                                   int nblk, int mem) {
  if (!c || !blocks || !vis || nblk < 1) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  for (int i = 0; i < nblk; ++i)
    if (!blocks[i] || !vis[i] || (mem == DSAX_MEM_DEVICE && (!aligned16(blocks[i]) || !aligned16(vis[i]))))
      return set_error(c, DSAX_ERR_ARG, "block %d: null or misaligned pointer", i);
  DeviceGuard g(c->device);
  int rc = ensure_pipeline(c);
  if (rc != DSAX_OK) return rc;
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nreo = dsax_block_bytes(&c->cfg, DSAX_FMT_CHANMAJOR);
  const size_t nvis = dsax_vis_bytes(&c->cfg);
  auto up = [](size_t n) { return (n + 255) & ~(size_t)255; };
  const bool host = mem == DSAX_MEM_HOST;
  // corr_path 6 / 7: the correlator reads the captured block itself (no
  // corner turn, no channel-major buffer); device blocks were checked for
  // 16-byte alignment above and the host-mode staging buffers are aligned
  CorrArgs probe{};
  probe.npkt = c->cfg.npkt;
  probe.nant_in = c->cfg.nant_in;
  probe.nchan = c->cfg.nchan;
  probe.in = host ? nullptr : static_cast<const uint8_t *>(blocks[0]);
  const bool fused = corr_path_fused(c->cfg.corr_path) && captured_cluster_ok(probe);
  const bool need_reo = !fused;
  const size_t need = (need_reo ? 2 * up(nreo) : 0) + (host ? 2 * up(nin) + 2 * up(nvis) : 0);
  if ((rc = ensure_buffer(c, c->aux[AUX_PIPE], need, "correlate_many buffers")) != DSAX_OK) return rc;
  uint8_t *base = static_cast<uint8_t *>(c->aux[AUX_PIPE].ptr);
  const size_t oreo = need_reo ? 2 * up(nreo) : 0;
  uint8_t *reo[2] = {base, base + up(nreo)};   // unused by the fused paths
  uint8_t *din[2] = {base + oreo, base + oreo + up(nin)};
  uint8_t *dvis[2] = {din[1] + up(nin), din[1] + up(nin) + up(nvis)};

  // The corner turns run on their own stream in both modes.  In device mode
  // block i+1's corner turn takes the SMs that the persistent correlator's
  // CTAs free as they finish their last channel (60 of 148 SMs idle for
  // the last third of a 384-channel block): 0.146 against 0.162 ms per
  // block with both on one stream.  (With one correlator CTA per channel
  // the overlap measured slower, 0.29 against 0.165 ms: the corner turn's
  // CTAs took the SMs the correlator's later waves needed.)  With host
  // buffers the PCIe copies set the pace.
  cudaStream_t cs = c->stream, h2d = c->side[S_H2D], d2h = c->side[S_D2H];
  cudaStream_t rs = c->side[S_REO];
  cudaEvent_t *ev = c->pev;
  // the side streams start after everything already queued on the context stream
  cudaError_t e = cudaEventRecord(ev[E_START], cs);
  for (cudaStream_t st : {h2d, rs, d2h})
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev[E_START], 0);
  if (e != cudaSuccess) return cuda_check(c, e, "pipeline start");

  CorrArgs a{};
  a.npkt = c->cfg.npkt;
  a.nant_in = 64;
  a.nchan = c->cfg.nchan;
  a.err = c->d_err;
  a.wait_limit_ns = c->cfg.wait_limit_ns;
  a.accumulate = 0;
  for (int i = 0; i < nblk && e == cudaSuccess; ++i) {
    const int b = i & 1;
    const uint8_t *src = static_cast<const uint8_t *>(blocks[i]);
    if (host) {
      // copy in: the stage that read din[b] for block i-2 has finished
      if (i >= 2) e = cudaStreamWaitEvent(h2d, ev[(fused ? E_CORR : E_REO) + b], 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(din[b], src, nin, cudaMemcpyHostToDevice, h2d);
      if (e == cudaSuccess) e = cudaEventRecord(ev[E_H2D + b], h2d);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(fused ? cs : rs, ev[E_H2D + b], 0);
      src = din[b];
    }
    if (!fused) {
      // corner turn: the correlation of block i-2 has finished reading reo[b]
      if (e == cudaSuccess && i >= 2) e = cudaStreamWaitEvent(rs, ev[E_CORR + b], 0);
      if (e != cudaSuccess) break;
      if (launch_reorder_chanmajor(src, reo[b], c->cfg.npkt, c->cfg.nant_in, c->cfg.nchan, rs) != 0) {
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaErrorInvalidValue;
        break;
      }
      e = cudaEventRecord(ev[E_REO + b], rs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ev[E_REO + b], 0);
    }
    // correlate: in host mode the copy-out of block i-2 has finished reading dvis[b]
    if (e == cudaSuccess && host && i >= 2) e = cudaStreamWaitEvent(cs, ev[E_D2H + b], 0);
    if (e != cudaSuccess) break;
    a.vis = host ? reinterpret_cast<float *>(dvis[b]) : static_cast<float *>(vis[i]);
    int lrc;
    if (fused) {
      a.in = src;
      a.nant_in = c->cfg.nant_in;
      lrc = launch_correlate_captured_cluster(a, cs, corr_path_unpack_warps(c->cfg.corr_path));
    } else {
      a.in = reo[b];
      a.nant_in = 64;
      lrc = launch_correlate_chanmajor(a, cs, c->cfg.corr_path);
    }
    if (lrc != 0) {
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaErrorInvalidValue;
      break;
    }
    e = cudaEventRecord(ev[E_CORR + b], cs);
    if (host && e == cudaSuccess) {
      e = cudaStreamWaitEvent(d2h, ev[E_CORR + b], 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(vis[i], dvis[b], nvis, cudaMemcpyDeviceToHost, d2h);
      if (e == cudaSuccess) e = cudaEventRecord(ev[E_D2H + b], d2h);
    }
  }
  // everything the side streams did is ordered before later context-stream work
  for (cudaStream_t st : {h2d, rs, d2h}) {
    cudaError_t e2 = cudaEventRecord(ev[E_START], st);
    if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(cs, ev[E_START], 0);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) return cuda_check(c, e, "correlate_many");
  return host ? dsax_sync(c) : DSAX_OK;
}

// dsax_flag_host.cu -- plain-flagger entry points of the C-ABI.
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

extern "C" {

void dsax_default_flag_params(dsax_flag_params *p, int nbeam, int ntime, int nchan) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->nbeam = nbeam;
  p->ntime = ntime;
  p->nchan = nchan;
  p->guard = (nchan * 128 + 512) / 1024;   // ZeroChannels 128 of 1024, scaled
  p->filt = 21;
  p->tbin = 128;
  p->fbin = 8;
  p->ts_base = ntime / 16;
  p->tsflag = 1;
  p->parity = 0;
  p->thresh = 5.0f;
  p->var_add = 0.5f;
  p->ts_thresh = 10.0f;
  p->nperm = 0;
}

int dsax_flag(dsax_ctx *c, const dsax_flag_params *p, const float *x, const float *oldspec,
              uint8_t *chanmask, uint8_t *tsmask, float *stats, int *counts, int mem) {
  if (!c || !p || !x || !chanmask || !tsmask) return DSAX_ERR_ARG;
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  if (B < 1 || T < 1 || C < 1 || C > 128 || p->guard < 0 || C - 2 * p->guard < 1 ||
      p->filt < 1 || p->filt > C - 2 * p->guard || p->tbin < 1 || p->fbin < 1 ||
      p->ts_base < 1 || p->ts_base > T || p->ts_base > 4096 || p->nperm < 0 || p->nperm > 8)
    return set_error(c, DSAX_ERR_ARG, "flag parameters out of range (nchan <= 128, ts_base <= 4096)");
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  const size_t nbc = (size_t)B * C, nbt = (size_t)B * T;
  const size_t nstat = 4 * nbc + nbt;
  int rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_FLAG_STATS], nstat * 4 + 64, "flag statistics")) != DSAX_OK)
    return rc;
  FlagArgs a{};
  a.nbeam = B; a.ntime = T; a.nchan = C;
  a.guard = p->guard; a.filt = p->filt; a.tbin = p->tbin; a.fbin = p->fbin;
  a.ts_base = p->ts_base; a.tsflag = p->tsflag; a.parity = p->parity;
  a.thresh = p->thresh; a.var_add = p->var_add; a.ts_thresh = p->ts_thresh;
  a.nperm = p->nperm;
  for (int i = 0; i < p->nperm; ++i) a.perm[i] = p->perm[i];
  float *sbuf = (mem == DSAX_MEM_DEVICE && stats) ? stats
                                                  : static_cast<float *>(c->aux[AUX_FLAG_STATS].ptr);
  a.spec = sbuf; a.var = sbuf + nbc; a.maxs = sbuf + 2 * nbc; a.pp = sbuf + 3 * nbc;
  a.ts = sbuf + 4 * nbc;
  int *dcounts = reinterpret_cast<int *>(static_cast<uint8_t *>(c->aux[AUX_FLAG_STATS].ptr) +
                                         nstat * 4);
  a.counts = (mem == DSAX_MEM_DEVICE && counts) ? counts : dcounts;
  cudaError_t e = cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "clear counts");
  if (mem == DSAX_MEM_DEVICE) {
    a.x = x; a.oldspec = oldspec; a.chanmask = chanmask; a.tsmask = tsmask;
    if (launch_flag(a, c->stream) != 0) return cuda_check(c, cudaGetLastError(), "flagger launch");
    return DSAX_OK;
  }
  const size_t nx = (size_t)B * T * C * 4;
  if ((rc = ensure_buffer(c, c->aux[AUX_FLAG_X], nx + nbc * 4, "filterbank")) != DSAX_OK) return rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_FLAG_MASK], nbc + nbt, "masks")) != DSAX_OK) return rc;
  float *dx = static_cast<float *>(c->aux[AUX_FLAG_X].ptr);
  float *dold = dx + (size_t)B * T * C;
  uint8_t *dm = static_cast<uint8_t *>(c->aux[AUX_FLAG_MASK].ptr);
  if ((e = cudaMemcpyAsync(dx, x, nx, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "H2D filterbank");
  if (oldspec &&
      (e = cudaMemcpyAsync(dold, oldspec, nbc * 4, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "H2D oldspec");
  a.x = dx; a.oldspec = oldspec ? dold : nullptr; a.chanmask = dm; a.tsmask = dm + nbc;
  if (launch_flag(a, c->stream) != 0) return cuda_check(c, cudaGetLastError(), "flagger launch");
  if ((e = cudaMemcpyAsync(chanmask, dm, nbc, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(tsmask, dm + nbc, nbt, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H masks");
  if (stats && (e = cudaMemcpyAsync(stats, sbuf, nstat * 4, cudaMemcpyDeviceToHost, c->stream)) !=
                   cudaSuccess)
    return cuda_check(c, e, "D2H statistics");
  if (counts && (e = cudaMemcpyAsync(counts, dcounts, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                     c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H counts");
  return dsax_sync(c);
}

}  // extern "C"

// dsax_flag_host.cu -- plain-flagger entry points of the C-ABI: the
// stateless mask call (dsax_flag) and the per-block data path with its
// state (dsax_flag_state / dsax_flag_clean), src/gpu_flagger.cu:1260-1487.
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace {

int check_params(const dsax_flag_params *p) {
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  if (B < 1 || T < 1 || C < 4 || C > 1024 || p->guard < 0 || C - 2 * p->guard < 1 ||
      p->filt < 1 || p->filt > C - 2 * p->guard || p->tbin < 1 || p->fbin < 1 ||
      p->ts_base < 1 || p->ts_base > T || p->ts_base > 4096 || p->nperm < 0 || p->nperm > 8)
    return DSAX_ERR_ARG;
  return DSAX_OK;
}

void fill_args(FlagArgs &a, const dsax_flag_params *p) {
  a.nbeam = p->nbeam; a.ntime = p->ntime; a.nchan = p->nchan;
  a.guard = p->guard; a.filt = p->filt; a.tbin = p->tbin; a.fbin = p->fbin;
  a.ts_base = p->ts_base; a.tsflag = p->tsflag; a.parity = p->parity;
  a.thresh = p->thresh; a.var_add = p->var_add; a.ts_thresh = p->ts_thresh;
  a.nperm = p->nperm;
  for (int i = 0; i < p->nperm; ++i) a.perm[i] = p->perm[i];
}

int nslabs(int nchan) { return (nchan + kFlagSlab - 1) / kFlagSlab; }

uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace

// The flagger state behind dsax_flag_state: the baseline, its history, the
// previous spectrum and total power, per-beam levels and the noise block,
// all in one device allocation.
struct dsax_flag_state {
  dsax_flag_params p{};
  dsax_flag_clean_params cp{};
  int dtype = DSAX_DTYPE_F32;
  int device = 0;
  int nseen = 0, started = 0, blocks = 0, last_flagged = 0;
  DevBuf buf, stage;
  float *spec0 = nullptr, *var0 = nullptr, *hist_spec = nullptr, *hist_var = nullptr;
  float *oldspec = nullptr, *stats = nullptr, *rowsum = nullptr, *bpwr = nullptr;
  double *tpwr = nullptr;   // [0] previous flagged block's total power, [1] this
                            // block's, [2] the value [0] held when this block ran
  int *status = nullptr;    // [0] replaced (4 ints)
  int *counts = nullptr;    // [2], directly after status
  void *noise = nullptr;
  uint8_t *dmask = nullptr; // masks when the caller passes none (device mode)
  int *ctr = nullptr;       // completion counters of the flagger launches
};

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

void dsax_default_flag_clean_params(dsax_flag_clean_params *cp) {
  if (!cp) return;
  memset(cp, 0, sizeof(*cp));
  cp->mn = 48.0f;
  cp->sig = 6.0f;
  cp->mod_thresh = 0.0005f;
  cp->naver = 5;
  cp->scale = 1;
  cp->pwr = 0;
  cp->modcheck = 1;
  cp->seed = 1;
}

int dsax_flag(dsax_ctx *c, const dsax_flag_params *p, const float *x, const float *oldspec,
              uint8_t *chanmask, uint8_t *tsmask, float *stats, int *counts, int mem) {
  if (!c || !p || !x || !chanmask || !tsmask) return DSAX_ERR_ARG;
  if (check_params(p) != DSAX_OK || p->nchan % 4)
    return set_error(c, DSAX_ERR_ARG,
                     "flag parameters out of range (4 <= nchan <= 1024, multiple of 4; "
                     "ts_base <= 4096)");
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  const size_t nbc = (size_t)B * C, nbt = (size_t)B * T;
  const size_t nstat = 4 * nbc + nbt;
  const size_t nrow = nslabs(C) > 1 ? (size_t)B * nslabs(C) * T : 0;
  int rc;
  const size_t nctr = flag_ctr_ints(B);
  if ((rc = ensure_buffer(c, c->aux[AUX_FLAG_STATS], (nstat + nrow + 2 + nctr) * 4 + 64,
                          "flag statistics")) != DSAX_OK)
    return rc;
  FlagArgs a{};
  fill_args(a, p);
  a.err = c->d_err;
  a.wait_limit_ns = c->cfg.wait_limit_ns;
  float *sbuf = (mem == DSAX_MEM_DEVICE && stats) ? stats
                                                  : static_cast<float *>(c->aux[AUX_FLAG_STATS].ptr);
  a.spec = sbuf; a.var = sbuf + nbc; a.maxs = sbuf + 2 * nbc; a.pp = sbuf + 3 * nbc;
  a.ts = sbuf + 4 * nbc;
  float *scratch = static_cast<float *>(c->aux[AUX_FLAG_STATS].ptr);
  a.rowsum = nrow ? scratch + nstat : nullptr;
  int *dcounts = reinterpret_cast<int *>(scratch + nstat + nrow);
  a.ctr = dcounts + 2;
  a.counts = (mem == DSAX_MEM_DEVICE && counts) ? counts : dcounts;
  cudaError_t e = cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "clear counts");
  if (mem == DSAX_MEM_DEVICE) {
    a.x = x; a.oldspec = oldspec; a.chanmask = chanmask; a.tsmask = tsmask;
    if (!aligned16(x)) return set_error(c, DSAX_ERR_ARG, "filterbank must be 16-byte aligned");
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

int dsax_flag_state_create(dsax_ctx *c, const dsax_flag_params *p,
                           const dsax_flag_clean_params *cp, int dtype, dsax_flag_state **out) {
  if (!c || !p || !cp || !out) return DSAX_ERR_ARG;
  *out = nullptr;
  if (check_params(p) != DSAX_OK || (dtype != DSAX_DTYPE_F32 && dtype != DSAX_DTYPE_U8))
    return set_error(c, DSAX_ERR_ARG, "flag parameters out of range");
  if (p->nchan % (dtype == DSAX_DTYPE_U8 ? 16 : 4))
    return set_error(c, DSAX_ERR_ARG, "nchan must be a multiple of 16 (uint8) or 4 (FP32)");
  if (cp->naver < 1 || cp->naver > 64 || !(cp->mn >= 0.0f) || !(cp->sig > 0.0f))
    return set_error(c, DSAX_ERR_ARG, "clean parameters out of range (1 <= naver <= 64)");
  DeviceGuard dg(c->device);
  auto *st = new dsax_flag_state();
  st->p = *p;
  st->cp = *cp;
  st->dtype = dtype;
  st->device = c->device;
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  const size_t bc = (size_t)B * C, bt = (size_t)B * T;
  const size_t es = dtype == DSAX_DTYPE_U8 ? 1 : 4;
  const size_t nrow = nslabs(C) > 1 ? (size_t)B * nslabs(C) * T : 0;
  // float section, then doubles / ints, then the noise block and masks
  const size_t nf = 2 * bc + 2 * (size_t)cp->naver * bc + bc + (4 * bc + bt) + nrow + B;
  const size_t off_d = ((nf * 4 + 255) / 256) * 256;
  const size_t off_noise = off_d + 256;
  const size_t off_mask = ((off_noise + (size_t)T * C * es + 255) / 256) * 256;
  const size_t off_ctr = ((off_mask + bc + bt + 255) / 256) * 256;
  const size_t total = off_ctr + sizeof(int) * flag_ctr_ints(B);
  cudaError_t e = cudaMalloc(&st->buf.ptr, total);
  if (e != cudaSuccess) {
    delete st;
    return set_error(c, DSAX_ERR_NOMEM, "flag state: %zu bytes", total);
  }
  st->buf.bytes = total;
  float *f = static_cast<float *>(st->buf.ptr);
  st->spec0 = f; f += bc;
  st->var0 = f; f += bc;
  st->hist_spec = f; f += (size_t)cp->naver * bc;
  st->hist_var = f; f += (size_t)cp->naver * bc;
  st->oldspec = f; f += bc;
  st->stats = f; f += 4 * bc + bt;
  st->rowsum = nrow ? f : nullptr; f += nrow;
  st->bpwr = f; f += B;
  uint8_t *base = static_cast<uint8_t *>(st->buf.ptr);
  st->tpwr = reinterpret_cast<double *>(base + off_d);
  st->status = reinterpret_cast<int *>(base + off_d + 32);
  st->counts = reinterpret_cast<int *>(base + off_d + 48);
  st->noise = base + off_noise;
  st->dmask = base + off_mask;
  st->ctr = reinterpret_cast<int *>(base + off_ctr);
  // zero everything (oldspec starts at 0, as h_oldspec does at :1214), then
  // the levels at 1 (:1234) and the noise block
  if ((e = cudaMemsetAsync(st->buf.ptr, 0, total, c->stream)) != cudaSuccess) {
    st->buf.release();
    delete st;
    return cuda_check(c, e, "flag state clear");
  }
  std::vector<float> ones(B, 1.0f);
  std::vector<uint8_t> nz((size_t)T * C * es);
  const double two_pi = 6.283185307179586;
  for (size_t i = 0; i < (size_t)T * C; ++i) {
    const uint64_t r1 = splitmix(cp->seed * 0x100000001B3ull + 2 * i);
    const uint64_t r2 = splitmix(cp->seed * 0x100000001B3ull + 2 * i + 1);
    const double u1 = (double)((r1 % 16384) + 1) / 16384.0;
    const double u2 = (double)(r2 % 16384) / 16384.0;
    const double va = std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
    const float v = (float)(va * cp->sig + cp->mn);
    if (es == 1) {
      const double w = std::nearbyint(2.0 * (double)v);
      const unsigned u = w <= 0.0 ? 0u : (w >= 4294967295.0 ? 4294967295u : (unsigned)w);
      nz[i] = (uint8_t)((u / 2u) & 255u);
    } else {
      memcpy(&nz[i * 4], &v, 4);
    }
  }
  if ((e = cudaMemcpy(st->bpwr, ones.data(), B * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(st->noise, nz.data(), nz.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
    st->buf.release();
    delete st;
    return cuda_check(c, e, "flag state upload");
  }
  *out = st;
  return DSAX_OK;
}

void dsax_flag_state_destroy(dsax_flag_state *st) {
  if (!st) return;
  DeviceGuard dg(st->device);
  st->buf.release();
  st->stage.release();
  delete st;
}

int dsax_flag_clean(dsax_ctx *c, dsax_flag_state *st, void *data, uint8_t *chanmask,
                    uint8_t *tsmask, int mem) {
  if (!c || !st || !data) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  if (st->device != c->device) return set_error(c, DSAX_ERR_ARG, "state belongs to another device");
  DeviceGuard dg(c->device);
  const dsax_flag_params *p = &st->p;
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  const size_t bc = (size_t)B * C, bt = (size_t)B * T;
  const size_t es = st->dtype == DSAX_DTYPE_U8 ? 1 : 4;
  const size_t nx = (size_t)B * T * C * es;
  cudaError_t e;
  void *dx = data;
  uint8_t *dcm = chanmask, *dtm = tsmask;
  if (mem == DSAX_MEM_HOST) {
    int rc = ensure_buffer(c, st->stage, nx, "flag staging");
    if (rc != DSAX_OK) return rc;
    dx = st->stage.ptr;
    if ((e = cudaMemcpyAsync(dx, data, nx, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
      return cuda_check(c, e, "H2D filterbank");
    dcm = st->dmask;
    dtm = st->dmask + bc;
  } else {
    if (!dcm) dcm = st->dmask;
    if (!dtm) dtm = st->dmask + bc;
  }
  if (!aligned16(dx)) return set_error(c, DSAX_ERR_ARG, "filterbank must be 16-byte aligned");
  FlagArgs a{};
  fill_args(a, p);
  a.err = c->d_err;
  a.wait_limit_ns = c->cfg.wait_limit_ns;
  if (es == 1) {
    a.xu8 = static_cast<const uint8_t *>(dx);
    a.xw8 = static_cast<uint8_t *>(dx);
  } else {
    a.x = static_cast<const float *>(dx);
    a.xw = static_cast<float *>(dx);
  }
  a.spec = st->stats; a.var = st->stats + bc; a.maxs = st->stats + 2 * bc; a.pp = st->stats + 3 * bc;
  a.ts = st->stats + 4 * bc;
  a.rowsum = st->rowsum;
  a.chanmask = dcm;
  a.tsmask = dtm;
  a.counts = st->counts;
  a.status = st->status;
  a.ctr = st->ctr;
  a.mn = st->cp.mn;
  a.sig = st->cp.sig;
  a.bpwr = st->bpwr;
  a.noise = st->noise;
  if ((e = cudaMemsetAsync(st->status, 0, 16 + 8, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "clear status");
  if (!st->started) {
    // measured only: statistics for the baseline history, no flagging
    a.ts_mean = 1;
    if (launch_flag_stats(a, c->stream) != 0) return cuda_check(c, cudaGetLastError(), "flag stats");
    if ((e = cudaMemsetAsync(dcm, 0, bc, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(dtm, 0, bt, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(st->hist_spec + (size_t)st->nseen * bc, a.spec, bc * 4,
                             cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(st->hist_var + (size_t)st->nseen * bc, a.var, bc * 4,
                             cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess)
      return cuda_check(c, e, "flag history");
    ++st->nseen;
    if (st->nseen >= st->cp.naver) {
      if (launch_flag_baseline(st->hist_spec, st->hist_var, st->cp.naver, B, C, st->spec0,
                               st->var0, c->stream) != 0)
        return cuda_check(c, cudaGetLastError(), "flag baseline");
      st->started = 1;
    }
    st->last_flagged = 0;
  } else {
    a.spec0 = st->cp.scale ? st->spec0 : nullptr;
    a.var0 = st->cp.scale ? st->var0 : nullptr;
    a.oldspec = st->oldspec;
    a.clean = 1;
    a.pwr = st->cp.pwr;
    a.modcheck = st->cp.modcheck;
    a.mod_thresh = st->cp.mod_thresh;
    a.prev_tpwr = st->tpwr;
    a.tpwr_out = st->tpwr + 1;
    if ((e = cudaMemcpyAsync(st->tpwr + 2, st->tpwr, 8, cudaMemcpyDeviceToDevice, c->stream)) !=
        cudaSuccess)
      return cuda_check(c, e, "total power");
    if (launch_flag(a, c->stream) != 0) return cuda_check(c, cudaGetLastError(), "flagger launch");
    // after a flagged block its total power is the next comparison (:1401)
    if ((e = cudaMemcpyAsync(st->tpwr, st->tpwr + 1, 8, cudaMemcpyDeviceToDevice, c->stream)) !=
        cudaSuccess)
      return cuda_check(c, e, "total power");
    st->last_flagged = 1;
  }
  // the next block's references: this block's spectrum (every block,
  // :1484-1486) and, after a flagged block, its total power (:1401)
  if ((e = cudaMemcpyAsync(st->oldspec, a.spec, bc * 4, cudaMemcpyDeviceToDevice, c->stream)) !=
      cudaSuccess)
    return cuda_check(c, e, "oldspec");
  ++st->blocks;
  if (mem == DSAX_MEM_HOST) {
    if ((e = cudaMemcpyAsync(data, dx, nx, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
      return cuda_check(c, e, "D2H filterbank");
    if (chanmask &&
        (e = cudaMemcpyAsync(chanmask, dcm, bc, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
      return cuda_check(c, e, "D2H chanmask");
    if (tsmask && (e = cudaMemcpyAsync(tsmask, dtm, bt, cudaMemcpyDeviceToHost, c->stream)) !=
                      cudaSuccess)
      return cuda_check(c, e, "D2H tsmask");
    return dsax_sync(c);
  }
  return DSAX_OK;
}

int dsax_flag_state_info(dsax_ctx *c, dsax_flag_state *st, dsax_flag_block_info *info) {
  if (!c || !st || !info) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  int rc = dsax_sync(c);
  if (rc != DSAX_OK) return rc;
  double tp[3];
  int w[6];
  cudaError_t e;
  if ((e = cudaMemcpy(tp, st->tpwr, sizeof tp, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(w, st->status, sizeof w, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_check(c, e, "flag state info");
  memset(info, 0, sizeof(*info));
  info->blocks = st->blocks;
  info->started = st->started;
  info->flagged = st->last_flagged;
  info->replaced = w[0];
  info->nchan_flagged = w[4];
  info->nts_flagged = w[5];
  info->prev_tpwr = st->last_flagged ? tp[2] : 0.0;
  info->tpwr = st->last_flagged ? tp[1] : 0.0;
  return DSAX_OK;
}

int dsax_flag_state_get_baseline(dsax_ctx *c, dsax_flag_state *st, float *spec0, float *var0) {
  if (!c || !st) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  int rc = dsax_sync(c);
  if (rc != DSAX_OK) return rc;
  const size_t bc = (size_t)st->p.nbeam * st->p.nchan;
  cudaError_t e;
  if (spec0 && (e = cudaMemcpy(spec0, st->spec0, bc * 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_check(c, e, "D2H spec0");
  if (var0 && (e = cudaMemcpy(var0, st->var0, bc * 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_check(c, e, "D2H var0");
  return DSAX_OK;
}

int dsax_flag_state_set_baseline(dsax_ctx *c, dsax_flag_state *st, const float *spec0,
                                 const float *var0) {
  if (!c || !st || !spec0 || !var0) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  const size_t bc = (size_t)st->p.nbeam * st->p.nchan;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(st->spec0, spec0, bc * 4, cudaMemcpyHostToDevice, c->stream)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(st->var0, var0, bc * 4, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "H2D baseline");
  st->started = 1;
  return dsax_sync(c);
}

int dsax_flag_state_noise(dsax_ctx *c, dsax_flag_state *st, void *noise) {
  if (!c || !st || !noise) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  const size_t n = (size_t)st->p.ntime * st->p.nchan * (st->dtype == DSAX_DTYPE_U8 ? 1 : 4);
  cudaError_t e = cudaMemcpy(noise, st->noise, n, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? DSAX_OK : cuda_check(c, e, "D2H noise");
}

}  // extern "C"

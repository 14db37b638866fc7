// dsax_lflag_host.cu -- learned-flagger entry points of the C-ABI: network
// state on the context, one training step (features -> labels -> forward ->
// BCE -> backward -> Adam), inference to a pixel mask.
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"
#include "dsax_lflag.h"

using namespace dsax;

namespace {

uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Standard normal by Box-Muller on two SplitMix64 uniforms in (0, 1).
double normal(uint64_t &s) {
  const double u1 = ((splitmix64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((splitmix64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

int ensure_net(dsax_ctx *c) {
  LfNet &n = *c->lf;
  if (n.params) return DSAX_OK;
  const int np = lf_nparams();
  int rc = ensure_buffer(c, c->aux[AUX_LF_STATE], sizeof(float) * 4 * np, "learned-flagger state");
  if (rc != DSAX_OK) return rc;
  rc = ensure_buffer(c, c->aux[AUX_LF_WLAYOUT], sizeof(float) * 2 * np, "learned-flagger layouts");
  if (rc != DSAX_OK) return rc;
  float *base = static_cast<float *>(c->aux[AUX_LF_STATE].ptr);
  n.params = base;
  n.grads = base + np;
  n.m = base + 2 * np;
  n.v = base + 3 * np;
  float *lay = static_cast<float *>(c->aux[AUX_LF_WLAYOUT].ptr);
  for (int l = 0; l < kLfLayers; ++l) {
    n.w[l] = n.params + lf_w_offset(l);
    n.b[l] = n.params + lf_b_offset(l);
    n.gw[l] = n.grads + lf_w_offset(l);
    n.gb[l] = n.grads + lf_b_offset(l);
    n.wt[l] = lay + lf_w_offset(l);
    n.wf[l] = lay + np + lf_w_offset(l);
  }
  cudaMemsetAsync(base, 0, sizeof(float) * 4 * np, c->stream);
  n.step = 0;
  return DSAX_OK;
}

int check_lf_shape(dsax_ctx *c, const dsax_flag_params *p, int tds) {
  if (!p) return DSAX_ERR_ARG;
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  if (B < 1 || T < 1 || C < 1 || p->guard < 0 || C - 2 * p->guard < 1 || p->filt < 1 ||
      p->filt > C - 2 * p->guard || p->tbin < 1 || p->fbin < 1 || p->ts_base < 1 ||
      p->ts_base > T || p->ts_base > 4096 || p->nperm < 0 || p->nperm > 8)
    return set_error(c, DSAX_ERR_ARG, "flag parameters out of range");
  if (tds < 1 || T % tds || C % 4 || C > 64 || p->tbin % tds || T % p->tbin ||
      p->tbin > 256 || (size_t)p->tbin * C * 4 > 32768 ||
      sizeof(float) * ((size_t)6 * C + p->ts_base + T + 2 * (T / tds)) > 200 * 1024)
    return set_error(c, DSAX_ERR_ARG,
                     "learned flagger needs ntime %% tbin == 0, tbin %% tds == 0, nchan %% 4 == 0, "
                     "nchan <= 64, tbin * nchan <= 8192");
  return DSAX_OK;
}

// Scratch for B beams on an H x W grid (T samples per beam).
struct LfScratch {
  float *F, *a1, *a2, *a3, *z, *d4, *da, *db, *part;
  float *stats, *pix;   // statistics pass: spec, var, max, pp [B][W]; ts [B][T]; pixel sum, max
  uint8_t *L;
  double *loss;
};

int lf_scratch(dsax_ctx *c, int B, int H, int W, int T, LfScratch &s) {
  const size_t px = (size_t)B * H * W;
  const size_t nstat = (size_t)4 * B * W + (size_t)B * T;
  const size_t nf = px * (8 + 32 + 64 + 64 + 1 + 1 + 64 + 64) + lf_part_floats(B, H) + nstat + 2 * px;
  int rc = ensure_buffer(c, c->aux[AUX_LF_SCRATCH], nf * 4 + px + 64 + 64, "learned-flagger scratch");
  if (rc != DSAX_OK) return rc;
  float *f = static_cast<float *>(c->aux[AUX_LF_SCRATCH].ptr);
  s.loss = reinterpret_cast<double *>(f);  f += 16;
  s.F = f;  f += px * 8;
  s.a1 = f; f += px * 32;
  s.a2 = f; f += px * 64;
  s.a3 = f; f += px * 64;
  s.z = f;  f += px;
  s.d4 = f; f += px;
  s.da = f; f += px * 64;
  s.db = f; f += px * 64;
  s.part = f; f += lf_part_floats(B, H);
  s.stats = f; f += nstat;
  s.pix = f; f += 2 * px;
  s.L = reinterpret_cast<uint8_t *>(f);
  return DSAX_OK;
}

// Features of a device filterbank: the statistics pass (the plain flagger's
// staged kernel, also writing the downsampled spectrogram) then the
// per-beam feature kernel.
int lf_make_features(const dsax_flag_params *p, const float *x, int tds, const LfScratch &s,
                     float *F, uint16_t *Fbf, cudaStream_t st) {
  const int B = p->nbeam, T = p->ntime, C = p->nchan, H = T / tds;
  FlagArgs a{};
  a.x = x;
  a.nbeam = B; a.ntime = T; a.nchan = C;
  a.guard = p->guard; a.filt = p->filt; a.tbin = p->tbin; a.fbin = p->fbin;
  a.ts_base = p->ts_base; a.tsflag = p->tsflag; a.parity = p->parity;
  a.thresh = p->thresh; a.var_add = p->var_add; a.ts_thresh = p->ts_thresh;
  const size_t nbc = (size_t)B * C;
  a.spec = s.stats; a.var = s.stats + nbc; a.maxs = s.stats + 2 * nbc; a.pp = s.stats + 3 * nbc;
  a.ts = s.stats + 4 * nbc;
  a.pix_sum = s.pix;
  a.pix_max = s.pix + (size_t)B * H * C;
  a.tds = tds;
  a.ts_mean = 1;
  if (!flag_shape_ok(a)) return -1;
  int rc = launch_flag_stats(a, st);
  if (rc != 0) return rc;
  return launch_lf_stat_features(a, F, Fbf, st);
}

}  // namespace

extern "C" {

int dsax_lf_init(dsax_ctx *c, unsigned long long seed) {
  if (!c) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = ensure_net(c);
  if (rc != DSAX_OK) return rc;
  std::vector<float> h(lf_nparams(), 0.f);
  uint64_t s = seed;
  for (int l = 0; l < kLfLayers; ++l) {
    const double sd = sqrt(2.0 / (9.0 * kLfCin[l]));
    float *w = h.data() + lf_w_offset(l);
    for (int i = 0; i < kLfCout[l] * 9 * kLfCin[l]; ++i) w[i] = (float)(sd * normal(s));
  }
  return dsax_lf_set_params(c, h.data(), lf_nparams());
}

int dsax_lf_nparams(void) { return lf_nparams(); }

int dsax_lf_set_params(dsax_ctx *c, const float *params, int n) {
  if (!c || !params || n != lf_nparams()) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = ensure_net(c);
  if (rc != DSAX_OK) return rc;
  LfNet &net = *c->lf;
  cudaError_t e = cudaMemcpyAsync(net.params, params, sizeof(float) * n, cudaMemcpyHostToDevice,
                                  c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "upload parameters");
  cudaMemsetAsync(net.m, 0, sizeof(float) * 2 * n, c->stream);  // m and v
  net.step = 0;
  net.version += 1;
  return dsax_sync(c);
}

int dsax_lf_get_params(dsax_ctx *c, float *params, int n) {
  if (!c || !params || n != lf_nparams() || !c->lf->params) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaError_t e = cudaMemcpyAsync(params, c->lf->params, sizeof(float) * n, cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "download parameters");
  return dsax_sync(c);
}

int dsax_lf_features(dsax_ctx *c, const float *x, const dsax_flag_params *p, int tds, float *F) {
  if (!c || !x || !F) return DSAX_ERR_ARG;
  int rc = check_lf_shape(c, p, tds);
  if (rc != DSAX_OK) return rc;
  DeviceGuard g(c->device);
  LfScratch s;
  if ((rc = lf_scratch(c, p->nbeam, p->ntime / tds, p->nchan, p->ntime, s)) != DSAX_OK) return rc;
  if (lf_make_features(p, x, tds, s, F, nullptr, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "feature launch");
  return DSAX_OK;
}

int dsax_lf_train_step(dsax_ctx *c, const float *x, const uint8_t *chanmask, const uint8_t *tsmask,
                       const dsax_flag_params *p, int tds, float lr, float pos_weight, int update,
                       float *loss, float *grads) {
  if (!c || !x || !chanmask || !tsmask) return DSAX_ERR_ARG;
  int rc = check_lf_shape(c, p, tds);
  if (rc != DSAX_OK) return rc;
  if (!c->lf->params) return set_error(c, DSAX_ERR_ARG, "dsax_lf_init not called");
  DeviceGuard g(c->device);
  const int B = p->nbeam, H = p->ntime / tds, W = p->nchan;
  LfScratch s;
  if ((rc = lf_scratch(c, B, H, W, p->ntime, s)) != DSAX_OK) return rc;
  LfNet &net = *c->lf;
  float *acts[5] = {s.F, s.a1, s.a2, s.a3, s.z};
  const int nvalid = B * H * (W - 2 * p->guard);
  int e = 0;
  e |= lf_make_features(p, x, tds, s, s.F, nullptr, c->stream);
  e |= lf_labels(chanmask, tsmask, s.L, B, p->ntime, W, tds, p->guard, c->stream);
  e |= lf_prepare_weights(net, c->stream);
  e |= lf_forward(net, acts, B, H, W, c->stream);
  cudaMemsetAsync(s.loss, 0, sizeof(double), c->stream);
  e |= lf_bce(s.z, s.L, s.d4, s.loss, B, H, W, p->guard, pos_weight, 1.0f / (float)nvalid,
              c->stream);
  e |= lf_backward(net, acts, s.d4, s.da, s.db, s.part, B, H, W, c->stream);
  if (update) e |= lf_adam(net, lr, c->stream);
  if (e) return cuda_check(c, cudaGetLastError(), "training step launch");
  if (loss) {
    double h = 0.0;
    cudaError_t ce = cudaMemcpyAsync(&h, s.loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (ce != cudaSuccess) return cuda_check(c, ce, "loss readback");
    if ((rc = dsax_sync(c)) != DSAX_OK) return rc;
    *loss = (float)(h / nvalid);
  }
  if (grads) {
    cudaError_t ce = cudaMemcpyAsync(grads, net.grads, sizeof(float) * lf_nparams(),
                                     cudaMemcpyDeviceToHost, c->stream);
    if (ce != cudaSuccess) return cuda_check(c, ce, "gradient readback");
    return dsax_sync(c);
  }
  return DSAX_OK;
}

int dsax_flag_learned(dsax_ctx *c, const float *x, const dsax_flag_params *p, int tds,
                      uint8_t *mask, float *logits, int mem) {
  if (!c || !x || !mask) return DSAX_ERR_ARG;
  int rc = check_lf_shape(c, p, tds);
  if (rc != DSAX_OK) return rc;
  if (!c->lf->params) return set_error(c, DSAX_ERR_ARG, "dsax_lf_init not called");
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const int B = p->nbeam, H = p->ntime / tds, W = p->nchan;
  LfScratch s;
  if ((rc = lf_scratch(c, B, H, W, p->ntime, s)) != DSAX_OK) return rc;
  LfNet &net = *c->lf;
  const float *xd = x;
  const size_t px = (size_t)B * H * W;
  if (mem == DSAX_MEM_HOST) {
    const size_t nx = (size_t)B * p->ntime * W * 4;
    if ((rc = ensure_buffer(c, c->aux[AUX_FLAG_X], nx, "filterbank")) != DSAX_OK) return rc;
    cudaError_t ce = cudaMemcpyAsync(c->aux[AUX_FLAG_X].ptr, x, nx, cudaMemcpyHostToDevice, c->stream);
    if (ce != cudaSuccess) return cuda_check(c, ce, "H2D filterbank");
    xd = static_cast<const float *>(c->aux[AUX_FLAG_X].ptr);
  }
  // Inference on the tensor cores: BF16 features and activations in the
  // FP32 training buffers' space, FP32 accumulation.
  void *const prev_w = c->aux[AUX_LF_TCW].ptr;
  if ((rc = ensure_buffer(c, c->aux[AUX_LF_TCW], lf_tc_wimg_bytes(), "learned-flagger weight images")) !=
      DSAX_OK)
    return rc;
  if (c->aux[AUX_LF_TCW].ptr != prev_w) c->lf_wimg_version = ~0u;
  // zero-bordered grids: layer-1 output, layer-2 output, features
  const size_t npad = lf_pad_bytes(B, H, W), nfeat = lf_feat_pad_bytes(B, H, W);
  void *const prev_pad = c->aux[AUX_LF_PAD].ptr;
  if ((rc = ensure_buffer(c, c->aux[AUX_LF_PAD], 2 * npad + nfeat,
                          "learned-flagger padded activations")) != DSAX_OK)
    return rc;
  uint8_t *const padb = static_cast<uint8_t *>(c->aux[AUX_LF_PAD].ptr);
  // No kernel writes a border pixel or channels 32-63 of the layer-1 grid, so
  // they stay zero until the geometry (or the allocation) changes; then the
  // layer-1 grid is cleared and the other grids' borders zeroed.
  if (c->aux[AUX_LF_PAD].ptr != prev_pad) c->lf_pad_geom[0] = 0;
  const bool zero_borders = c->lf_pad_geom[0] != B || c->lf_pad_geom[1] != H || c->lf_pad_geom[2] != W;
  if (zero_borders) {
    cudaError_t ce = cudaMemsetAsync(padb, 0, npad, c->stream);
    if (ce != cudaSuccess) return cuda_check(c, ce, "padded grid clear");
  }
  LfTcBuffers tb;
  uint16_t *fbf = reinterpret_cast<uint16_t *>(padb + 2 * npad);
  tb.featp = fbf;
  tb.act1p = reinterpret_cast<uint16_t *>(padb);
  tb.act2p = reinterpret_cast<uint16_t *>(padb + npad);
  tb.z9 = s.a3;
  tb.logit = s.z;
  tb.mask = mem == DSAX_MEM_DEVICE ? mask : s.L;
  tb.wimg = static_cast<const uint8_t *>(c->aux[AUX_LF_TCW].ptr);
  LfPerm perm;
  perm.n = p->nperm;
  for (int k = 0; k < p->nperm; ++k) perm.ch[k] = p->perm[k];
  int e = 0;
  e |= lf_make_features(p, xd, tds, s, nullptr, fbf, c->stream);
  if (c->lf_wimg_version != net.version) {   // weight images of the current parameters
    e |= lf_tc_prepare(net, static_cast<uint8_t *>(c->aux[AUX_LF_TCW].ptr), c->stream);
    if (!e) c->lf_wimg_version = net.version;
  }
  e |= lf_tc_forward(net, tb, B, H, W, p->guard, perm, zero_borders, c->num_sms, c->d_err,
                     c->cfg.wait_limit_ns, c->stream);
  if (e) return cuda_check(c, cudaGetLastError(), "learned flagger launch");
  if (zero_borders) {
    c->lf_pad_geom[0] = B;
    c->lf_pad_geom[1] = H;
    c->lf_pad_geom[2] = W;
  }
  if (mem == DSAX_MEM_DEVICE) {
    if (logits)
      cudaMemcpyAsync(logits, s.z, px * 4, cudaMemcpyDeviceToDevice, c->stream);
    return DSAX_OK;
  }
  cudaError_t ce = cudaMemcpyAsync(mask, s.L, px, cudaMemcpyDeviceToHost, c->stream);
  if (ce == cudaSuccess && logits)
    ce = cudaMemcpyAsync(logits, s.z, px * 4, cudaMemcpyDeviceToHost, c->stream);
  if (ce != cudaSuccess) return cuda_check(c, ce, "D2H learned mask");
  return dsax_sync(c);
}

}  // extern "C"

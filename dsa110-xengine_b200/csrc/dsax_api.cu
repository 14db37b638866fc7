// dsax_api.cu -- the C-ABI layer (include/dsax.h): contexts, argument
// checks, host<->device staging, error reporting.  No torch types, no
// exceptions across the boundary, never exits the process.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace dsax {

int set_error(dsax_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->errmsg, sizeof(c->errmsg), fmt, ap);
    va_end(ap);
  }
  return code;
}

int cuda_check(dsax_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return DSAX_OK;
  return set_error(c, DSAX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Makes the context's device current for the duration of a call.
DeviceGuard::DeviceGuard(int dev) {
  cudaGetDevice(&prev_);
  if (prev_ != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != prev_ && prev_ >= 0) cudaSetDevice(prev_);
}

int ensure_buffer(dsax_ctx *c, DevBuf &b, size_t nbytes, const char *what) {
  if (b.bytes >= nbytes) return DSAX_OK;
  if (b.ptr) cudaFree(b.ptr);
  b.ptr = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.ptr, nbytes);
  if (e != cudaSuccess)
    return set_error(c, DSAX_ERR_NOMEM, "cudaMalloc(%zu) for %s: %s", nbytes, what,
                     cudaGetErrorString(e));
  b.bytes = nbytes;
  return DSAX_OK;
}

// Reads and clears the device error word (synchronous on the ctx stream).
int check_device_error(dsax_ctx *c) {
  cudaError_t e = cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "device error readback");
  const int v = *c->h_err;
  if (v == 0) return DSAX_OK;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  cudaStreamSynchronize(c->stream);
  if (v & (DEV_ERR_WAIT_FULL | DEV_ERR_WAIT_EMPTY | DEV_ERR_WAIT_ACCUM))
    return set_error(c, DSAX_ERR_TIMEOUT, "device wait expired (flags 0x%x)", v);
  return set_error(c, DSAX_ERR_DEVICE, "device-side check failed (flags 0x%x)", v);
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace dsax

extern "C" {

void dsax_default_config(dsax_config *cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->npkt = 2048;
  cfg->nant_in = 63;
  cfg->nchan = 384;
  cfg->nbeam = 256;
  cfg->bf_pkt_per_out = 16;
  cfg->bf_scale = 1.0f;
  cfg->wait_limit_ns = 0;
}

size_t dsax_block_bytes(const dsax_config *c, int fmt) {
  if (!c) return 0;
  switch (fmt) {
    case DSAX_FMT_CAPTURED: return (size_t)c->npkt * c->nant_in * c->nchan * 4;
    case DSAX_FMT_REORDERED: return (size_t)c->npkt * 2 * c->nchan * 64 * 2;
    case DSAX_FMT_XGPU_INT8: return (size_t)c->npkt * 2 * c->nchan * 64 * 4;
    case DSAX_FMT_CHANMAJOR: return (size_t)c->nchan * c->npkt * 64 * 4;
    default: return 0;
  }
}

size_t dsax_vis_bytes(const dsax_config *c) {
  return c ? (size_t)2 * c->nchan * 2080 * 4 * 2 * sizeof(float) : 0;
}

size_t dsax_beam_bytes(const dsax_config *c) {
  if (!c || c->bf_pkt_per_out <= 0) return 0;
  return (size_t)(c->npkt / c->bf_pkt_per_out) * c->nbeam * (c->nchan / 8);
}

const char *dsax_strerror(int s) {
  switch (s) {
    case DSAX_OK: return "ok";
    case DSAX_ERR_ARG: return "invalid argument";
    case DSAX_ERR_CUDA: return "CUDA runtime error";
    case DSAX_ERR_TIMEOUT: return "device-side wait timed out";
    case DSAX_ERR_NOMEM: return "out of memory";
    case DSAX_ERR_UNSUPPORTED: return "unsupported device (needs sm_100)";
    case DSAX_ERR_DEVICE: return "device-side check failed";
    default: return "unknown status";
  }
}

const char *dsax_last_error(const dsax_ctx *c) { return c ? c->errmsg : "null context"; }

int dsax_create(dsax_ctx **out, const dsax_config *cfg, int device) {
  if (!out || !cfg) return DSAX_ERR_ARG;
  *out = nullptr;
  if (cfg->npkt < 1 || cfg->npkt > (1 << 16) || cfg->nant_in < 1 || cfg->nant_in > 64 ||
      cfg->nchan < 1 || cfg->nchan > 8192 || cfg->bf_path < 0 || cfg->bf_path > 2 ||
      cfg->bf_variant < 0 || cfg->bf_variant > 4)
    return DSAX_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return DSAX_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return DSAX_ERR_CUDA;
  if (prop.major != 10 || prop.minor != 0) return DSAX_ERR_UNSUPPORTED;

  dsax_ctx *c = new (std::nothrow) dsax_ctx();
  if (!c) return DSAX_ERR_NOMEM;
  c->cfg = *cfg;
  if (c->cfg.wait_limit_ns == 0) c->cfg.wait_limit_ns = 1000000000ull;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  DeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc((void **)&c->d_err, sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_err, sizeof(int)) != cudaSuccess ||
      cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
    dsax_destroy(c);
    return DSAX_ERR_CUDA;
  }
  *out = c;
  return DSAX_OK;
}

void dsax_destroy(dsax_ctx *c) {
  if (!c) return;
  DeviceGuard g(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release_batch_plan(c);
  c->release_all();
  for (auto &st : c->side)
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (auto &ev : c->pev)
    if (ev) cudaEventDestroy(ev);
  if (c->bstream) {
    cudaStreamSynchronize(c->bstream);
    cudaStreamDestroy(c->bstream);
  }
  for (auto &ev : c->bev)
    if (ev) cudaEventDestroy(ev);
  if (c->d_err) cudaFree(c->d_err);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

void *dsax_stream(dsax_ctx *c) { return c ? (void *)c->stream : nullptr; }

int dsax_sync(dsax_ctx *c) {
  if (!c) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "cudaStreamSynchronize");
  return check_device_error(c);
}

int dsax_register_host(dsax_ctx *c, void *p, size_t n) {
  if (!c || !p || n == 0) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaError_t e = cudaHostRegister(p, n, cudaHostRegisterPortable);
  if (e != cudaSuccess) return cuda_check(c, e, "cudaHostRegister");
  return DSAX_OK;
}

int dsax_unregister_host(dsax_ctx *c, void *p) {
  if (!c || !p) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaError_t e = cudaHostUnregister(p);
  if (e != cudaSuccess) return cuda_check(c, e, "cudaHostUnregister");
  return DSAX_OK;
}

int dsax_host_alloc(dsax_ctx *c, size_t n, void **p) {
  if (!c || !p || n == 0) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  cudaError_t e = cudaHostAlloc(p, n, cudaHostAllocPortable);
  if (e != cudaSuccess) return set_error(c, DSAX_ERR_NOMEM, "cudaHostAlloc: %s", cudaGetErrorString(e));
  return DSAX_OK;
}

int dsax_host_free(dsax_ctx *c, void *p) {
  if (!c) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  return cuda_check(c, cudaFreeHost(p), "cudaFreeHost");
}

// Enqueues the correlation of one device-resident block on the ctx stream.
static int correlate_device(dsax_ctx *c, int fmt, const void *in, float *vis, int accumulate) {
  CorrArgs a{};
  a.npkt = c->cfg.npkt;
  a.nant_in = fmt == DSAX_FMT_CAPTURED ? c->cfg.nant_in : 64;
  a.nchan = c->cfg.nchan;
  a.err = c->d_err;
  a.wait_limit_ns = c->cfg.wait_limit_ns;
  a.accumulate = accumulate ? 1 : 0;
  a.vis = vis;
  a.in = static_cast<const uint8_t *>(in);
  if (fmt == DSAX_FMT_CHANMAJOR) {
    a.nant_in = 64;
    if (launch_correlate_chanmajor(a, c->stream, c->cfg.corr_path) != 0)
      return cuda_check(c, cudaGetLastError(), "correlator launch");
    return DSAX_OK;
  }
  if (fmt == DSAX_FMT_CAPTURED && corr_path_fused(c->cfg.corr_path) && captured_cluster_ok(a)) {
    // the correlator reads the captured block directly (no corner turn)
    if (launch_correlate_captured_cluster(a, c->stream, corr_path_unpack_warps(c->cfg.corr_path)) != 0)
      return cuda_check(c, cudaGetLastError(), "correlator launch");
    return DSAX_OK;
  }
  if (fmt == DSAX_FMT_CAPTURED && c->cfg.corr_path != 1) {
    // corner turn into the context's buffer, then correlate from it
    const size_t nre = dsax_block_bytes(&c->cfg, DSAX_FMT_REORDERED);
    int rc = ensure_buffer(c, c->aux[AUX_REORDERED], nre, "corner-turned block");
    if (rc != DSAX_OK) return rc;
    uint8_t *tmp = static_cast<uint8_t *>(c->aux[AUX_REORDERED].ptr);
    if (c->cfg.corr_path == 2) {   // REORDER-key layout (massage) + row loads
      if (launch_reorder(a.in, tmp, c->cfg.npkt, c->cfg.nant_in, c->cfg.nchan, c->stream) != 0)
        return cuda_check(c, cudaGetLastError(), "corner-turn launch");
      a.in = tmp;
      a.nant_in = 64;
      fmt = DSAX_FMT_REORDERED;
    } else {                       // channel-major streams + correlator (3: direct, else bulk-fed)
      if (launch_reorder_chanmajor(a.in, tmp, c->cfg.npkt, c->cfg.nant_in, c->cfg.nchan,
                                   c->stream) != 0)
        return cuda_check(c, cudaGetLastError(), "corner-turn launch");
      a.in = tmp;
      a.nant_in = 64;
      if (launch_correlate_chanmajor(a, c->stream, c->cfg.corr_path) != 0)
        return cuda_check(c, cudaGetLastError(), "correlator launch");
      return DSAX_OK;
    }
  }
  if (launch_correlate(a, fmt, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "correlator launch");
  return DSAX_OK;
}

int dsax_correlate_fmt(dsax_ctx *c, int fmt, const void *in, void *vis, int mem,
                       int accumulate) {
  if (!c || !in || !vis) return DSAX_ERR_ARG;
  if (fmt < DSAX_FMT_CAPTURED || fmt > DSAX_FMT_CHANMAJOR)
    return set_error(c, DSAX_ERR_ARG, "unknown input format %d", fmt);
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE)
    return set_error(c, DSAX_ERR_ARG, "mem must be DSAX_MEM_HOST or DSAX_MEM_DEVICE");
  DeviceGuard g(c->device);
  const size_t nin = dsax_block_bytes(&c->cfg, fmt);
  const size_t nvis = dsax_vis_bytes(&c->cfg);
  if (mem == DSAX_MEM_DEVICE) {
    if (!aligned16(in) || !aligned16(vis))
      return set_error(c, DSAX_ERR_ARG, "device pointers must be 16-byte aligned");
    return correlate_device(c, fmt, in, static_cast<float *>(vis), accumulate);
  }
  int rc;
  if ((rc = ensure_buffer(c, c->in_buf, nin, "input block")) != DSAX_OK) return rc;
  if ((rc = ensure_buffer(c, c->vis_buf, nvis, "visibilities")) != DSAX_OK) return rc;
  cudaError_t e = cudaMemcpyAsync(c->in_buf.ptr, in, nin, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "H2D block");
  if ((rc = correlate_device(c, fmt, c->in_buf.ptr, static_cast<float *>(c->vis_buf.ptr), 0)) !=
      DSAX_OK)
    return rc;
  e = cudaMemcpyAsync(vis, c->vis_buf.ptr, nvis, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "D2H visibilities");
  return dsax_sync(c);
}

int dsax_corner_turn(dsax_ctx *c, const void *captured, void *out, int out_fmt, int mem) {
  if (!c || !captured || !out) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  if (out_fmt != DSAX_FMT_REORDERED && out_fmt != DSAX_FMT_CHANMAJOR)
    return set_error(c, DSAX_ERR_ARG, "corner turn output must be REORDERED or CHANMAJOR");
  DeviceGuard g(c->device);
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nout = dsax_block_bytes(&c->cfg, out_fmt);
  auto launch = [&](const uint8_t *src, uint8_t *dst) {
    return out_fmt == DSAX_FMT_REORDERED
               ? launch_reorder(src, dst, c->cfg.npkt, c->cfg.nant_in, c->cfg.nchan, c->stream)
               : launch_reorder_chanmajor(src, dst, c->cfg.npkt, c->cfg.nant_in, c->cfg.nchan,
                                          c->stream);
  };
  if (mem == DSAX_MEM_DEVICE) {
    if (!aligned16(captured) || !aligned16(out))
      return set_error(c, DSAX_ERR_ARG, "device pointers must be 16-byte aligned");
    if (launch(static_cast<const uint8_t *>(captured), static_cast<uint8_t *>(out)) != 0)
      return cuda_check(c, cudaGetLastError(), "corner-turn launch");
    return DSAX_OK;
  }
  int rc;
  if ((rc = ensure_buffer(c, c->in_buf, nin, "input block")) != DSAX_OK) return rc;
  if ((rc = ensure_buffer(c, c->aux[AUX_REORDER_OUT], nout, "corner-turned block")) != DSAX_OK)
    return rc;
  cudaError_t e = cudaMemcpyAsync(c->in_buf.ptr, captured, nin, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "H2D block");
  if (launch(static_cast<const uint8_t *>(c->in_buf.ptr),
             static_cast<uint8_t *>(c->aux[AUX_REORDER_OUT].ptr)) != 0)
    return cuda_check(c, cudaGetLastError(), "corner-turn launch");
  e = cudaMemcpyAsync(out, c->aux[AUX_REORDER_OUT].ptr, nout, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "D2H corner-turned block");
  return dsax_sync(c);
}

int dsax_reorder(dsax_ctx *c, const void *captured, void *reordered, int mem) {
  return dsax_corner_turn(c, captured, reordered, DSAX_FMT_REORDERED, mem);
}

int dsax_correlate(dsax_ctx *c, const void *in, void *vis, int mem) {
  return dsax_correlate_fmt(c, DSAX_FMT_CAPTURED, in, vis, mem, 0);
}

}  // extern "C"

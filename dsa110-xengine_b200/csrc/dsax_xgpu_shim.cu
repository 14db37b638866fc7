// dsax_xgpu_shim.cu -- xGPU-shaped entry points (include/xgpu_dsax.h) over
// the dsax C-ABI: a dsax context with the reference geometry, a device
// integration buffer, and the SYNCOP semantics of the reference call sites.
#include <cstring>
#include <new>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "../../include/xgpu_dsax.h"

namespace {

constexpr unsigned kNpol = 2, kNstation = 64, kNfreq = 768, kNtime = 2048, kNtimePipe = 128;
constexpr unsigned kNbl = kNstation * (kNstation + 1) / 2;

struct ShimState {
  dsax_ctx *ctx = nullptr;
  float *d_vis = nullptr;  // integration buffer
  int own_array = 0, own_matrix = 0;
};

}  // namespace

extern "C" {

void xgpuInfo(XGPUInfo *info) {
  if (!info) return;
  memset(info, 0, sizeof(*info));
  info->npol = kNpol;
  info->nstation = kNstation;
  info->nbaseline = kNbl;
  info->nfrequency = kNfreq;
  info->ntime = kNtime;
  info->ntimepipe = kNtimePipe;
  info->vecLength = (size_t)kNtime * kNfreq * kNstation * kNpol;
  info->vecLengthPipe = (size_t)kNtimePipe * kNfreq * kNstation * kNpol;
  info->matLength = (size_t)kNfreq * kNbl * kNpol * kNpol;
  info->triLength = info->matLength;
  info->matrix_order = TRIANGULAR_ORDER;
}

int xgpuInit(XGPUContext *context, int device_flags) {
  if (!context) return 1;
  XGPUInfo info;
  xgpuInfo(&info);
  ShimState *s = new (std::nothrow) ShimState();
  if (!s) return 2;
  dsax_config cfg;
  dsax_default_config(&cfg);
  cfg.npkt = kNtime;
  cfg.nant_in = kNstation;
  cfg.nchan = kNfreq / 2;
  const int dev = device_flags & 0xFFFF;
  int rc = dsax_create(&s->ctx, &cfg, dev);
  if (rc != DSAX_OK) {
    delete s;
    return 3;
  }
  context->array_len = info.vecLength;
  context->matrix_len = info.matLength;
  const size_t nvis = dsax_vis_bytes(&cfg);
  if (cudaMalloc((void **)&s->d_vis, nvis) != cudaSuccess ||
      cudaMemset(s->d_vis, 0, nvis) != cudaSuccess) {
    dsax_destroy(s->ctx);
    delete s;
    return 4;
  }
  if (!context->array_h) {
    if (dsax_host_alloc(s->ctx, context->array_len * sizeof(ComplexInput),
                        (void **)&context->array_h) != DSAX_OK)
      return 5;
    s->own_array = 1;
  }
  if (!context->matrix_h) {
    if (dsax_host_alloc(s->ctx, context->matrix_len * sizeof(Complex),
                        (void **)&context->matrix_h) != DSAX_OK)
      return 6;
    s->own_matrix = 1;
  }
  context->internal = s;
  return 0;
}

int xgpuCudaXengine(XGPUContext *context, ComplexInput *array_d, int syncOp) {
  if (!context || !context->internal || !array_d) return 1;
  ShimState *s = static_cast<ShimState *>(context->internal);
  int rc = dsax_correlate_fmt(s->ctx, DSAX_FMT_XGPU_INT8, array_d, s->d_vis, DSAX_MEM_DEVICE, 1);
  if (rc != DSAX_OK) return 10 - rc;
  cudaStream_t st = static_cast<cudaStream_t>(dsax_stream(s->ctx));
  if (syncOp == SYNCOP_DUMP) {
    if (cudaMemcpyAsync(context->matrix_h, s->d_vis, context->matrix_len * sizeof(Complex),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return 20;
  }
  if (syncOp != SYNCOP_NONE) {
    rc = dsax_sync(s->ctx);
    if (rc != DSAX_OK) return 10 - rc;
  }
  return 0;
}

void xgpuClearDeviceIntegrationBuffer(XGPUContext *context) {
  if (!context || !context->internal) return;
  ShimState *s = static_cast<ShimState *>(context->internal);
  cudaStream_t st = static_cast<cudaStream_t>(dsax_stream(s->ctx));
  cudaMemsetAsync(s->d_vis, 0, context->matrix_len * sizeof(Complex), st);
  cudaStreamSynchronize(st);
}

void xgpuReorderMatrix(Complex *matrix) { (void)matrix; }

void xgpuFree(XGPUContext *context) {
  if (!context || !context->internal) return;
  ShimState *s = static_cast<ShimState *>(context->internal);
  if (s->own_array && context->array_h) dsax_host_free(s->ctx, context->array_h);
  if (s->own_matrix && context->matrix_h) dsax_host_free(s->ctx, context->matrix_h);
  if (s->own_array) context->array_h = nullptr;
  if (s->own_matrix) context->matrix_h = nullptr;
  if (s->d_vis) cudaFree(s->d_vis);
  dsax_destroy(s->ctx);
  delete s;
  context->internal = nullptr;
}

}  // extern "C"

// dsax_extract.cu -- visibility post-processing after the correlator:
// simple_extract of src/dsaX_writevis.c:55-74 on the GPU.  For every
// baseline, channel and parallel hand (XX = pol-product 0, YY = 3) the two
// time slots f' = 2f, 2f+1 of the xGPU triangular matrix are averaged:
//   out[bl][f][pol][re, im] = 0.5 (V[2f][bl][3 pol] + V[2f+1][bl][3 pol]).
// dsax_correlate_extract runs the correlator into a device buffer and this
// kernel after it, so only the 1/16-size product leaves the GPU.
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

namespace dsax {

__global__ void extract_kernel(const float2 *__restrict__ vis, float2 *__restrict__ out, int nchan) {
  const int64_t n = (int64_t)2080 * nchan * 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int pol = (int)(i & 1);
    const int64_t bf = i >> 1;
    const int f = (int)(bf % nchan);
    const int bl = (int)(bf / nchan);
    const float2 a = vis[((2 * (int64_t)f) * 2080 + bl) * 4 + 3 * pol];
    const float2 b = vis[((2 * (int64_t)f + 1) * 2080 + bl) * 4 + 3 * pol];
    out[i] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
  }
}

int launch_extract(const float *vis, float *out, int nchan, cudaStream_t st) {
  extract_kernel<<<1184, 256, 0, st>>>(reinterpret_cast<const float2 *>(vis),
                                       reinterpret_cast<float2 *>(out), nchan);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

using namespace dsax;

extern "C" size_t dsax_extract_bytes(const dsax_config *c) {
  return c ? (size_t)2080 * c->nchan * 2 * 2 * sizeof(float) : 0;
}

extern "C" int dsax_extract(dsax_ctx *c, const void *vis, void *out, int mem) {
  if (!c || !vis || !out) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const size_t nvis = dsax_vis_bytes(&c->cfg), nout = dsax_extract_bytes(&c->cfg);
  if (mem == DSAX_MEM_DEVICE) {
    if (!aligned16(vis) || !aligned16(out)) return set_error(c, DSAX_ERR_ARG, "misaligned pointer");
    if (launch_extract(static_cast<const float *>(vis), static_cast<float *>(out), c->cfg.nchan,
                       c->stream) != 0)
      return cuda_check(c, cudaGetLastError(), "extract launch");
    return DSAX_OK;
  }
  int rc;
  if ((rc = ensure_buffer(c, c->vis_buf, nvis + nout + 256, "visibilities")) != DSAX_OK) return rc;
  float *dv = static_cast<float *>(c->vis_buf.ptr);
  float *dout = reinterpret_cast<float *>(static_cast<uint8_t *>(c->vis_buf.ptr) +
                                          ((nvis + 255) & ~(size_t)255));
  cudaError_t e = cudaMemcpyAsync(dv, vis, nvis, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "H2D visibilities");
  if (launch_extract(dv, dout, c->cfg.nchan, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "extract launch");
  if ((e = cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H extract");
  return dsax_sync(c);
}

extern "C" int dsax_correlate_extract(dsax_ctx *c, const void *blk, void *out, int mem) {
  if (!c || !blk || !out) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nvis = dsax_vis_bytes(&c->cfg), nout = dsax_extract_bytes(&c->cfg);
  int rc;
  // device visibilities, then (host mode) the input block and the product
  const size_t o_in = (nvis + 255) & ~(size_t)255, o_out = o_in + ((nin + 255) & ~(size_t)255);
  if ((rc = ensure_buffer(c, c->aux[AUX_EXTRACT], o_out + nout, "extract buffers")) != DSAX_OK)
    return rc;
  uint8_t *base = static_cast<uint8_t *>(c->aux[AUX_EXTRACT].ptr);
  float *dv = reinterpret_cast<float *>(base);
  const void *din = blk;
  if (mem == DSAX_MEM_HOST) {
    cudaError_t e = cudaMemcpyAsync(base + o_in, blk, nin, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "H2D block");
    din = base + o_in;
  } else if (!aligned16(blk) || !aligned16(out)) {
    return set_error(c, DSAX_ERR_ARG, "misaligned pointer");
  }
  if ((rc = dsax_correlate_fmt(c, DSAX_FMT_CAPTURED, din, dv, DSAX_MEM_DEVICE, 0)) != DSAX_OK)
    return rc;
  float *dout = mem == DSAX_MEM_DEVICE ? static_cast<float *>(out)
                                       : reinterpret_cast<float *>(base + o_out);
  if (launch_extract(dv, dout, c->cfg.nchan, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "extract launch");
  if (mem == DSAX_MEM_DEVICE) return DSAX_OK;
  cudaError_t e = cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "D2H extract");
  return dsax_sync(c);
}

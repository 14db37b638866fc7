// dsax_extract.cu -- visibility post-processing after the correlator:
// simple_extract of src/dsaX_writevis.c:55-74 on the GPU.  For every
// baseline, channel and parallel hand (XX = pol-product 0, YY = 3) the two
// time slots f' = 2f, 2f+1 of the xGPU triangular matrix are averaged:
//   out[bl][f][pol][re, im] = 0.5 (V[2f][bl][3 pol] + V[2f+1][bl][3 pol]).
// dsax_correlate_extract runs the correlator into a device buffer and this
// kernel after it, so only the 1/16-size product leaves the GPU.
// Options of the _ex forms: the "Greg" baseline order of
// src/dsaX_wrangleAndWrite.c gen_lookup / reorder_gh (:46-93) -- pairs
// (i, j >= i), i major -- and auto_extract (src/dsaX_wrangle.c:47-70): the
// real parts of both hands of every autocorrelation added into a caller
// spectrum array.
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

namespace dsax {

// Baseline k of the "Greg" order (row i holds pairs (i, i..63)) -> its
// index in xGPU's triangular order, where pair (i <= j) sits at j(j+1)/2 + i.
__device__ __forceinline__ int greg_to_xgpu(int k) {
  int i = 0;
  while (k >= 64 - i) {
    k -= 64 - i;
    ++i;
  }
  const int j = i + k;
  return j * (j + 1) / 2 + i;
}

__global__ void extract_kernel(const float2 *__restrict__ vis, float2 *__restrict__ out, int nchan,
                               int greg) {
  const int64_t n = (int64_t)2080 * nchan * 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int pol = (int)(i & 1);
    const int64_t bf = i >> 1;
    const int f = (int)(bf % nchan);
    const int blo = (int)(bf / nchan);
    const int bl = greg ? greg_to_xgpu(blo) : blo;
    const float2 a = vis[((2 * (int64_t)f) * 2080 + bl) * 4 + 3 * pol];
    const float2 b = vis[((2 * (int64_t)f + 1) * 2080 + bl) * 4 + 3 * pol];
    out[i] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
  }
}

// auto_extract: specs[a][f] += Re XX_a(f), then += Re YY_a(f), in that order
// and in FP32 as the reference's loop (both hands time-slot averaged as in
// simple_extract), for antennas a < nant.
__global__ void autos_kernel(const float2 *__restrict__ vis, float *__restrict__ specs, int nchan,
                             int nant) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nant * nchan) return;
  const int a = i / nchan, f = i - a * nchan;
  const int bl = a * (a + 1) / 2 + a;
  float s = specs[i];
#pragma unroll
  for (int pol = 0; pol < 2; ++pol) {
    const float r0 = vis[((2 * (int64_t)f) * 2080 + bl) * 4 + 3 * pol].x;
    const float r1 = vis[((2 * (int64_t)f + 1) * 2080 + bl) * 4 + 3 * pol].x;
    s += 0.5f * (r0 + r1);
  }
  specs[i] = s;
}

int launch_extract(const float *vis, float *out, int nchan, int greg, float *autos, int nant,
                   cudaStream_t st) {
  if (out)
    extract_kernel<<<1184, 256, 0, st>>>(reinterpret_cast<const float2 *>(vis),
                                         reinterpret_cast<float2 *>(out), nchan, greg);
  if (autos)
    autos_kernel<<<(nant * nchan + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float2 *>(vis),
                                                             autos, nchan, nant);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

using namespace dsax;

extern "C" size_t dsax_extract_bytes(const dsax_config *c) {
  return c ? (size_t)2080 * c->nchan * 2 * 2 * sizeof(float) : 0;
}

extern "C" int dsax_extract_ex(dsax_ctx *c, const void *vis, void *out, int order, float *autos,
                               int mem) {
  if (!c || !vis || (!out && !autos)) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  if (order != DSAX_BL_XGPU && order != DSAX_BL_GREG) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const int nant = c->cfg.nant_in, nchan = c->cfg.nchan;
  const size_t nvis = dsax_vis_bytes(&c->cfg), nout = dsax_extract_bytes(&c->cfg);
  const size_t nauto = (size_t)nant * nchan * sizeof(float);
  if (mem == DSAX_MEM_DEVICE) {
    if (!aligned16(vis) || (out && !aligned16(out)))
      return set_error(c, DSAX_ERR_ARG, "misaligned pointer");
    if (launch_extract(static_cast<const float *>(vis), static_cast<float *>(out), nchan, order,
                       autos, nant, c->stream) != 0)
      return cuda_check(c, cudaGetLastError(), "extract launch");
    return DSAX_OK;
  }
  int rc;
  const size_t o_out = (nvis + 255) & ~(size_t)255, o_auto = o_out + ((nout + 255) & ~(size_t)255);
  if ((rc = ensure_buffer(c, c->vis_buf, o_auto + nauto, "visibilities")) != DSAX_OK) return rc;
  uint8_t *base = static_cast<uint8_t *>(c->vis_buf.ptr);
  float *dv = reinterpret_cast<float *>(base);
  float *dout = out ? reinterpret_cast<float *>(base + o_out) : nullptr;
  float *dauto = autos ? reinterpret_cast<float *>(base + o_auto) : nullptr;
  cudaError_t e = cudaMemcpyAsync(dv, vis, nvis, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "H2D visibilities");
  if (autos && (e = cudaMemcpyAsync(dauto, autos, nauto, cudaMemcpyHostToDevice, c->stream)) !=
                   cudaSuccess)
    return cuda_check(c, e, "H2D autos");
  if (launch_extract(dv, dout, nchan, order, dauto, nant, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "extract launch");
  if (out && (e = cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H extract");
  if (autos && (e = cudaMemcpyAsync(autos, dauto, nauto, cudaMemcpyDeviceToHost, c->stream)) !=
                   cudaSuccess)
    return cuda_check(c, e, "D2H autos");
  return dsax_sync(c);
}

extern "C" int dsax_extract(dsax_ctx *c, const void *vis, void *out, int mem) {
  if (!out) return DSAX_ERR_ARG;
  return dsax_extract_ex(c, vis, out, DSAX_BL_XGPU, nullptr, mem);
}

extern "C" int dsax_correlate_extract(dsax_ctx *c, const void *blk, void *out, int mem) {
  if (!out) return DSAX_ERR_ARG;
  return dsax_correlate_extract_ex(c, blk, out, DSAX_BL_XGPU, nullptr, mem);
}

extern "C" int dsax_correlate_extract_ex(dsax_ctx *c, const void *blk, void *out, int order,
                                         float *autos, int mem) {
  if (!c || !blk || (!out && !autos)) return DSAX_ERR_ARG;
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  if (order != DSAX_BL_XGPU && order != DSAX_BL_GREG) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const int nant = c->cfg.nant_in, nchan = c->cfg.nchan;
  const size_t nin = dsax_block_bytes(&c->cfg, DSAX_FMT_CAPTURED);
  const size_t nvis = dsax_vis_bytes(&c->cfg), nout = dsax_extract_bytes(&c->cfg);
  const size_t nauto = (size_t)nant * nchan * sizeof(float);
  int rc;
  // device visibilities, then (host mode) the input block, the product and
  // the autocorrelation spectra
  const size_t o_in = (nvis + 255) & ~(size_t)255, o_out = o_in + ((nin + 255) & ~(size_t)255);
  const size_t o_auto = o_out + ((nout + 255) & ~(size_t)255);
  if ((rc = ensure_buffer(c, c->aux[AUX_EXTRACT], o_auto + nauto, "extract buffers")) != DSAX_OK)
    return rc;
  uint8_t *base = static_cast<uint8_t *>(c->aux[AUX_EXTRACT].ptr);
  float *dv = reinterpret_cast<float *>(base);
  const void *din = blk;
  cudaError_t e;
  if (mem == DSAX_MEM_HOST) {
    e = cudaMemcpyAsync(base + o_in, blk, nin, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "H2D block");
    din = base + o_in;
    if (autos && (e = cudaMemcpyAsync(base + o_auto, autos, nauto, cudaMemcpyHostToDevice,
                                      c->stream)) != cudaSuccess)
      return cuda_check(c, e, "H2D autos");
  } else if (!aligned16(blk) || (out && !aligned16(out))) {
    return set_error(c, DSAX_ERR_ARG, "misaligned pointer");
  }
  if ((rc = dsax_correlate_fmt(c, DSAX_FMT_CAPTURED, din, dv, DSAX_MEM_DEVICE, 0)) != DSAX_OK)
    return rc;
  float *dout = !out ? nullptr
                : mem == DSAX_MEM_DEVICE ? static_cast<float *>(out)
                                         : reinterpret_cast<float *>(base + o_out);
  float *dauto = !autos ? nullptr
                 : mem == DSAX_MEM_DEVICE ? autos : reinterpret_cast<float *>(base + o_auto);
  if (launch_extract(dv, dout, nchan, order, dauto, nant, c->stream) != 0)
    return cuda_check(c, cudaGetLastError(), "extract launch");
  if (mem == DSAX_MEM_DEVICE) return DSAX_OK;
  if (out && (e = cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H extract");
  if (autos && (e = cudaMemcpyAsync(autos, dauto, nauto, cudaMemcpyDeviceToHost, c->stream)) !=
                   cudaSuccess)
    return cuda_check(c, e, "D2H autos");
  return dsax_sync(c);
}

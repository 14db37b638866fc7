// dsax_reorder.cu -- the packet corner turn of src/dsaX_reorder_raw.c
// massage() (:153-169) on the GPU: captured [pkt][nant_in][nchan][2 t][2 pol]
// -> xGPU order [pkt][2*nchan][64][2 pol], one packed 4+4-bit byte per
// sample, padded antennas zero (the reference leaves them as the ring
// buffer's previous bytes).  HBM-bound byte transpose staged through shared
// memory: 128-byte antenna rows in, 128-byte frequency rows out.
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"

namespace dsax {

namespace reorder {
constexpr int kChan = 32;        // channels per CTA (128 bytes of each antenna row)
constexpr int kThreads = 256;
constexpr int kStride = kChan + 1;  // padded shared-memory row (words)
}  // namespace reorder

__global__ void __launch_bounds__(reorder::kThreads) reorder_kernel(const uint8_t *__restrict__ in,
                                                                    uint8_t *__restrict__ out,
                                                                    int npkt, int nant_in,
                                                                    int nchan) {
  using namespace reorder;
  __shared__ uint32_t W[64 * kStride];  // [ant][chan] words = {t0p0, t0p1, t1p0, t1p1}
  const int p = blockIdx.y;
  const int c0 = blockIdx.x * kChan;
  const int nc = min(kChan, nchan - c0);
  const uint32_t *src = reinterpret_cast<const uint32_t *>(in) + ((int64_t)p * nant_in) * nchan + c0;
  for (int i = threadIdx.x; i < 64 * kChan; i += kThreads) {
    const int a = i / kChan, c = i % kChan;
    W[a * kStride + c] = (a < nant_in && c < nc) ? __ldg(src + (int64_t)a * nchan + c) : 0u;
  }
  __syncthreads();
  // thread -> (antenna group of 8, channel): two 16-byte output chunks
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ag = lane & 7;
  const int c = 4 * warp + (lane >> 3);
  if (c < nc) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = W[(8 * ag + i) * kStride + c];
    uint4 lo, hi;  // t = 0 halves, t = 1 halves
    lo.x = __byte_perm(w[0], w[1], 0x5410u); hi.x = __byte_perm(w[0], w[1], 0x7632u);
    lo.y = __byte_perm(w[2], w[3], 0x5410u); hi.y = __byte_perm(w[2], w[3], 0x7632u);
    lo.z = __byte_perm(w[4], w[5], 0x5410u); hi.z = __byte_perm(w[4], w[5], 0x7632u);
    lo.w = __byte_perm(w[6], w[7], 0x5410u); hi.w = __byte_perm(w[6], w[7], 0x7632u);
    uint8_t *row = out + (((int64_t)p * 2 * nchan + 2 * (c0 + c)) * 64) * 2 + 16 * ag;
    *reinterpret_cast<uint4 *>(row) = lo;
    *reinterpret_cast<uint4 *>(row + 128) = hi;
  }
}

int launch_reorder(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                   cudaStream_t st) {
  if (npkt < 1 || npkt > 65535 || nant_in < 1 || nant_in > 64 || nchan < 1) return -1;
  dim3 grid((nchan + reorder::kChan - 1) / reorder::kChan, npkt);
  reorder_kernel<<<grid, reorder::kThreads, 0, st>>>(in, out, npkt, nant_in, nchan);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

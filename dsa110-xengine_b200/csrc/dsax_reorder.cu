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

namespace dsax {

namespace reorder_cm {
constexpr int kPkt = 4;          // packets per CTA
constexpr int kChan = 32;        // channels per CTA
constexpr int kThreads = 256;
constexpr int kAStride = 65;     // words per channel row (64 antennas + 1 pad)
}  // namespace reorder_cm

// Captured [pkt][nant_in][nchan][4 B] -> channel-major [nchan][npkt][64][4 B]
// (padded antennas zero): each channel's samples become one contiguous
// stream, so the correlator can fetch a 64-packet stage with one bulk copy.
__global__ void __launch_bounds__(reorder_cm::kThreads) reorder_cm_kernel(
    const uint8_t *__restrict__ in, uint8_t *__restrict__ out, int npkt, int nant_in, int nchan) {
  using namespace reorder_cm;
  __shared__ uint32_t W[kPkt * kChan * kAStride];  // [pkt][chan][ant]
  const int c0 = blockIdx.x * kChan;
  const int p0 = blockIdx.y * kPkt;
  const int nc = min(kChan, nchan - c0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // load: lanes cover 8 x 16 B (32 channels) of 4 antenna rows; each warp
  // issues all of its rows' loads before the shared-memory stores, so eight
  // 16-byte loads per thread are in flight
  constexpr int kRows = kPkt * 16 / (kThreads / 32);   // rows per warp
  uint4 v[kRows];
#pragma unroll
  for (int i = 0; i < kRows; ++i) {
    const int r = warp + i * (kThreads / 32);           // 4 pkts x 16 groups of 4 ants
    const int pq = r >> 4;
    const int a = 4 * (r & 15) + (lane >> 3);
    const int cq = lane & 7;
    const int p = p0 + pq;
    v[i] = make_uint4(0u, 0u, 0u, 0u);
    if (p < npkt && a < nant_in && 4 * cq < nc) {
      const uint8_t *src = in + (((int64_t)p * nant_in + a) * nchan + c0 + 4 * cq) * 4;
      if (4 * cq + 4 <= nc && ((nchan & 3) == 0)) {
        v[i] = __ldg(reinterpret_cast<const uint4 *>(src));
      } else {
        const uint32_t *s32 = reinterpret_cast<const uint32_t *>(src);
        v[i].x = s32[0];
        v[i].y = 4 * cq + 1 < nc ? s32[1] : 0u;
        v[i].z = 4 * cq + 2 < nc ? s32[2] : 0u;
        v[i].w = 4 * cq + 3 < nc ? s32[3] : 0u;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kRows; ++i) {
    const int r = warp + i * (kThreads / 32);
    const int pq = r >> 4;
    const int a = 4 * (r & 15) + (lane >> 3);
    const int cq = lane & 7;
    uint32_t *w = W + (pq * kChan + 4 * cq) * kAStride + a;
    w[0] = v[i].x;
    w[kAStride] = v[i].y;
    w[2 * kAStride] = v[i].z;
    w[3 * kAStride] = v[i].w;
  }
  __syncthreads();
  // store: per channel, kPkt x 256 B contiguous; a warp writes one channel
  for (int c = warp; c < nc; c += kThreads / 32) {
    uint8_t *dst = out + ((int64_t)(c0 + c) * npkt + p0) * 256;
#pragma unroll
    for (int k = lane; k < kPkt * 16; k += 32) {   // 16-byte chunks
      const int pq = k >> 4, a = 4 * (k & 15);
      if (p0 + pq >= npkt) continue;
      const uint32_t *w = W + (pq * kChan + c) * kAStride + a;
      *reinterpret_cast<uint4 *>(dst + 16 * k) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

int launch_reorder_chanmajor(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                             cudaStream_t st) {
  using namespace reorder_cm;
  if (npkt < 1 || nant_in < 1 || nant_in > 64 || nchan < 1) return -1;
  dim3 grid((nchan + kChan - 1) / kChan, (npkt + kPkt - 1) / kPkt);
  if (grid.y > 65535) return -1;
  reorder_cm_kernel<<<grid, kThreads, 0, st>>>(in, out, npkt, nant_in, nchan);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

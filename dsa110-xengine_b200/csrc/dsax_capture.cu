// dsax_capture.cu -- packet placement for block assembly on the GPU
// (src/dsaX_capture.c receive_obs :870-960), for packets already in device
// memory (e.g. a GPUDirect-style ingest buffer).  Each packet is an 8-byte
// header and a payload; the header holds (big-endian) a 35-bit sequence
// number in bytes 0-4 (top 3 bits of byte 4), a 13-bit channel id and a
// 16-bit antenna id in bytes 6-7 (:872-891).  The payload goes to slot
//   act = seq_no * slots_per_seq + ant_lookup[ant_id]   (:897)
// of the current block (slots act0 .. act0 + nslots - 1, :925-948); later
// slots go to the next block if one is given (the reference keeps them in
// temp buffers for it, :950-960), earlier ones are dropped as late.  Each
// CTA places one packet with 8-byte vector copies.  Counters (uint64):
// [0] placed in the block, [1] placed in the next block, [2] late,
// [3] beyond the next block or unknown antenna.
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

namespace dsax {

__global__ void place_packets_kernel(const uint8_t *__restrict__ pkts, int npk, int stride,
                                     int payload, const int *__restrict__ ant_lookup, int nlookup,
                                     uint64_t act0, uint64_t nslots, int slots_per_seq,
                                     uint8_t *block, uint8_t *next, unsigned long long *counts) {
  __shared__ long long dst_slot;
  __shared__ int which;
  for (int k = blockIdx.x; k < npk; k += gridDim.x) {
    const uint8_t *p = pkts + (int64_t)k * stride;
    if (threadIdx.x == 0) {
      uint64_t seq = ((uint64_t)(p[4] & 0xE0) >> 5) | ((uint64_t)p[3] << 3) | ((uint64_t)p[2] << 11) |
                     ((uint64_t)p[1] << 19) | ((uint64_t)p[0] << 27);
      const int ant_id = ((int)p[6] << 8) | (int)p[7];
      const int aid = ant_id < nlookup ? ant_lookup[ant_id] : -1;
      which = 3;
      dst_slot = -1;
      if (aid >= 0) {
        const uint64_t act = seq * (uint64_t)slots_per_seq + (uint64_t)aid;
        if (act < act0) {
          which = 2;
        } else if (act - act0 < nslots) {
          which = 0;
          dst_slot = (long long)(act - act0);
        } else if (next && act - act0 < 2 * nslots) {
          which = 1;
          dst_slot = (long long)(act - act0 - nslots);
        }
      }
      atomicAdd(counts + which, 1ull);
    }
    __syncthreads();
    if (which <= 1) {
      uint8_t *dst = (which == 0 ? block : next) + dst_slot * (int64_t)payload;
      const uint2 *src = reinterpret_cast<const uint2 *>(p + 8);
      uint2 *d = reinterpret_cast<uint2 *>(dst);
      for (int i = threadIdx.x; i < payload / 8; i += blockDim.x) d[i] = src[i];
    }
    __syncthreads();
  }
}

}  // namespace dsax

using namespace dsax;

extern "C" int dsax_place_packets(dsax_ctx *c, const void *pkts, int npk, int stride, int payload,
                                  const int *ant_lookup, int nlookup, unsigned long long act0,
                                  unsigned long long nslots, int slots_per_seq, void *block,
                                  void *next_block, unsigned long long *counts) {
  if (!c || !pkts || npk < 0 || payload < 8 || payload % 8 || stride < payload + 8 || stride % 8 ||
      !ant_lookup || nlookup < 1 || slots_per_seq < 1 || !block || !counts)
    return DSAX_ERR_ARG;
  if (npk == 0) return DSAX_OK;
  DeviceGuard g(c->device);
  const int grid = npk < 4 * c->num_sms ? npk : 4 * c->num_sms;
  place_packets_kernel<<<grid, 256, 0, c->stream>>>(
      static_cast<const uint8_t *>(pkts), npk, stride, payload, ant_lookup, nlookup, act0, nslots,
      slots_per_seq, static_cast<uint8_t *>(block), static_cast<uint8_t *>(next_block), counts);
  return cudaGetLastError() == cudaSuccess ? DSAX_OK
                                           : cuda_check(c, cudaGetLastError(), "packet placement");
}

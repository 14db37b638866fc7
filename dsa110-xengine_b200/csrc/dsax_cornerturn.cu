// dsax_cornerturn.cu -- the beam corner turn between the beamformer and the
// search-side flagger, as two device-side reorders around one all-to-all.
//
// The reference does it over sockets: every subband node (dsaX_dbnic)
// transposes its beamformer output [t][256 beams][48 ch] into one
// [64 beams][t][48 ch] message per search node (src/dsaX_dbnic.c:84-152),
// and every search node (dsaX_nicdb) places the 16 subbands' messages at
// channel CHOFF/8 + chgroup*48 of its [64 beams][16384 t][1024 ch]
// filterbank (src/dsaX_nicdb.c:180-196).  Here a GPU per subband packs its
// beams into one contiguous chunk per destination (dsax_ct_pack), an NCCL
// all-to-all over NVLink moves the chunks (the caller's collective:
// dsax.dist.beam_corner_turn), and the destination places them into its
// filterbank (dsax_ct_unpack), which dsax_flag_clean then reads as uint8.
// Both reorders are byte moves of whole channel rows: HBM-bound, 16-byte
// loads and stores when the row length allows.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

namespace dsax {

// in [nt][nb][nc] -> out [ndest][nb/ndest][nt][nc]: one row of nc bytes per
// (t, beam); thread = one 16-byte (or 1-byte) piece.
template <int V>
__global__ void ct_pack_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, int nt,
                               int nb, int nc, int ndest) {
  const int nbl = nb / ndest, pr = nc / V;
  const int64_t n = (int64_t)nt * nb * pr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / pr;
    const int p = (int)(i - row * pr);
    const int t = (int)(row / nb), b = (int)(row - (int64_t)t * nb);
    const int d = b / nbl, j = b - d * nbl;
    const int64_t o = (((int64_t)d * nbl + j) * nt + t) * nc + (int64_t)p * V;
    if constexpr (V == 16)
      *reinterpret_cast<uint4 *>(out + o) = *reinterpret_cast<const uint4 *>(in + row * nc + p * V);
    else
      out[o] = in[row * nc + p];
  }
}

// recv [nsrc][nbl][nt][nc] -> fil[nbl][t0 + t][ch0 + s nc + k] of a
// filterbank with fil_nt samples and fil_nc channels per row.
template <int V>
__global__ void ct_unpack_kernel(const uint8_t *__restrict__ recv, uint8_t *__restrict__ fil,
                                 int nsrc, int nbl, int nt, int nc, int fil_nt, int fil_nc, int t0,
                                 int ch0) {
  const int pr = nc / V;
  const int64_t n = (int64_t)nsrc * nbl * nt * pr;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / pr;
    const int p = (int)(i - row * pr);
    const int t = (int)(row % nt);
    const int64_t sb = row / nt;
    const int j = (int)(sb % nbl), s = (int)(sb / nbl);
    const int64_t o = ((int64_t)j * fil_nt + t0 + t) * fil_nc + ch0 + (int64_t)s * nc + (int64_t)p * V;
    if constexpr (V == 16)
      *reinterpret_cast<uint4 *>(fil + o) = *reinterpret_cast<const uint4 *>(recv + row * nc + p * V);
    else
      fil[o] = recv[row * nc + p];
  }
}

}  // namespace dsax

using namespace dsax;

extern "C" int dsax_ct_pack(dsax_ctx *c, const uint8_t *beams, int nt, int nb, int nc, int ndest,
                            uint8_t *send) {
  if (!c || !beams || !send || nt < 1 || nb < 1 || nc < 1 || ndest < 1 || nb % ndest)
    return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const bool v16 = nc % 16 == 0 && aligned16(beams) && aligned16(send);
  const int64_t n = (int64_t)nt * nb * (v16 ? nc / 16 : nc);
  const int grid = (int)((n + 255) / 256 < 8 * (int64_t)c->num_sms ? (n + 255) / 256
                                                                     : 8 * (int64_t)c->num_sms);
  if (v16)
    ct_pack_kernel<16><<<grid, 256, 0, c->stream>>>(beams, send, nt, nb, nc, ndest);
  else
    ct_pack_kernel<1><<<grid, 256, 0, c->stream>>>(beams, send, nt, nb, nc, ndest);
  return cuda_check(c, cudaGetLastError(), "corner-turn pack");
}

extern "C" int dsax_ct_unpack(dsax_ctx *c, const uint8_t *recv, int nsrc, int nbl, int nt, int nc,
                              uint8_t *fil, int fil_nt, int fil_nc, int t0, int ch0) {
  if (!c || !recv || !fil || nsrc < 1 || nbl < 1 || nt < 1 || nc < 1 || t0 < 0 || ch0 < 0 ||
      t0 + nt > fil_nt || ch0 + nsrc * nc > fil_nc)
    return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const bool v16 = nc % 16 == 0 && fil_nc % 16 == 0 && ch0 % 16 == 0 && aligned16(recv) &&
                   aligned16(fil);
  const int64_t n = (int64_t)nsrc * nbl * nt * (v16 ? nc / 16 : nc);
  const int grid = (int)((n + 255) / 256 < 8 * (int64_t)c->num_sms ? (n + 255) / 256
                                                                     : 8 * (int64_t)c->num_sms);
  if (v16)
    ct_unpack_kernel<16><<<grid, 256, 0, c->stream>>>(recv, fil, nsrc, nbl, nt, nc, fil_nt, fil_nc,
                                                      t0, ch0);
  else
    ct_unpack_kernel<1><<<grid, 256, 0, c->stream>>>(recv, fil, nsrc, nbl, nt, nc, fil_nt, fil_nc,
                                                     t0, ch0);
  return cuda_check(c, cudaGetLastError(), "corner-turn unpack");
}

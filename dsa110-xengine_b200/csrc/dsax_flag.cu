// dsax_flag.cu -- the plain RFI flagger on the GPU: one HBM pass for all
// per-(beam, channel) and per-(beam, time) statistics, then the
// median/MAD decisions on the device (the reference does them on the host).
//
// Replaces src/gpu_flagger.cu: calc_spectrum (:175-223), calc_varspec
// (:229-278), calc_maxspec (:283-319; the reference calls calc_spectrum in
// its place at :1334 -- parity mode keeps that), calc_ppspec (:324-376),
// make_ts (:414-453), and the host decisions medval/channflag/
// simple_channflag/simple_tsflag (:534-720) run in the order of
// :1340-1398.  The shapes the reference hard-codes ([64][16384][1024],
// ZeroChannels 128, nFiltSize 21, TBIN 128, FBIN 8, T/16) are parameters.
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_ptx.cuh"
#include "../../include/dsax.h"

namespace dsax {

namespace flag {
constexpr int kStatThreads = 512;   // 16 warps per beam
constexpr int kMaxChan = 128;       // four channels per lane
constexpr int kDecThreads = 256;
}  // namespace flag

// ---------------------------------------------------------------- stats
// One CTA per beam.  Warp w owns the TBIN-sample bins w, w+16, ...; lane l
// owns channels l, l+32, l+64, l+96.  Sums are FP64 in sample order within a
// bin (the oracle's order), max/bin extremes exact.
__global__ void __launch_bounds__(flag::kStatThreads) flag_stats_kernel(FlagArgs a) {
  constexpr int NL = flag::kMaxChan / 32;   // channels per lane
  const int b = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const int T = a.ntime, C = a.nchan, TB = a.tbin;
  const int nbins = T / TB;
  const float *xb = a.x + (int64_t)b * T * C;

  double s[NL], q[NL], bmax[NL], bmin[NL], bs[NL];
  float m[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    s[k] = 0.0; q[k] = 0.0; bmax[k] = -1e300; bmin[k] = 1e300; m[k] = -INFINITY;
  }
  auto row = [&](int t, bool bin) {
    const float *rp = xb + (int64_t)t * C;
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      const int c = lane + 32 * k;
      const float v = c < C ? __ldg(rp + c) : 0.0f;
      if (bin) bs[k] += v; else s[k] += v;
      q[k] += (double)v * v;
      if (c < C) m[k] = fmaxf(m[k], v);
      r += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (lane == 0) a.ts[(int64_t)b * T + t] = (float)(r / C);
  };
  for (int bin = warp; bin < nbins; bin += nw) {
#pragma unroll
    for (int k = 0; k < NL; ++k) bs[k] = 0.0;
    for (int t = bin * TB; t < (bin + 1) * TB; ++t) row(t, true);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      s[k] += bs[k];
      const double mb = bs[k] / TB;
      bmax[k] = fmax(bmax[k], mb);
      bmin[k] = fmin(bmin[k], mb);
    }
  }
  // samples beyond the last whole bin (T % TB): sums and max only
  for (int t = nbins * TB + warp; t < T; t += nw) row(t, false);

  extern __shared__ double fsh[];
  double *sh_s = fsh, *sh_q = sh_s + 16 * flag::kMaxChan;
  double *sh_bmax = sh_q + 16 * flag::kMaxChan, *sh_bmin = sh_bmax + 16 * flag::kMaxChan;
  float *sh_m = reinterpret_cast<float *>(sh_bmin + 16 * flag::kMaxChan);
#pragma unroll
  for (int k = 0; k < NL; ++k) {
    const int c = lane + 32 * k;
    sh_s[warp * flag::kMaxChan + c] = s[k];
    sh_q[warp * flag::kMaxChan + c] = q[k];
    sh_m[warp * flag::kMaxChan + c] = m[k];
    sh_bmax[warp * flag::kMaxChan + c] = bmax[k];
    sh_bmin[warp * flag::kMaxChan + c] = bmin[k];
  }
  __syncthreads();
  if (threadIdx.x < C) {
    const int c = threadIdx.x;
    double ss = 0.0, qq = 0.0, bx = -1e300, bn = 1e300;
    float mm = -INFINITY;
    for (int w = 0; w < nw; ++w) {
      ss += sh_s[w * flag::kMaxChan + c]; qq += sh_q[w * flag::kMaxChan + c];
      mm = fmaxf(mm, sh_m[w * flag::kMaxChan + c]);
      bx = fmax(bx, sh_bmax[w * flag::kMaxChan + c]); bn = fmin(bn, sh_bmin[w * flag::kMaxChan + c]);
    }
    const double mean = ss / T;
    const double var = fmax(qq / T - mean * mean, 0.0);
    const int o = b * C + c;
    a.spec[o] = (float)mean;
    a.var[o] = (float)var;
    a.maxs[o] = a.parity ? (float)mean : mm;
    a.pp[o] = nbins > 0 ? (float)(bx - bn) : 0.0f;
  }
}

// ---------------------------------------------------------------- decisions
// Lower median sorted[(n+1)/2 - 1] of v[0..n) in shared memory, by rank
// counting with ties broken by index (the element a stable sort would put
// at that position has the same value).  All threads of the block call it.
__device__ float block_lower_median(const float *v, int n, float *result_slot) {
  const int k = (n + 1) / 2 - 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = v[i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const float y = v[j];
      r += (y < x) || (y == x && j < i);
    }
    if (r == k) *result_slot = x;
  }
  __syncthreads();
  const float med = *result_slot;
  __syncthreads();
  return med;
}

// channflag() on one statistic of one beam: forward median detrend over
// `filt` channels (the last windows clamped at C-G-filt), median and MAD
// over the guard-banded channels, flag |x| > thr*MAD.
__device__ void channflag_dev(const float *sb, float thr, const FlagArgs &a, uint8_t *mask,
                              float *corr, float *tmp, float *slot) {
  const int C = a.nchan, G = a.guard, F = a.filt, n = C - 2 * G;
  for (int j = G + threadIdx.x; j < C - G; j += blockDim.x) {
    const int w0 = (C - G - j >= F) ? j : C - G - F;
    const int k = (F + 1) / 2 - 1;
    float med = 0.0f;
    for (int i = 0; i < F; ++i) {   // rank-count median of the window
      const float x = sb[w0 + i];
      int r = 0;
      for (int q = 0; q < F; ++q) {
        const float y = sb[w0 + q];
        r += (y < x) || (y == x && q < i);
      }
      if (r == k) med = x;
    }
    corr[j - G] = sb[j] - med;
  }
  __syncthreads();
  const float med = block_lower_median(corr, n, slot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = fabsf(corr[i] - med);
  __syncthreads();
  const float mad = block_lower_median(tmp, n, slot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float v = corr[i];
    if (v > thr * mad || v < -thr * mad) mask[G + i] = 1;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(flag::kDecThreads) flag_decide_kernel(FlagArgs a) {
  const int b = blockIdx.x;
  const int C = a.nchan, G = a.guard, T = a.ntime, n = C - 2 * G;
  extern __shared__ float dsh[];
  float *spec = dsh;                    // C
  float *corr = spec + C;               // C
  float *tmp = corr + C;                // max(C, ts_base)
  float *tsb = tmp + (a.ts_base > C ? a.ts_base : C);  // ts_base
  __shared__ uint8_t cmask[flag::kMaxChan * 2];
  __shared__ float slot;

  for (int c = threadIdx.x; c < C; c += blockDim.x) cmask[c] = 0;
  __syncthreads();

  // 1) channflag(spec - oldspec, Thr)
  for (int c = threadIdx.x; c < C; c += blockDim.x)
    spec[c] = a.spec[b * C + c] - (a.oldspec ? a.oldspec[b * C + c] : 0.0f);
  __syncthreads();
  channflag_dev(spec, a.thresh, a, cmask, corr, tmp, &slot);
  // 2) channflag(var, Thr + 0.5)
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.var[b * C + c];
  __syncthreads();
  channflag_dev(spec, a.thresh + a.var_add, a, cmask, corr, tmp, &slot);
  // 3) channflag(max, Thr)
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.maxs[b * C + c];
  __syncthreads();
  channflag_dev(spec, a.thresh, a, cmask, corr, tmp, &slot);
  // 4) simple_channflag(pp, Thr): one-sided, Thr/sqrt(FBIN)
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.pp[b * C + c];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) corr[i] = spec[G + i];
  __syncthreads();
  {
    const float med = block_lower_median(corr, n, &slot);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = fabsf(corr[i] - med);
    __syncthreads();
    const float mad = block_lower_median(tmp, n, &slot);
    const float mythr = a.thresh / sqrtf((float)a.fbin);
    for (int j = G + threadIdx.x; j < C - G - a.fbin; j += blockDim.x) {
      float vv = 0.0f;
      for (int k = 0; k < a.fbin; ++k) vv += a.parity ? spec[j] : spec[j + k];
      vv = vv / (float)a.fbin - med;
      if (vv > mythr * mad) cmask[j] = 1;
    }
  }
  __syncthreads();
  for (int k = 0; k < a.nperm; ++k) {
    const int j = a.perm[k];
    if (threadIdx.x == 0 && j >= G && j < C - G) cmask[j] = 1;
  }
  __syncthreads();
  int nflag = 0;
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    a.chanmask[b * C + c] = cmask[c];
    nflag += cmask[c];
  }
  if (nflag) atomicAdd(a.counts, nflag);

  // 5) simple_tsflag(ts, TsThr): median/MAD over the first ts_base samples
  const float *tb = a.ts + (int64_t)b * T;
  if (a.tsflag) {
    for (int i = threadIdx.x; i < a.ts_base; i += blockDim.x) tsb[i] = tb[i];
    __syncthreads();
    const float med = block_lower_median(tsb, a.ts_base, &slot);
    for (int i = threadIdx.x; i < a.ts_base; i += blockDim.x) tmp[i] = fabsf(tsb[i] - med);
    __syncthreads();
    const float mad = block_lower_median(tmp, a.ts_base, &slot);
    int nts = 0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      const uint8_t f = (tb[t] - med) > a.ts_thresh * mad ? 1 : 0;
      a.tsmask[(int64_t)b * T + t] = f;
      nts += f;
    }
    if (nts) atomicAdd(a.counts + 1, nts);
  } else {
    for (int t = threadIdx.x; t < T; t += blockDim.x) a.tsmask[(int64_t)b * T + t] = 0;
  }
}

int launch_flag(const FlagArgs &a, cudaStream_t st) {
  if (a.nchan > flag::kMaxChan || a.ts_base > 4096) return -1;
  static bool attr = false;
  const size_t ssh = 16 * flag::kMaxChan * (4 * sizeof(double) + sizeof(float));
  if (!attr) {
    cudaFuncSetAttribute(flag_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssh);
    attr = true;
  }
  flag_stats_kernel<<<a.nbeam, flag::kStatThreads, ssh, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return -2;
  const int tmpn = a.ts_base > a.nchan ? a.ts_base : a.nchan;
  const size_t sh = sizeof(float) * (2 * a.nchan + tmpn + a.ts_base);
  flag_decide_kernel<<<a.nbeam, flag::kDecThreads, sh, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

// ---------------------------------------------------------------------------
// Allocation-free variant of the plain flagger for callers that cannot call
// cudaMalloc (a process whose device memory is owned by another runtime or
// pool, a real-time thread that must not enter the allocator, or code that
// runs while a CUDA graph is being recorded by someone else).  The
// statistics live in this file-scope device array instead of a context
// buffer: every GPU that loads the library holds it until the process
// exits, every call shares it, and it keeps the last call's contents.
namespace dsax {

constexpr long long kNoAllocScratchFloats = 1572864;  // 6 MiB
static __device__ __align__(256) float g_flag_scratch[kNoAllocScratchFloats];

namespace {
constexpr int kMaxDevices = 64;
float *g_scratch_addr[kMaxDevices] = {};   // device address per device, set up once
}  // namespace

// Resolves the array's device address on the current device (once per
// device).  Returns nullptr on failure.
static float *noalloc_scratch(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_flag_scratch) != cudaSuccess) return nullptr;
    g_scratch_addr[dev] = static_cast<float *>(p);
  }
  return g_scratch_addr[dev];
}

}  // namespace dsax

extern "C" int dsax_flag_noalloc(const dsax_flag_params *p, const float *x, const float *oldspec,
                                 uint8_t *chanmask, uint8_t *tsmask, int *counts, void *stream) {
  using namespace dsax;
  if (!p || !x || !chanmask || !tsmask) return DSAX_ERR_ARG;
  const int B = p->nbeam, T = p->ntime, C = p->nchan;
  if (B < 1 || T < 1 || C < 1 || C > 128 || p->guard < 0 || C - 2 * p->guard < 1 ||
      p->filt < 1 || p->filt > C - 2 * p->guard || p->tbin < 1 || p->fbin < 1 ||
      p->ts_base < 1 || p->ts_base > T || p->ts_base > 4096 || p->nperm < 0 || p->nperm > 8)
    return DSAX_ERR_ARG;
  const long long nbc = (long long)B * C, nbt = (long long)B * T;
  const long long need = 4 * nbc + nbt + 2;   // spec, var, max, pp, ts, two counters
  if (need > kNoAllocScratchFloats) return DSAX_ERR_ARG;   // beyond the fixed 6 MiB
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return DSAX_ERR_CUDA;
  float *s = noalloc_scratch(dev);
  if (!s) return DSAX_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  FlagArgs a{};
  a.x = x; a.oldspec = oldspec; a.chanmask = chanmask; a.tsmask = tsmask;
  a.nbeam = B; a.ntime = T; a.nchan = C;
  a.guard = p->guard; a.filt = p->filt; a.tbin = p->tbin; a.fbin = p->fbin;
  a.ts_base = p->ts_base; a.tsflag = p->tsflag; a.parity = p->parity;
  a.thresh = p->thresh; a.var_add = p->var_add; a.ts_thresh = p->ts_thresh;
  a.nperm = p->nperm;
  for (int i = 0; i < p->nperm; ++i) a.perm[i] = p->perm[i];
  a.spec = s; a.var = s + nbc; a.maxs = s + 2 * nbc; a.pp = s + 3 * nbc; a.ts = s + 4 * nbc;
  a.counts = reinterpret_cast<int *>(s + 4 * nbc + nbt);
  // the counters accumulate with atomics: clear them (the array keeps the
  // previous call's values)
  if (cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), st) != cudaSuccess) return DSAX_ERR_CUDA;
  if (launch_flag(a, st) != 0) return DSAX_ERR_CUDA;
  if (counts && cudaMemcpyAsync(counts, a.counts, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st) !=
                    cudaSuccess)
    return DSAX_ERR_CUDA;
  return DSAX_OK;
}

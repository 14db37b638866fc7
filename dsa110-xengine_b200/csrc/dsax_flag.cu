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

// ---------------------------------------------------------------- stats, staged
// Same statistics as flag_stats_kernel for the common shapes (nchan a
// multiple of 4, one TBIN-sample bin <= 32 KB): one CTA per beam streams the
// beam's bins through a 3-stage cp.async ring in shared memory (each bin is
// one contiguous TB x C x 4-byte run of the [T][C] filterbank), so the HBM
// reads stay in flight while the previous bin is reduced.  Thread (p, c4)
// owns channels 4c4..4c4+3 and rows p, p+P, ... of every bin; per-row sums
// (the time series) and per-bin sums are finished in shared memory in a
// fixed order, so results do not depend on scheduling.
namespace flag {
constexpr int kFastThreads = 256;
constexpr int kFastStages = 3;
constexpr int kFastStageMax = 32768;
}  // namespace flag

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(flag::kFastThreads, 2) flag_stats_staged_kernel(FlagArgs a) {
  constexpr int S = flag::kFastStages;
  const int b = blockIdx.x, tid = threadIdx.x;
  const int T = a.ntime, C = a.nchan, TB = a.tbin;
  const int C4 = C >> 2, P = flag::kFastThreads / C4;
  const int p = tid / C4, c4 = tid - p * C4;
  const bool active = p < P;
  const int nbins = T / TB;
  const int stage_f4 = TB * C4;                     // float4 per bin
  const int stage_bytes = (stage_f4 * 16 + 127) & ~127;
  const float4 *xb = reinterpret_cast<const float4 *>(a.x + (int64_t)b * T * C);

  extern __shared__ __align__(16) uint8_t fs_raw[];
  const uint32_t sbase = smem_u32(fs_raw);
  double *sm_rs = reinterpret_cast<double *>(fs_raw + S * stage_bytes);   // [TB][C4]
  double *sm_bp = sm_rs + TB * C4;                                         // [P][C]

  auto issue = [&](int bin) {
    if (bin < nbins) {
      const float4 *src = xb + (int64_t)bin * stage_f4;
      const uint32_t dst = sbase + (uint32_t)(bin % S) * stage_bytes;
      for (int i = tid; i < stage_f4; i += flag::kFastThreads) cp_async16(dst + 16u * i, src + i);
    }
    cp_async_commit();
  };

  double s[4], q[4];
  float m[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) { s[j] = 0.0; q[j] = 0.0; m[j] = -INFINITY; }
  double bmax = -1e300, bmin = 1e300;   // owned by thread tid < C (channel tid)

#pragma unroll
  for (int i = 0; i < S - 1; ++i) issue(i);
  for (int bin = 0; bin < nbins; ++bin) {
    issue(bin + S - 1);
    cp_async_wait<S - 1>();
    __syncthreads();
    if (active) {
      const float4 *st = reinterpret_cast<const float4 *>(fs_raw + (bin % S) * stage_bytes);
      double bs[4] = {0.0, 0.0, 0.0, 0.0};
      for (int t = p; t < TB; t += P) {
        const float4 v4 = st[t * C4 + c4];
        const float v[4] = {v4.x, v4.y, v4.z, v4.w};
        double r = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bs[j] += v[j];
          q[j] += (double)v[j] * v[j];
          m[j] = fmaxf(m[j], v[j]);
          r += v[j];
        }
        sm_rs[t * C4 + c4] = r;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        s[j] += bs[j];
        sm_bp[p * C + 4 * c4 + j] = bs[j];
      }
    }
    if (a.pix_sum) {   // downsampled spectrogram: tbin / tds whole pixel rows per bin
      const float *sf = reinterpret_cast<const float *>(fs_raw + (bin % S) * stage_bytes);
      const int npr = TB / a.tds, H = T / a.tds;
      for (int i = tid; i < npr * C; i += flag::kFastThreads) {
        const int pr = i / C, c = i - pr * C;
        float sum = 0.f, mx = -INFINITY;
        for (int r = 0; r < a.tds; ++r) {
          const float v = sf[(pr * a.tds + r) * C + c];
          sum += v;
          mx = fmaxf(mx, v);
        }
        const int64_t o = ((int64_t)b * H + bin * npr + pr) * C + c;
        a.pix_sum[o] = sum;
        a.pix_max[o] = mx;
      }
    }
    __syncthreads();
    if (tid < TB) {
      double r = 0.0;
      for (int k = 0; k < C4; ++k) r += sm_rs[tid * C4 + k];
      a.ts[(int64_t)b * T + (int64_t)bin * TB + tid] = (float)(r / C);
    }
    if (tid < C) {
      double bsum = 0.0;
      for (int k = 0; k < P; ++k) bsum += sm_bp[k * C + tid];
      const double mb = bsum / TB;
      bmax = fmax(bmax, mb);
      bmin = fmin(bmin, mb);
    }
  }
  cp_async_wait<0>();
  // rows beyond the last whole bin (T % TB): sums, squares, max and the
  // time series, read directly
  for (int t0 = nbins * TB; t0 < T; t0 += TB) {
    __syncthreads();
    const int rows = min(TB, T - t0);
    if (active) {
      for (int t = p; t < rows; t += P) {
        const float4 v4 = __ldg(xb + (int64_t)(t0 + t) * C4 + c4);
        const float v[4] = {v4.x, v4.y, v4.z, v4.w};
        double r = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          s[j] += v[j];
          q[j] += (double)v[j] * v[j];
          m[j] = fmaxf(m[j], v[j]);
          r += v[j];
        }
        sm_rs[t * C4 + c4] = r;
      }
    }
    __syncthreads();
    if (tid < rows) {
      double r = 0.0;
      for (int k = 0; k < C4; ++k) r += sm_rs[tid * C4 + k];
      a.ts[(int64_t)b * T + t0 + tid] = (float)(r / C);
    }
  }
  // per-channel totals over the P row phases, in phase order
  double tot[3] = {0.0, 0.0, -INFINITY};
#pragma unroll
  for (int pass = 0; pass < 3; ++pass) {
    __syncthreads();
    if (active) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        sm_bp[p * C + 4 * c4 + j] = pass == 0 ? s[j] : pass == 1 ? q[j] : (double)m[j];
    }
    __syncthreads();
    if (tid < C) {
      for (int k = 0; k < P; ++k) {
        const double v = sm_bp[k * C + tid];
        tot[pass] = pass < 2 ? tot[pass] + v : fmax(tot[pass], v);
      }
    }
  }
  if (tid < C) {
    const double mean = tot[0] / T;
    const double var = fmax(tot[1] / T - mean * mean, 0.0);
    const int o = b * C + tid;
    a.spec[o] = (float)mean;
    a.var[o] = (float)var;
    a.maxs[o] = a.parity ? (float)mean : (float)tot[2];
    a.pp[o] = nbins > 0 ? (float)(bmax - bmin) : 0.0f;
  }
}

bool flag_stats_staged_ok(const FlagArgs &a) {
  const bool pix_ok = !a.pix_sum || (a.tds > 0 && a.tbin % a.tds == 0 && a.ntime % a.tbin == 0);
  return a.nchan % 4 == 0 && (reinterpret_cast<uintptr_t>(a.x) & 15u) == 0 &&
         (int64_t)a.tbin * a.nchan * 4 <= flag::kFastStageMax && a.tbin <= flag::kFastThreads &&
         pix_ok;
}

static size_t staged_stats_smem(const FlagArgs &a) {
  const int C4 = a.nchan / 4, P = flag::kFastThreads / C4;
  const size_t stage = ((size_t)a.tbin * a.nchan * 4 + 127) & ~(size_t)127;
  return flag::kFastStages * stage + sizeof(double) * ((size_t)a.tbin * C4 + (size_t)P * a.nchan);
}

// ---------------------------------------------------------------- decisions
// Lower median sorted[(n+1)/2 - 1] of v[0..n) in shared memory, by rank
// counting with ties broken by index (the element a stable sort would put
// at that position has the same value).  All threads of the block call it.
__device__ float block_lower_median(const float *v, int n, float *result_slot) {
  const int k = (n + 1) / 2 - 1;
  // gs threads (a power of two <= 32) share one element's count
  int gs = 1;
  while (gs < 32 && gs * 2 * n <= (int)blockDim.x) gs *= 2;
  const int sub = threadIdx.x & (gs - 1);
  const int per = (n + gs - 1) / gs;
  const int rounds = (n * gs + blockDim.x - 1) / blockDim.x;   // uniform trip count
  for (int rd = 0; rd < rounds; ++rd) {
    const int i = (rd * (int)blockDim.x + (int)threadIdx.x) / gs;
    const bool live = i < n;
    const float x = live ? v[i] : 0.0f;
    int r = 0;
    if (live) {
      const int j0 = sub * per, j1 = min(n, j0 + per);
#pragma unroll 8
      for (int j = j0; j < j1; ++j) {
        const float y = v[j];
        r += (y < x) || (y == x && j < i);
      }
    }
    for (int o = gs >> 1; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (live && sub == 0 && r == k) *result_slot = x;
  }
  __syncthreads();
  const float med = *result_slot;
  __syncthreads();
  return med;
}

// corr[j - G] = sb[j] - lower median of sb[w0 .. w0 + F), w0 = j, or
// C - G - F for the last windows (channflag's forward detrend), for j in
// [G, C - G); one thread per (channel, window element) rank count.
__device__ void window_detrend(const float *sb, const FlagArgs &a, float *corr) {
  const int C = a.nchan, G = a.guard, F = a.filt, n = C - 2 * G;
  const int k = (F + 1) / 2 - 1;
  for (int idx = threadIdx.x; idx < n * F; idx += blockDim.x) {
    const int jj = idx / F, i = idx - jj * F;
    const int j = G + jj;
    const int w0 = (C - G - j >= F) ? j : C - G - F;
    const float x = sb[w0 + i];
    int r = 0;
    for (int q = 0; q < F; ++q) {
      const float y = sb[w0 + q];
      r += (y < x) || (y == x && q < i);
    }
    if (r == k) corr[jj] = sb[j] - x;
  }
  __syncthreads();
}

// channflag()'s test statistic as a number: corr[j] / (thr * MAD), so the
// channel is flagged exactly when |z| > 1 (z = +-1e6 when the MAD is 0 and
// corr is not; 0 in the guard band).  Used as a learned-flagger feature.
__device__ void channflag_z(const float *sb, float thr, const FlagArgs &a, float *zout,
                            float *corr, float *tmp, float *slot) {
  const int C = a.nchan, G = a.guard, n = C - 2 * G;
  for (int j = threadIdx.x; j < C; j += blockDim.x) zout[j] = 0.0f;
  window_detrend(sb, a, corr);
  const float med = block_lower_median(corr, n, slot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = fabsf(corr[i] - med);
  __syncthreads();
  const float mad = block_lower_median(tmp, n, slot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float v = corr[i];
    zout[G + i] = mad > 0.0f ? v / (thr * mad) : (v > 0.0f ? 1e6f : (v < 0.0f ? -1e6f : 0.0f));
  }
  __syncthreads();
}

__device__ __forceinline__ float slogf(float v) { return copysignf(log1pf(fabsf(v)), v); }

// Learned-flagger input features of one beam (one CTA per beam) from the
// statistics pass: the plain flagger's four channel test statistics and its
// time-series statistic z, each scaled so that the plain rule fires at
// |z| = 1 (z > 1 for the one-sided pp and time-series rules), given as
// margins 10 (|z| - 1), plus the downsampled spectrogram.  F[b][h][c][8],
// log-compressed by slog(v) = sign(v) log(1 + |v|):
//   f0 (pixel mean - mu) / sigma * sqrt(tds)   f1 (pixel max - mu) / sigma
//   f2 10 (max over the pixel's samples of z_ts - 1)
//   f3 10 (|z_spec| - 1)   f4 10 (|z_var| - 1)   f5 10 (|z_max| - 1)
//   f6 10 (z_pp - 1)       f7 mean over the pixel's samples of z_ts
// mu, sigma: mean and standard deviation of the beam's samples (from the
// per-channel mean and variance).
__global__ void __launch_bounds__(2 * flag::kDecThreads) lf_stat_features_kernel(FlagArgs a, float *F,
                                                                            uint16_t *Fbf) {
  const int b = blockIdx.x;
  const int C = a.nchan, G = a.guard, T = a.ntime, n = C - 2 * G, tds = a.tds, H = T / tds;
  extern __shared__ float lsh[];
  float *spec = lsh;                                   // C
  float *corr = spec + C;                              // C
  float *tmp = corr + C;                               // max(C, ts_base)
  float *z = tmp + (a.ts_base > C ? a.ts_base : C);    // [4][C]
  float *zt = z + 4 * C;                               // T
  float *rmax = zt + T;                                // H
  float *rmean = rmax + H;                             // H
  __shared__ float slot;
  __shared__ float mu_sd[2];

  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.spec[b * C + c];
  __syncthreads();
  channflag_z(spec, a.thresh, a, z, corr, tmp, &slot);
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.var[b * C + c];
  __syncthreads();
  channflag_z(spec, a.thresh + a.var_add, a, z + C, corr, tmp, &slot);
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.maxs[b * C + c];
  __syncthreads();
  channflag_z(spec, a.thresh, a, z + 2 * C, corr, tmp, &slot);
  // simple_channflag(pp): one-sided, FBIN-channel mean against med + Thr/sqrt(FBIN) MAD
  for (int c = threadIdx.x; c < C; c += blockDim.x) spec[c] = a.pp[b * C + c];
  for (int i = threadIdx.x; i < n; i += blockDim.x) corr[i] = a.pp[b * C + G + i];
  __syncthreads();
  {
    const float med = block_lower_median(corr, n, &slot);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = fabsf(corr[i] - med);
    __syncthreads();
    const float mad = block_lower_median(tmp, n, &slot);
    const float mythr = a.thresh / sqrtf((float)a.fbin);
    for (int j = threadIdx.x; j < C; j += blockDim.x) {
      float zz = 0.0f;
      if (j >= G && j < C - G - a.fbin) {
        float vv = 0.0f;
        for (int k = 0; k < a.fbin; ++k) vv += a.parity ? spec[j] : spec[j + k];
        vv = vv / (float)a.fbin - med;
        zz = mad > 0.0f ? vv / (mythr * mad) : (vv > 0.0f ? 1e6f : (vv < 0.0f ? -1e6f : 0.0f));
      }
      z[3 * C + j] = zz;
    }
  }
  __syncthreads();
  // simple_tsflag: median and MAD over the first ts_base samples
  const float *tsb = a.ts + (int64_t)b * T;
  for (int i = threadIdx.x; i < a.ts_base; i += blockDim.x) tmp[i] = tsb[i];
  __syncthreads();
  {
    const float med = block_lower_median(tmp, a.ts_base, &slot);
    for (int i = threadIdx.x; i < a.ts_base; i += blockDim.x) tmp[i] = fabsf(tsb[i] - med);
    __syncthreads();
    const float mad = block_lower_median(tmp, a.ts_base, &slot);
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      const float vv = tsb[t] - med;
      float zz = mad > 0.0f ? vv / (a.ts_thresh * mad) : (vv > 0.0f ? 1e6f : (vv < 0.0f ? -1e6f : 0.0f));
      zt[t] = a.tsflag ? zz : 0.0f;
    }
  }
  if (threadIdx.x < 32) {   // beam mean and variance over channels, one warp
    double s = 0.0, q = 0.0;
    for (int c = threadIdx.x; c < C; c += 32) {
      const double m = a.spec[b * C + c];
      s += m;
      q += (double)a.var[b * C + c] + m * m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      q += __shfl_xor_sync(0xffffffffu, q, o);
    }
    if (threadIdx.x == 0) {
      const double mu = s / C;
      mu_sd[0] = (float)mu;
      mu_sd[1] = (float)sqrt(fmax(q / C - mu * mu, 1e-30));
    }
  }
  __syncthreads();
  for (int h = threadIdx.x; h < H; h += blockDim.x) {
    float mx = -INFINITY, sm = 0.0f;
    for (int r = 0; r < tds; ++r) {
      const float v = zt[h * tds + r];
      mx = fmaxf(mx, v);
      sm += v;
    }
    rmax[h] = mx;
    rmean[h] = sm / tds;
  }
  __syncthreads();
  const float mu = mu_sd[0], inv = 1.0f / mu_sd[1], kpix = sqrtf((float)tds);
  constexpr float kMargin = 10.0f;   // margins scaled so the rule's edge is steep
  // features that depend only on the channel (f3..f6) or only on the row
  // (f2, f7): once each, in place
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    z[c] = slogf(kMargin * (fabsf(z[c]) - 1.0f));
    z[C + c] = slogf(kMargin * (fabsf(z[C + c]) - 1.0f));
    z[2 * C + c] = slogf(kMargin * (fabsf(z[2 * C + c]) - 1.0f));
    z[3 * C + c] = slogf(kMargin * (z[3 * C + c] - 1.0f));
  }
  for (int h = threadIdx.x; h < H; h += blockDim.x) {
    rmax[h] = slogf(kMargin * (rmax[h] - 1.0f));
    rmean[h] = slogf(rmean[h]);
  }
  __syncthreads();
  float4 *Fb = F ? reinterpret_cast<float4 *>(F + (int64_t)b * H * C * 8) : nullptr;
  const float *ps = a.pix_sum + (int64_t)b * H * C;
  const float *pm = a.pix_max + (int64_t)b * H * C;
  const float invC = 1.0f / (float)C, invT = 1.0f / (float)tds;
  constexpr int kBatch = 4;   // pixel loads issued together
  for (int i0 = threadIdx.x; i0 < H * C; i0 += kBatch * blockDim.x) {
    float pv[kBatch], mv[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const int i = i0 + k * blockDim.x;
      pv[k] = i < H * C ? ps[i] : 0.0f;
      mv[k] = i < H * C ? pm[i] : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
    const int i = i0 + k * blockDim.x;
    if (i >= H * C) break;
    int h = __float2int_rz((float)i * invC);   // i / C, corrected (i < 2^24)
    h += (i - h * C >= C) - (i - h * C < 0);
    const int c = i - h * C;
    float4 f, g;
    f.x = slogf((pv[k] * invT - mu) * inv * kpix);
    f.y = slogf((mv[k] - mu) * inv);
    f.z = rmax[h];
    f.w = z[c];
    g.x = z[C + c];
    g.y = z[2 * C + c];
    g.z = z[3 * C + c];
    g.w = rmean[h];
    if (F) {
      Fb[2 * i] = f;
      Fb[2 * i + 1] = g;
    }
    if (Fbf) {
      uint4 o;
      asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(o.x) : "f"(f.y), "f"(f.x));
      asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(o.y) : "f"(f.w), "f"(f.z));
      asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(o.z) : "f"(g.y), "f"(g.x));
      asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(o.w) : "f"(g.w), "f"(g.z));
      // zero-bordered grid [B][H+2][C+2][8] read by the first conv layer
      reinterpret_cast<uint4 *>(Fbf)[((int64_t)b * (H + 2) + h + 1) * (C + 2) + c + 1] = o;
    }
    }
  }
}

int launch_lf_stat_features(const FlagArgs &a, float *F, uint16_t *Fbf, cudaStream_t st) {
  if (!a.pix_sum || a.tds < 1 || a.ntime % a.tds || a.nchan > flag::kMaxChan) return -1;
  const int H = a.ntime / a.tds;
  const size_t sh = sizeof(float) * (2 * a.nchan + (a.ts_base > a.nchan ? a.ts_base : a.nchan) +
                                     4 * a.nchan + a.ntime + 2 * H);
  if (sh > 200 * 1024) return -1;
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, lf_stat_features_kernel, 200 * 1024) != cudaSuccess) return -2;
  lf_stat_features_kernel<<<a.nbeam, 2 * flag::kDecThreads, sh, st>>>(a, F, Fbf);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Group versions of the median and detrend: `gsize` threads (whole warps)
// with group-local index gtid synchronise on named barrier `bid`.
__device__ float grp_lower_median(const float *v, int n, float *result_slot, int gtid, int gsize,
                                  int bid) {
  const int k = (n + 1) / 2 - 1;
  int gs = 1;
  while (gs < 32 && gs * 2 * n <= gsize) gs *= 2;
  const int sub = gtid & (gs - 1);
  const int per = (n + gs - 1) / gs;
  const int rounds = (n * gs + gsize - 1) / gsize;   // uniform trip count
  for (int rd = 0; rd < rounds; ++rd) {
    const int i = (rd * gsize + gtid) / gs;
    const bool live = i < n;
    const float x = live ? v[i] : 0.0f;
    int r = 0;
    if (live) {
      const int j0 = sub * per, j1 = min(n, j0 + per);
#pragma unroll 8
      for (int j = j0; j < j1; ++j) {
        const float y = v[j];
        r += (y < x) || (y == x && j < i);
      }
    }
    for (int o = gs >> 1; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (live && sub == 0 && r == k) *result_slot = x;
  }
  named_bar(bid, gsize);
  const float med = *result_slot;
  named_bar(bid, gsize);
  return med;
}

// The k-th smallest of v[0..n) (0-based; the value rank counting with
// ties by index returns) by a four-pass MSB-first radix select over
// order-preserving 32-bit keys: per pass a 256-bin shared histogram of the
// candidates that still match the selected prefix, then one warp finds the
// bin holding rank k.  O(n) work instead of O(n^2); finite inputs.
__device__ __forceinline__ uint32_t ordered_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ float grp_radix_select(const float *v, int n, int k, uint32_t *hist, uint32_t *sel,
                                  int gtid, int gsize, int bid) {
  uint32_t prefix = 0u, pmask = 0u;
  int kk = k;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = gtid; i < 256; i += gsize) hist[i] = 0u;
    named_bar(bid, gsize);
    for (int i = gtid; i < n; i += gsize) {
      const uint32_t u = ordered_key(v[i]);
      if ((u & pmask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1u);
    }
    named_bar(bid, gsize);
    if (gtid < 32) {   // the first warp: bin holding rank kk
      uint32_t c[8], tot = 0u;
#pragma unroll
      for (int e = 0; e < 8; ++e) { c[e] = hist[8 * gtid + e]; tot += c[e]; }
      uint32_t incl = tot;   // inclusive scan over lanes
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (gtid >= o) incl += y;
      }
      const uint32_t excl = incl - tot;
      if (excl <= (uint32_t)kk && (uint32_t)kk < incl) {
        uint32_t run = excl;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          if ((uint32_t)kk < run + c[e]) {
            sel[0] = (uint32_t)(8 * gtid + e);
            sel[1] = (uint32_t)kk - run;
            break;
          }
          run += c[e];
        }
      }
    }
    named_bar(bid, gsize);
    prefix |= sel[0] << shift;
    pmask |= 0xFFu << shift;
    kk = (int)sel[1];
    named_bar(bid, gsize);
  }
  const uint32_t u = (prefix & 0x80000000u) ? (prefix & 0x7FFFFFFFu) : ~prefix;
  return __uint_as_float(u);
}

__device__ void grp_channflag(const float *sb, float thr, const FlagArgs &a, uint8_t *mask,
                              float *corr, float *tmp, float *slot, int gtid, int gsize, int bid) {
  const int C = a.nchan, G = a.guard, F = a.filt, n = C - 2 * G;
  const int kf = (F + 1) / 2 - 1;
  for (int idx = gtid; idx < n * F; idx += gsize) {   // forward median detrend
    const int jj = idx / F, i = idx - jj * F;
    const int j = G + jj;
    const int w0 = (C - G - j >= F) ? j : C - G - F;
    const float x = sb[w0 + i];
    int r = 0;
    for (int q = 0; q < F; ++q) {
      const float y = sb[w0 + q];
      r += (y < x) || (y == x && q < i);
    }
    if (r == kf) corr[jj] = sb[j] - x;
  }
  named_bar(bid, gsize);
  const float med = grp_lower_median(corr, n, slot, gtid, gsize, bid);
  for (int i = gtid; i < n; i += gsize) tmp[i] = fabsf(corr[i] - med);
  named_bar(bid, gsize);
  const float mad = grp_lower_median(tmp, n, slot, gtid, gsize, bid);
  for (int i = gtid; i < n; i += gsize) {
    const float v = corr[i];
    if (v > thr * mad || v < -thr * mad) mask[G + i] = 1;
  }
}

// The decisions of one beam (one CTA): the four channel tests and the
// time-series test are independent, so five thread groups run them at once
// (the reference runs them in sequence, src/gpu_flagger.cu:1340-1398; the
// flags are the same):
//   group 0-2 (64 threads each): channflag(spec - oldspec, Thr),
//             channflag(var, Thr + 0.5), channflag(max, Thr)
//   group 3   (64 threads): simple_channflag(pp, Thr / sqrt(FBIN)), one-sided
//   group 4   (128 threads): simple_tsflag(ts, TsThr) over the first ts_base
// The channel groups OR their flags into one shared mask.
namespace flag {
constexpr int kDecideThreads = 384;
}

__global__ void __launch_bounds__(flag::kDecideThreads) flag_decide_kernel(FlagArgs a) {
  const int b = blockIdx.x, tid = threadIdx.x, warp = tid >> 5;
  const int C = a.nchan, G = a.guard, T = a.ntime, n = C - 2 * G;
  extern __shared__ float dsh[];          // [4 groups][3][C], then ts: [2][ts_base]
  __shared__ uint8_t cmask[flag::kMaxChan];
  __shared__ float slots[5];
  __shared__ uint32_t ts_hist[256], ts_sel[2];   // radix select of the time-series group

  for (int c = tid; c < C; c += blockDim.x) cmask[c] = 0;
  __syncthreads();
  const int g = warp < 8 ? warp >> 1 : 4;
  const int gsize = g < 4 ? 64 : 128, gtid = g < 4 ? tid - 64 * g : tid - 256, bid = 1 + g;
  if (g < 4) {
    float *sb = dsh + g * 3 * C, *corr = sb + C, *tmp = corr + C;
    const float *src = g == 0 ? a.spec : g == 1 ? a.var : g == 2 ? a.maxs : a.pp;
    for (int c = gtid; c < C; c += gsize)
      sb[c] = src[b * C + c] - ((g == 0 && a.oldspec) ? a.oldspec[b * C + c] : 0.0f);
    named_bar(bid, gsize);
    if (g < 3) {
      const float thr = g == 1 ? a.thresh + a.var_add : a.thresh;
      grp_channflag(sb, thr, a, cmask, corr, tmp, &slots[g], gtid, gsize, bid);
    } else {
      for (int i = gtid; i < n; i += gsize) corr[i] = sb[G + i];
      named_bar(bid, gsize);
      const float med = grp_lower_median(corr, n, &slots[g], gtid, gsize, bid);
      for (int i = gtid; i < n; i += gsize) tmp[i] = fabsf(corr[i] - med);
      named_bar(bid, gsize);
      const float mad = grp_lower_median(tmp, n, &slots[g], gtid, gsize, bid);
      const float mythr = a.thresh / sqrtf((float)a.fbin);
      for (int j = G + gtid; j < C - G - a.fbin; j += gsize) {
        float vv = 0.0f;
        for (int k = 0; k < a.fbin; ++k) vv += a.parity ? sb[j] : sb[j + k];
        vv = vv / (float)a.fbin - med;
        if (vv > mythr * mad) cmask[j] = 1;
      }
    }
  } else {
    const float *tb = a.ts + (int64_t)b * T;
    if (a.tsflag) {
      float *tsb = dsh + 12 * C, *tmp = tsb + a.ts_base;
      for (int i = gtid; i < a.ts_base; i += gsize) tsb[i] = tb[i];
      named_bar(bid, gsize);
      const int kmed = (a.ts_base + 1) / 2 - 1;   // lower median
      const float med = grp_radix_select(tsb, a.ts_base, kmed, ts_hist, ts_sel, gtid, gsize, bid);
      for (int i = gtid; i < a.ts_base; i += gsize) tmp[i] = fabsf(tsb[i] - med);
      named_bar(bid, gsize);
      const float mad = grp_radix_select(tmp, a.ts_base, kmed, ts_hist, ts_sel, gtid, gsize, bid);
      const float lim = a.ts_thresh * mad;
      int nts = 0;
      uint8_t *mb = a.tsmask + (int64_t)b * T;
      if ((T & 3) == 0 && (reinterpret_cast<uintptr_t>(tb) & 15u) == 0 &&
          (reinterpret_cast<uintptr_t>(mb) & 3u) == 0) {
        // four samples per load and one 32-bit mask word per store; all of a
        // thread's loads (read-only path) are issued before its stores, which
        // as byte stores could otherwise alias them
        const float4 *t4 = reinterpret_cast<const float4 *>(tb);
        uint32_t *m4 = reinterpret_cast<uint32_t *>(mb);
        constexpr int kU = 8;
        for (int i0 = gtid; i0 < T / 4; i0 += kU * gsize) {
          float4 v[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int i = i0 + u * gsize;
            v[u] = i < T / 4 ? __ldg(t4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int i = i0 + u * gsize;
            if (i >= T / 4) break;
            const uint32_t f0 = (v[u].x - med) > lim, f1 = (v[u].y - med) > lim;
            const uint32_t f2 = (v[u].z - med) > lim, f3 = (v[u].w - med) > lim;
            m4[i] = f0 | (f1 << 8) | (f2 << 16) | (f3 << 24);
            nts += (int)(f0 + f1 + f2 + f3);
          }
        }
      } else {
        for (int t = gtid; t < T; t += gsize) {
          const uint8_t f = (__ldg(tb + t) - med) > lim ? 1 : 0;
          mb[t] = f;
          nts += f;
        }
      }
      if (nts) atomicAdd(a.counts + 1, nts);
    } else {
      for (int t = gtid; t < T; t += gsize) a.tsmask[(int64_t)b * T + t] = 0;
    }
  }
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < a.nperm; ++k) {
      const int j = a.perm[k];
      if (j >= G && j < C - G) cmask[j] = 1;
    }
  __syncthreads();
  int nflag = 0;
  for (int c = tid; c < C; c += blockDim.x) {
    a.chanmask[b * C + c] = cmask[c];
    nflag += cmask[c];
  }
  if (nflag) atomicAdd(a.counts, nflag);
}

int launch_flag_stats(const FlagArgs &a, cudaStream_t st) {
  if (a.nchan > flag::kMaxChan) return -1;
  if (flag_stats_staged_ok(a)) {
    static SmemAttrOnce attr2;
    const int mx = flag::kFastStages * flag::kFastStageMax + 48 * 1024;
    if (smem_attr_once(attr2, flag_stats_staged_kernel, mx) != cudaSuccess) return -2;
    flag_stats_staged_kernel<<<a.nbeam, flag::kFastThreads, staged_stats_smem(a), st>>>(a);
  } else {
    if (a.pix_sum) return -1;
    static SmemAttrOnce attr;
    const size_t ssh = 16 * flag::kMaxChan * (4 * sizeof(double) + sizeof(float));
    if (smem_attr_once(attr, flag_stats_kernel, (int)ssh) != cudaSuccess) return -2;
    flag_stats_kernel<<<a.nbeam, flag::kStatThreads, ssh, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_flag(const FlagArgs &a, cudaStream_t st) {
  if (a.nchan > flag::kMaxChan || a.ts_base > 4096) return -1;
  const int rc = launch_flag_stats(a, st);
  if (rc != 0) return rc;
  const size_t sh = sizeof(float) * (12 * (size_t)a.nchan + 2 * (size_t)a.ts_base);
  flag_decide_kernel<<<a.nbeam, flag::kDecideThreads, sh, st>>>(a);
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
// device address of the array per device, looked up once; atomic because
// host threads may make their first call on a device concurrently (they
// store the same value)
std::atomic<float *> g_scratch_addr[kMaxDevices] = {};
}  // namespace

// Resolves the array's device address on the current device `dev` (once per
// device).  Returns nullptr on failure.
static float *noalloc_scratch(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  float *s = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!s) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_flag_scratch) != cudaSuccess) return nullptr;
    s = static_cast<float *>(p);
    g_scratch_addr[dev].store(s, std::memory_order_release);
  }
  return s;
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

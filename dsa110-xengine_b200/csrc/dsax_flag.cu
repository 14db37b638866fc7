// dsax_flag.cu -- the plain RFI flagger on the GPU, statistics and data path.
//
// Replaces src/gpu_flagger.cu, per block in the order of its main loop
// (:1290-1410):
//   scaley (:382-394, once a baseline exists)        -> fused into the
//   calc_spectrum / calc_varspec / calc_maxspec /       statistics pass
//   calc_ppspec (:175-376; the reference calls           (one HBM read)
//   calc_spectrum in calc_maxspec's place at :1334 -- parity mode keeps that)
//   total-power modulation check (:1313-1330)        -> the statistics CTAs
//   channflag x3, simple_channflag (:1340-1347)         (the last one of a
//                                                       beam / of the grid)
//   calc_bpwr (:759-769), gather_mask,               -> flag_apply_kernel
//   flag (:459-474), then make_ts (:414-453),           (reads only the
//   simple_tsflag (:612-653), flagts (:479-494)         flagged chunks; the
//                                                       beam's last CTA does
//                                                       the series tests)
// and fix_zspec (:114-170) + median_calc (:771-798) for the scaley
// baseline.  The shapes the reference hard-codes ([64][16384][1024] uint8,
// ZeroChannels 128, nFiltSize 21, TBIN 128, FBIN 8, T/16) are parameters;
// the filterbank may be uint8 (the reference's type) or FP32.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <cuda.h>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_ptx.cuh"
#include "dsax_scaley.h"
#include "dsax_tmap.h"
#include "../../include/dsax.h"

namespace dsax {

namespace flag {
constexpr int kStatThreads = 256;
constexpr int kStages = 3;
constexpr int kStageTarget = 24576;   // bytes per pipeline stage (upper bound)
constexpr int kMaxChan = 1024;
constexpr int kApplyThreads = 256;    // apply / time-series CTA
constexpr int kApplyRows = 256;       // rows per apply CTA
constexpr int kMaxTsBase = 4096;
constexpr int kLfMaxChan = 128;       // learned-flagger features: channels per beam
constexpr int kDecThreads = 256;
}  // namespace flag

// ---------------------------------------------------------------- elements
// Four consecutive channels of one row: FP32 (16 bytes) or uint8 (4 bytes).
template <typename E>
__device__ __forceinline__ void ld4(const void *p, float (&v)[4]) {
  if constexpr (std::is_same<E, float>::value) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const uint32_t w = *reinterpret_cast<const uint32_t *>(p);
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = (float)((w >> (8 * j)) & 255u);
  }
}
template <typename E>
__device__ __forceinline__ void st4(void *p, const float (&v)[4]) {
  if constexpr (std::is_same<E, float>::value) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {   // values are already integers in [0, 255]
    *reinterpret_cast<uint32_t *>(p) = (uint32_t)v[0] | ((uint32_t)v[1] << 8) |
                                       ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
  }
}
template <typename E>
__device__ __forceinline__ const E *elem_in(const FlagArgs &a) {
  if constexpr (std::is_same<E, float>::value) return a.x; else return a.xu8;
}
template <typename E>
__device__ __forceinline__ E *elem_out(const FlagArgs &a) {
  if constexpr (std::is_same<E, float>::value) return a.xw; else return a.xw8;
}

// scaley (src/gpu_flagger.cu:382-394): (x - spec0) * (SIG / sqrtf(var0)) + MN,
// with the reference's mixed float / double evaluation; uint8 data are
// requantised as (unsigned char)(__float2uint_rn(2 val) / 2), which wraps
// modulo 256 above 255.
template <typename E>
__device__ __forceinline__ float scaley1(float x, float s0, double k, float mn) {
  const float val = (float)((double)(x - s0) * k + (double)mn);
  if constexpr (std::is_same<E, float>::value) {
    return val;
  } else {
    return (float)((__float2uint_rn(2.0f * val) / 2u) & 255u);
  }
}

// The replacement level MN * bpwr as the element type: uint8 is the C
// conversion of `data[idx] = MN * bpwr[bm]` (:473): truncation toward zero,
// clamped to [0, 255] by the device conversion.
template <typename E>
__device__ __forceinline__ E repl_elem(float r) {
  if constexpr (std::is_same<E, float>::value) {
    return r;
  } else {
    return (uint8_t)__float2uint_rz(fminf(r, 255.0f));
  }
}

// The channel decisions of beam b (defined with the order statistics below)
// and the block's total power; both run at the end of the statistics pass.
__device__ void flag_decide_beam(const FlagArgs &a, int b, uint8_t *smem);
__device__ void flag_total_power(const FlagArgs &a);

// ---------------------------------------------------------------- statistics
// One CTA per (channel slab of up to kFlagSlab channels, beam).  The slab's
// rows stream through a three-stage ring of `rs` rows each (rs divides
// TBIN), one 2-D TMA box [rs rows][min(nchan, 128) channels] per stage
// (channels past nchan read zero), completing on the stage's mbarrier; the
// waits are bounded (a.wait_limit_ns, recorded in a.err).  Every thread
// fences its generic reads of a stage before the barrier after which the
// stage is loaded again.  Thread (p, g) owns channels 4g..4g+3 of the slab and rows
// p, p + P, ... of every stage (the lanes of a warp cover consecutive
// 16-byte pieces of a row: conflict-free shared reads, coalesced global
// writes); sums are FP64 for FP32 data and 32-bit integers for uint8 (at
// most 32768 rows per thread, so 255^2 products stay below 2^31; the
// launcher checks it), finished in shared memory in a fixed order (four
// interleaved partial sums per reduction), so results do not depend on
// scheduling.  With a scaley
// baseline the stage is normalised in shared memory first and written back
// (the statistics then describe the normalised block, as in the reference).
// Per row the slab's raw sum goes to rowsum (or to ts when there is one
// slab); flag_apply_kernel turns it into the channel-mean series after the
// flagged columns are replaced.
template <typename E>
__global__ void __launch_bounds__(flag::kStatThreads, 2)
    flag_stats_kernel(const __grid_constant__ CUtensorMap tmap, FlagArgs a) {
  constexpr int S = flag::kStages;
  constexpr int ES = (int)sizeof(E);
  const int slab = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
  const int T = a.ntime, C = a.nchan, TB = a.tbin, RS = a.rs;
  const int c0 = slab * kFlagSlab;
  const int cs = min(kFlagSlab, C - c0);
  const int G4 = cs >> 2, P = flag::kStatThreads / G4;
  const int p = tid / G4, g = tid - p * G4;
  const bool active = p < P;
  const int nbins = T / TB, spb = TB / RS, nst = nbins * spb;
  const int bx = C < kFlagSlab ? C : kFlagSlab;   // channels of a TMA box row
  const int rb = bx * ES;                        // bytes of one staged row (multiple of 16)
  const int stage_bytes = (RS * rb + 127) & ~127;
  const int64_t rstride = (int64_t)C * ES;
  const uint8_t *xb =
      reinterpret_cast<const uint8_t *>(elem_in<E>(a) + (int64_t)b * T * C + c0);
  E *xw = elem_out<E>(a);
  const bool scale = a.spec0 != nullptr;

  constexpr bool kU8 = std::is_same<E, uint8_t>::value;
  // row partials: exact ints for uint8, doubles for FP32
  using RsT = typename std::conditional<kU8, int, double>::type;
  extern __shared__ __align__(128) uint8_t fs_raw[];
  __shared__ __align__(8) uint64_t sfull[S];
  __shared__ volatile int sabort;
  if (tid == 0) {
    for (int s2 = 0; s2 < S; ++s2) mbar_init(&sfull[s2], 1);
    sabort = 0;
    mbar_fence_init();
  }
  const uint32_t sbase = smem_u32(fs_raw);
  const int GS = G4 | 1;   // odd row stride: the row sums read column-wise conflict-free
  RsT *sm_rs = reinterpret_cast<RsT *>(fs_raw + S * stage_bytes);         // [RS][GS]
  double *sm_bp = reinterpret_cast<double *>(
      fs_raw + S * stage_bytes + ((sizeof(RsT) * RS * GS + 15) & ~(size_t)15));   // [P][cs]
  double *sm_k = sm_bp + P * cs;                                           // [cs]
  float *sm_s0 = reinterpret_cast<float *>(sm_k + cs);                     // [cs]
  float *sm_k2 = sm_s0 + cs;                                               // [cs] float(2k)
  uint8_t *sm_lut = reinterpret_cast<uint8_t *>(sm_k2 + cs);               // uint8: [256][cs]
  const double inv_tb = 1.0 / TB;

  if (scale) {
    for (int c = tid; c < cs; c += flag::kStatThreads) {
      sm_s0[c] = a.spec0[b * C + c0 + c];
      sm_k[c] = (double)a.sig / (double)sqrtf(a.var0[b * C + c0 + c]);
      sm_k2[c] = (float)(2.0 * sm_k[c]);
    }
    if constexpr (kU8) {
      // uint8 has 256 inputs per channel: scaley as a table [x][channel],
      // read by the lanes of a warp (consecutive channel groups) from
      // distinct banks
      __syncthreads();
      for (int i = tid; i < 256 * cs; i += flag::kStatThreads) {
        const int x = i / cs, c = i - x * cs;
        sm_lut[i] = (uint8_t)scaley_u8((float)x, sm_s0[c], sm_k2[c], sm_k[c], a.mn);
      }
    }
  }
  __syncthreads();
  // sum of n values at v[0], v[stride], ... in four interleaved chains
  auto sum4 = [](const auto *v, int n, int stride) -> double {
    using V = typename std::remove_cv<typename std::remove_pointer<decltype(v)>::type>::type;
    V a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    int k = 0;
    for (; k + 4 <= n; k += 4) {
      a0 += v[k * stride];
      a1 += v[(k + 1) * stride];
      a2 += v[(k + 2) * stride];
      a3 += v[(k + 3) * stride];
    }
    for (; k < n; ++k) a0 += v[k * stride];
    return (double)((a0 + a1) + (a2 + a3));
  };

  // stage st: one TMA box, issued by thread 0
  const uint32_t box_bytes = (uint32_t)(RS * rb);
  int issued = 0;
  auto issue = [&](int st) {
    if (st < nst) {
      mbar_arrive_expect_tx(&sfull[st % S], box_bytes);
      tma_load_2d(sbase + (uint32_t)(st % S) * stage_bytes, &tmap, c0, b * T + st * RS,
                  &sfull[st % S]);
      issued = st + 1;
    }
  };
  auto put_row = [&](int t, double r) {
    if (a.nslab == 1)
      a.ts[(int64_t)b * T + t] = a.ts_mean ? (float)(r / C) : (float)r;
    else
      a.rowsum[((int64_t)b * a.nslab + slab) * T + t] = (float)r;
  };
  // normalise (if scaling) and accumulate the four channels of one row:
  // FP64 for FP32 data, exact 32-bit integers for uint8 (no FP64 work)
  using Acc = typename std::conditional<kU8, int, double>::type;
  using MaxT = typename std::conditional<kU8, int, float>::type;
  Acc s[4], q[4], bs[4];
  MaxT m[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    s[j] = 0; q[j] = 0; bs[j] = 0;
    m[j] = kU8 ? (MaxT)0 : (MaxT)-INFINITY;
  }
  auto take = [&](uint8_t *src, int t, bool bin, bool keep) -> RsT {
    float v[4];
    if constexpr (kU8) {
      uint32_t w = *reinterpret_cast<const uint32_t *>(src);
      if (scale) {
        uint32_t o = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          o |= (uint32_t)sm_lut[((w >> (8 * j)) & 255u) * cs + 4 * g + j] << (8 * j);
        w = o;
        if (xw) *reinterpret_cast<uint32_t *>(xw + ((int64_t)b * T + t) * C + c0 + 4 * g) = w;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int x = (int)((w >> (8 * j)) & 255u);
        if (bin) bs[j] += x; else s[j] += x;
        q[j] += x * x;
        m[j] = max(m[j], x);
      }
      return (int)__dp4a(w, 0x01010101u, 0u);   // the row's four bytes summed
    } else {
      ld4<E>(src, v);
      if (scale) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          v[j] = scaley1<E>(v[j], sm_s0[4 * g + j], sm_k[4 * g + j], a.mn);
        if (xw) st4<E>(xw + ((int64_t)b * T + t) * C + c0 + 4 * g, v);
        if (keep) st4<E>(src, v);   // the pixel sums read the normalised stage
      }
      double r = 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (bin) bs[j] += v[j]; else s[j] += v[j];
        q[j] += (double)v[j] * v[j];
        m[j] = fmaxf(m[j], v[j]);
        r += v[j];
      }
      return r;
    }
  };
  double bmax = -1e300, bmin = 1e300;   // owned by thread tid < cs (channel tid)

  if (tid == 0)
    for (int i = 0; i < S - 1; ++i) issue(i);
  int consumed = 0;
  for (int st = 0; st < nst; ++st) {
    if (tid == 0) issue(st + S - 1);   // its slot was released at the end of stage st - 1
    const bool ok = mbar_wait_bounded(&sfull[st % S], (uint32_t)(st / S) & 1u, &sabort, a.err,
                                      DEV_ERR_WAIT_FULL, a.wait_limit_ns);
    if (__syncthreads_or(!ok)) break;
    consumed = st + 1;
    uint8_t *sp = fs_raw + (st % S) * stage_bytes;
    const int t0 = st * RS;
    if (active) {
      for (int r = p; r < RS; r += P) {
        sm_rs[r * GS + g] = take(sp + r * rb + 4 * g * ES, t0 + r, true, a.pix_sum != nullptr);
      }
    }
    const bool bin_end = (st + 1) % spb == 0;
    if (spb == 1 && active) {   // one stage per bin: its partials go out with the rows
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        sm_bp[p * cs + 4 * g + j] = (double)bs[j];
        s[j] += bs[j];
        bs[j] = 0;
      }
    }
    if (a.pix_sum) {   // downsampled spectrogram: rs / tds whole pixel rows per stage
      __syncthreads();
      const float *sf = reinterpret_cast<const float *>(sp);
      const int npr = RS / a.tds, H = T / a.tds;
      for (int i = tid; i < npr * cs; i += flag::kStatThreads) {
        const int pr = i / cs, c = i - pr * cs;
        float sum = 0.f, mx = -INFINITY;
        for (int r = 0; r < a.tds; ++r) {
          const float v = sf[(pr * a.tds + r) * cs + c];
          sum += v;
          mx = fmaxf(mx, v);
        }
        const int64_t o = ((int64_t)b * H + t0 / a.tds + pr) * C + c0 + c;
        a.pix_sum[o] = sum;
        a.pix_max[o] = mx;
      }
    }
    fence_proxy_async_smem();   // this stage's generic reads before its next TMA write
    __syncthreads();
    if (tid < RS) put_row(t0 + tid, sum4(sm_rs + tid * GS, G4, 1));
    if (bin_end) {   // the last stage of a TBIN bin: bin means per channel
      if (spb > 1) {
        if (active) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            sm_bp[p * cs + 4 * g + j] = (double)bs[j];
            s[j] += bs[j];
            bs[j] = 0;
          }
        }
        __syncthreads();
      }
      if (tid < cs) {
        const double mb = sum4(sm_bp + tid, P, cs) * inv_tb;
        bmax = fmax(bmax, mb);
        bmin = fmin(bmin, mb);
      }
    }
  }
  // boxes still landing after an abort: wait for them before exit
  if (tid == 0) {
    volatile int no_abort = 0;
    for (int k = consumed; k < issued; ++k)
      mbar_wait_bounded(&sfull[k % S], (uint32_t)(k / S) & 1u, &no_abort, a.err, DEV_ERR_WAIT_FULL,
                        drain_limit(a.wait_limit_ns));
  }
  __syncthreads();
  if (sabort) return;   // recorded in a.err; no statistics from this CTA
  // rows beyond the last whole bin (T % TB): sums, squares, max and row
  // sums, read directly
  for (int t0 = nbins * TB; t0 < T; t0 += RS) {
    __syncthreads();
    const int rows = min(RS, T - t0);
    if (active) {
      for (int r = p; r < rows; r += P)
        sm_rs[r * GS + g] = take(const_cast<uint8_t *>(xb) + (int64_t)(t0 + r) * rstride + 4 * g * ES,
                                 t0 + r, false, false);
    }
    __syncthreads();
    if (tid < rows) put_row(t0 + tid, sum4(sm_rs + tid * GS, G4, 1));
  }
  // per-channel totals over the P row phases, in phase order
  double tot[3] = {0.0, 0.0, -INFINITY};
#pragma unroll
  for (int pass = 0; pass < 3; ++pass) {
    __syncthreads();
    if (active) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        sm_bp[p * cs + 4 * g + j] =
            pass == 0 ? (double)s[j] : pass == 1 ? (double)q[j] : (double)m[j];
    }
    __syncthreads();
    if (tid < cs) {
      if (pass < 2) {
        tot[pass] = sum4(sm_bp + tid, P, cs);
      } else {
        for (int k = 0; k < P; ++k) tot[2] = fmax(tot[2], sm_bp[k * cs + tid]);
      }
    }
  }
  if (tid < cs) {
    const double mean = tot[0] / T;
    const double var = fmax(tot[1] / T - mean * mean, 0.0);
    const int o = b * C + c0 + tid;
    a.spec[o] = (float)mean;
    a.var[o] = (float)var;
    a.maxs[o] = a.parity ? (float)mean : (float)tot[2];
    a.pp[o] = nbins > 0 ? (float)(bmax - bmin) : 0.0f;
  }
  if (!a.decide) return;
  // The last slab CTA of the beam makes its channel decisions, and the last
  // CTA of the grid the block-level total power: each CTA publishes its
  // statistics (fence) before counting itself in; nothing waits.
  __shared__ int last_sh;
  __threadfence();
  __syncthreads();
  if (tid == 0) last_sh = a.nslab == 1 ? 1 : (atomicAdd(a.ctr + b, 1) == a.nslab - 1);
  __syncthreads();
  if (last_sh) {
    __threadfence();
    flag_decide_beam(a, b, fs_raw);
  }
  if (!a.modcheck && !a.tpwr_out) return;
  __syncthreads();
  if (tid == 0) last_sh = atomicAdd(a.ctr + 2 * a.nbeam, 1) == (int)(gridDim.x * gridDim.y) - 1;
  __syncthreads();
  if (last_sh) {
    __threadfence();
    flag_total_power(a);
  }
}

// ---------------------------------------------------------------- decisions
// (the order-statistic helpers: radix select below, the rank-count medians
// and the learned-flagger feature kernel)
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

// channflag (src/gpu_flagger.cu:655-720) for one beam in a group of `gsize`
// threads: forward nFiltSize-channel median detrend, then |x| > Thr * MAD
// of the detrended spectrum inside the guard band (compared against 0, as
// the reference does).  Medians are lower medians (medval, :534-556).
__device__ void grp_channflag(const float *sb, float thr, const FlagArgs &a, uint8_t *mask,
                              float *corr, float *tmp, uint32_t *hist, uint32_t *sel, int gtid,
                              int gsize, int bid) {
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
  const int k = (n + 1) / 2 - 1;
  const float med = grp_radix_select(corr, n, k, hist, sel, gtid, gsize, bid);
  for (int i = gtid; i < n; i += gsize) tmp[i] = fabsf(corr[i] - med);
  named_bar(bid, gsize);
  const float mad = grp_radix_select(tmp, n, k, hist, sel, gtid, gsize, bid);
  for (int i = gtid; i < n; i += gsize) {
    const float v = corr[i];
    if (v > thr * mad || v < -thr * mad) mask[G + i] = 1;
  }
}

// The channel decisions of beam b, by the 256 threads of the statistics CTA
// that completed the beam: the four tests concurrently in four groups of 64
// threads -- channflag(spec - oldspec, Thr), channflag(var, Thr + 0.5),
// channflag(max, Thr), simple_channflag(pp, Thr / sqrt(FBIN)) (one-sided
// FBIN-channel mean; parity mode keeps the reference's spec[j] sum, :594) --
// ORed into one mask, plus the permanent flag channels
// (src/gpu_flagger.cu:1340-1347).  smem: 12 nchan floats + nchan bytes.
__device__ void flag_decide_beam(const FlagArgs &a, int b, uint8_t *smem) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int C = a.nchan, G = a.guard, n = C - 2 * G;
  float *dsh = reinterpret_cast<float *>(smem);                 // [4 groups][3][C]
  uint8_t *cmask = reinterpret_cast<uint8_t *>(dsh + 12 * C);   // [C]
  __shared__ uint32_t hist[4][256], sel[4][2];
  for (int c = tid; c < C; c += flag::kStatThreads) cmask[c] = 0;
  __syncthreads();
  const int g = warp >> 1, gsize = 64, gtid = tid - 64 * g, bid = 1 + g;
  float *sb = dsh + g * 3 * C, *corr = sb + C, *tm = corr + C;
  const float *src = g == 0 ? a.spec : g == 1 ? a.var : g == 2 ? a.maxs : a.pp;
  for (int c = gtid; c < C; c += gsize)
    sb[c] = src[b * C + c] - ((g == 0 && a.oldspec) ? a.oldspec[b * C + c] : 0.0f);
  named_bar(bid, gsize);
  if (g < 3) {
    const float thr = g == 1 ? a.thresh + a.var_add : a.thresh;
    grp_channflag(sb, thr, a, cmask, corr, tm, hist[g], sel[g], gtid, gsize, bid);
  } else {   // simple_channflag (:559-610)
    for (int i = gtid; i < n; i += gsize) corr[i] = sb[G + i];
    named_bar(bid, gsize);
    const int k = (n + 1) / 2 - 1;
    const float med = grp_radix_select(corr, n, k, hist[g], sel[g], gtid, gsize, bid);
    for (int i = gtid; i < n; i += gsize) tm[i] = fabsf(corr[i] - med);
    named_bar(bid, gsize);
    const float mad = grp_radix_select(tm, n, k, hist[g], sel[g], gtid, gsize, bid);
    const float mythr = (float)((double)a.thresh / sqrt((double)a.fbin));
    for (int j = G + gtid; j < C - G - a.fbin; j += gsize) {
      float vv = 0.0f;
      for (int q = 0; q < a.fbin; ++q) vv += a.parity ? sb[j] : sb[j + q];
      vv = vv / (float)a.fbin - med;
      if (vv > mythr * mad) cmask[j] = 1;
    }
  }
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < a.nperm; ++q) {
      const int j = a.perm[q];
      if (j >= G && j < C - G) cmask[j] = 1;
    }
  __syncthreads();
  int nflag = 0;
  for (int c = tid; c < C; c += flag::kStatThreads) {
    a.chanmask[b * C + c] = cmask[c];
    nflag += cmask[c];
  }
  if (nflag && a.counts) atomicAdd(a.counts, nflag);
}

// Total power of the block (every beam's spectrum summed in FP64 in a fixed
// order) and, with modcheck, the modulation test against the previous
// flagged block (:1313-1330): at or above mod_thresh the block is replaced
// by the noise block and nothing is flagged.  One CTA, the last one of the
// statistics grid.
__device__ void flag_total_power(const FlagArgs &a) {
  __shared__ double red[flag::kStatThreads];
  const int tid = threadIdx.x, BC = a.nbeam * a.nchan;
  double acc = 0.0;
  for (int i = tid; i < BC; i += flag::kStatThreads) acc += a.spec[i];
  red[tid] = acc;
  __syncthreads();
  if (tid == 0) {
    double tp = 0.0;
    for (int k = 0; k < flag::kStatThreads; ++k) tp += red[k];
    int rep = 0;
    if (a.modcheck) {
      const double prev = *a.prev_tpwr;
      if (prev > 0.0 && fabs(tp - prev) / prev >= (double)a.mod_thresh) rep = 1;
    }
    if (a.tpwr_out) *a.tpwr_out = tp;
    if (a.status) a.status[0] = rep;
  }
}

// flag (:459-474) then make_ts (:414-453), and for the beam's last CTA
// simple_tsflag (:612-653) and flagts (:479-494).  Grid (row chunks of
// kApplyRows, beams).  The flagged channels' 16-byte chunks are listed once
// per CTA (ballot scan, channel order); L lanes share a row, L the power of
// two covering the listed chunks (at most 32), so a few flagged channels
// cost a few sectors per row and a fully flagged row is read once,
// coalesced.  Each listed chunk is read, its flagged channels set to the
// level MN * bpwr (clean mode) and written back, and
//   ts = (row sum from the statistics pass + sum over flagged channels of
//         (level - x)) / nchan,
// which for uint8 is a sum of exact integers, so it equals the reference's
// float tree sum / NCHAN_P bit for bit.  Each CTA then counts itself in; the
// beam's last one takes the median and MAD (lower medians, by radix select)
// of the first ts_base samples, flags rows with ts - med > TsThr * MAD
// (one-sided) and, in clean mode, sets channels [guard, nchan - guard) of
// the flagged rows to the level.  A block the modulation check replaced
// gets the noise block in every beam (clean mode, :1323-1324) and zero
// masks; its ts keeps the raw row sums.
template <typename E>
__global__ void __launch_bounds__(flag::kApplyThreads) flag_apply_kernel(FlagArgs a) {
  constexpr int ES = (int)sizeof(E), EPC = 16 / ES;   // elements per 16-byte chunk
  const int b = blockIdx.y, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int C = a.nchan, G = a.guard, T = a.ntime, NCH = C / EPC;
  const int t_begin = blockIdx.x * flag::kApplyRows;
  const int t_end = min(T, t_begin + flag::kApplyRows);
  constexpr int nw = flag::kApplyThreads / 32;
  extern __shared__ __align__(16) uint32_t ash[];
  uint32_t *chk = ash;                                            // [NCH]
  float *tsb = reinterpret_cast<float *>(ash + NCH);              // [ts_base]
  float *tmp = tsb + a.ts_base;                                   // [ts_base]
  __shared__ uint32_t hist[256], sel[2];
  __shared__ int nact_sh, last_sh;
  __shared__ float lev_sh, lvl_sh;
  E *xw = a.clean ? elem_out<E>(a) : nullptr;
  uint8_t *mb = a.tsmask + (int64_t)b * T;
  if (a.status && a.status[0]) {   // replaced by noise
    const E *nz = static_cast<const E *>(a.noise);
    if (xw && nz) {
      const uint4 *src = reinterpret_cast<const uint4 *>(nz + (int64_t)t_begin * C);
      uint4 *dst = reinterpret_cast<uint4 *>(xw + ((int64_t)b * T + t_begin) * C);
      const int64_t nv = (int64_t)(t_end - t_begin) * C / EPC;
      for (int64_t i = tid; i < nv; i += flag::kApplyThreads) dst[i] = src[i];
    }
    for (int t = t_begin + tid; t < t_end; t += flag::kApplyThreads) mb[t] = 0;
    if (blockIdx.x == 0)
      for (int c = tid; c < C; c += flag::kApplyThreads) a.chanmask[b * C + c] = 0;
    if (blockIdx.x == 0 && b == 0 && tid == 0 && a.counts) {
      a.counts[0] = 0;
      a.counts[1] = 0;
    }
    return;
  }
  if (tid == 0) {   // calc_bpwr (:759-769): float sum over every channel, in order
    float lvl = a.bpwr ? a.bpwr[b] : 1.0f;
    if (a.pwr && a.bpwr) {
      float acc = 0.0f;
      for (int c = 0; c < C; ++c) acc += a.spec[b * C + c];
      lvl = (float)(((double)acc / (double)(C - 2 * G)) / (double)a.mn);
    }
    lvl_sh = lvl;
    lev_sh = a.mn * lvl;
  }
  if (warp == 0) {   // the chunks holding flagged channels: index | element mask << 16
    int base = 0;
    for (int k0 = 0; k0 < NCH; k0 += 32) {
      const int k = k0 + lane;
      uint32_t m = 0u;
      if (k < NCH)
        for (int e = 0; e < EPC; ++e) m |= (uint32_t)a.chanmask[b * C + k * EPC + e] << e;
      const uint32_t bal = __ballot_sync(0xffffffffu, m != 0u);
      if (m) chk[base + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)k | (m << 16);
      base += __popc(bal);
    }
    if (lane == 0) nact_sh = base;
  }
  __syncthreads();
  const int nact = nact_sh;
  const E re = repl_elem<E>(lev_sh);
  const float rf = (float)re;
  int L = 1;
  while (L < nact && L < 32) L <<= 1;
  const int rpw = 32 / L, sub = lane & (L - 1);
  const E *xin = (a.spec0 && elem_out<E>(a)) ? elem_out<E>(a) : elem_in<E>(a);
  for (int r0 = t_begin + warp * rpw; r0 < t_end; r0 += nw * rpw) {   // uniform per warp
    const int t = r0 + lane / L;
    double corr = 0.0;
    if (t < t_end) {
      const uint4 *row = reinterpret_cast<const uint4 *>(xin + ((int64_t)b * T + t) * C);
      uint4 *wrow = xw ? reinterpret_cast<uint4 *>(xw + ((int64_t)b * T + t) * C) : nullptr;
      for (int i = sub; i < nact; i += L) {
        const uint32_t ce = chk[i];
        const int k = (int)(ce & 0xFFFFu);
        const uint32_t m = ce >> 16;
        uint4 v = row[k];
        E *ve = reinterpret_cast<E *>(&v);
#pragma unroll
        for (int e = 0; e < EPC; ++e)
          if ((m >> e) & 1u) {
            corr += (double)(rf - (float)ve[e]);
            ve[e] = re;
          }
        if (wrow) wrow[k] = v;
      }
    }
    for (int o = L >> 1; o > 0; o >>= 1) corr += __shfl_xor_sync(0xffffffffu, corr, o);
    if (t < t_end && sub == 0) {
      double rsum;
      if (a.nslab == 1) {
        rsum = a.ts[(int64_t)b * T + t];
      } else {
        rsum = 0.0;
        for (int s = 0; s < a.nslab; ++s) rsum += a.rowsum[((int64_t)b * a.nslab + s) * T + t];
      }
      a.ts[(int64_t)b * T + t] = (float)((rsum + corr) / C);
    }
  }
  // the beam's last CTA makes the time-series decisions
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    last_sh = atomicAdd(a.ctr + a.nbeam + b, 1) == (int)gridDim.x - 1;
    if (blockIdx.x == 0 && a.pwr && a.bpwr) a.bpwr[b] = lvl_sh;
  }
  __syncthreads();
  if (!last_sh) return;
  __threadfence();
  if (!a.tsflag) {
    for (int t = tid; t < T; t += flag::kApplyThreads) mb[t] = 0;
    return;
  }
  const float *tb = a.ts + (int64_t)b * T;
  for (int i = tid; i < a.ts_base; i += flag::kApplyThreads) tsb[i] = tb[i];
  __syncthreads();
  const int kmed = (a.ts_base + 1) / 2 - 1;   // lower median
  const float med =
      grp_radix_select(tsb, a.ts_base, kmed, hist, sel, tid, flag::kApplyThreads, 1);
  for (int i = tid; i < a.ts_base; i += flag::kApplyThreads) tmp[i] = fabsf(tsb[i] - med);
  __syncthreads();
  const float mad =
      grp_radix_select(tmp, a.ts_base, kmed, hist, sel, tid, flag::kApplyThreads, 1);
  const float lim = a.ts_thresh * mad;
  int nts = 0;
  for (int t = tid; t < T; t += flag::kApplyThreads) {
    const uint8_t f = (tb[t] - med) > lim ? 1 : 0;
    mb[t] = f;
    nts += f;
  }
  if (nts && a.counts) atomicAdd(a.counts + 1, nts);
  if (!xw) return;
  __syncthreads();   // the row flags written above are read back by other threads
  for (int t = warp; t < T; t += nw) {
    if (!mb[t]) continue;
    E *row = xw + ((int64_t)b * T + t) * C;
    for (int c = G + lane; c < C - G; c += 32) row[c] = re;
  }
}

// fix_zspec (:114-170) over naver blocks of history: per (beam, channel),
// the value whose count of other values <= it equals naver / 2 (ties
// resolve to one value); if no value has that count the first block's is
// kept, as the kernel leaves s0[block_id] unwritten then.
__global__ void flag_zspec_kernel(const float *hs, const float *hv, int naver, int bc, float *s0,
                                  float *v0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= bc) return;
  const int place = naver / 2;
  for (int which = 0; which < 2; ++which) {
    const float *h = which ? hv : hs;
    float out = h[i];
    for (int k = 0; k < naver; ++k) {
      const float x = h[(int64_t)k * bc + i];
      int ct = 0;
      for (int j = 0; j < naver; ++j)
        if (j != k && h[(int64_t)j * bc + i] <= x) ++ct;
      if (ct == place) out = x;
    }
    (which ? v0 : s0)[i] = out;
  }
}

// median_calc (:771-798): per channel the lower median over beams
// (sorted[(nbeam + 1) / 2 - 1]; beam 31 of 64 in the reference), then
// broadcast to every beam.  One thread per channel.
__global__ void flag_medcalc_kernel(float *arr0, float *arr1, int nbeam, int nchan) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchan) return;
  const int k = (nbeam + 1) / 2 - 1;
  for (int which = 0; which < 2; ++which) {
    float *arr = which ? arr1 : arr0;
    float med = arr[c];
    for (int i = 0; i < nbeam; ++i) {
      const float x = arr[(int64_t)i * nchan + c];
      int r = 0;
      for (int j = 0; j < nbeam; ++j) {
        const float y = arr[(int64_t)j * nchan + c];
        r += (y < x) || (y == x && j < i);
      }
      if (r == k) med = x;
    }
    for (int i = 0; i < nbeam; ++i) arr[(int64_t)i * nchan + c] = med;
  }
}

// ---------------------------------------------------------------- launchers
static int stage_rows(const FlagArgs &a, int es) {
  const int cs = a.nchan < kFlagSlab ? a.nchan : kFlagSlab;
  int lim = flag::kStageTarget / (cs * es);
  if (lim > flag::kStatThreads) lim = flag::kStatThreads;
  if (lim > a.tbin) lim = a.tbin;
  for (int d = lim; d >= 1; --d)
    if (a.tbin % d == 0 && (!a.pix_sum || d % a.tds == 0)) return d;
  return 0;
}

bool flag_shape_ok(const FlagArgs &a) {
  const bool u8 = a.xu8 != nullptr;
  const int es = u8 ? 1 : 4;
  const void *x = u8 ? (const void *)a.xu8 : (const void *)a.x;
  if (!x || a.nchan < 4 || a.nchan > flag::kMaxChan || a.tbin < 1 || a.ntime < 1) return false;
  if ((a.nchan * es) % 16 || (reinterpret_cast<uintptr_t>(x) & 15u)) return false;
  if (a.pix_sum && (u8 || a.nchan > kFlagSlab || a.tds < 1 || a.tbin % a.tds ||
                    a.ntime % a.tbin))
    return false;
  // uint8 sums are 32-bit: at most 32768 rows per thread (P of the full slab)
  const int cs = a.nchan < kFlagSlab ? a.nchan : kFlagSlab;
  const int P = flag::kStatThreads / (cs / 4);
  if (u8 && (a.ntime + P - 1) / P > 32768) return false;
  FlagArgs t = a;
  return stage_rows(t, es) > 0;
}

// The largest layout over the launch's slabs: the full slab width cs and,
// when nchan is not a multiple of it, the narrower last slab (whose P x cs
// bin partials can exceed the full slab's).  Kept tight: at 48 channels two
// CTAs must share an SM.
static size_t stats_smem(const FlagArgs &a, int es) {
  const int cs = a.nchan < kFlagSlab ? a.nchan : kFlagSlab;
  const int last = a.nchan > kFlagSlab ? a.nchan % kFlagSlab : 0;
  auto bp = [](int w) { return (size_t)(flag::kStatThreads / (w / 4)) * w; };
  size_t nbp = bp(cs);
  if (last && bp(last) > nbp) nbp = bp(last);
  const size_t stage = ((size_t)a.rs * cs * es + 127) & ~(size_t)127;
  // row partials (int for uint8, double for FP32), bin partials, scaley
  // constants, and for scaled uint8 the [256][cs] table
  const size_t rsb = ((size_t)(es == 1 ? 4 : 8) * a.rs * ((cs / 4) | 1) + 15) & ~(size_t)15;
  const size_t stats = flag::kStages * stage + rsb + sizeof(double) * (nbp + cs) +
                       sizeof(float) * 2 * cs + (es == 1 && a.spec0 ? (size_t)256 * cs : 0);
  // the channel decisions reuse the buffer: 12 nchan floats + nchan bytes
  const size_t dec = a.decide ? sizeof(float) * 12 * (size_t)a.nchan + a.nchan : 0;
  return stats > dec ? stats : dec;
}

// The library-wide error word of flagger launches made without a context
// (dsax_flag_noalloc, the learned-flagger features), one per device.
static __device__ int g_flag_err;
static int *flag_err_word() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  static std::atomic<int *> addr[64] = {};
  int *p = addr[dev].load(std::memory_order_acquire);
  if (!p) {
    void *q = nullptr;
    if (cudaGetSymbolAddress(&q, g_flag_err) != cudaSuccess) return nullptr;
    p = static_cast<int *>(q);
    addr[dev].store(p, std::memory_order_release);
  }
  return p;
}

// The filterbank as a 2-D tensor [nbeam * ntime rows][nchan] of its element
// type, boxes [rs rows][min(nchan, 128) channels], zero fill past nchan.
static int encode_filterbank_map(CUtensorMap *map, const FlagArgs &a) {
  EncodeTiledFn fn = tensor_map_encoder();
  if (!fn) return -1;
  const bool u8 = a.xu8 != nullptr;
  const int es = u8 ? 1 : 4;
  const int bx = a.nchan < kFlagSlab ? a.nchan : kFlagSlab;
  const cuuint64_t dims[2] = {(cuuint64_t)a.nchan, (cuuint64_t)a.nbeam * (cuuint64_t)a.ntime};
  const cuuint64_t strides[1] = {(cuuint64_t)a.nchan * es};
  const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)a.rs};
  const cuuint32_t estr[2] = {1u, 1u};
  void *base = u8 ? (void *)a.xu8 : (void *)a.x;
  const CUresult r = fn(map, u8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

int launch_flag_stats(FlagArgs a, cudaStream_t st) {
  if (!flag_shape_ok(a)) return -1;
  const bool u8 = a.xu8 != nullptr;
  const int es = u8 ? 1 : 4;
  a.rs = stage_rows(a, es);
  a.nslab = (a.nchan + kFlagSlab - 1) / kFlagSlab;
  if (a.nslab > 1 && !a.rowsum) return -1;
  if (!a.err) a.err = flag_err_word();
  if (!a.err) return -2;
  if (!a.wait_limit_ns) a.wait_limit_ns = 1000000000ull;
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  if (encode_filterbank_map(&map, a) != 0) return -2;
  const size_t sh = stats_smem(a, es);
  const dim3 grid(a.nslab, a.nbeam);
  if (u8) {
    static SmemAttrOnce attr;
    if (smem_attr_once(attr, flag_stats_kernel<uint8_t>, 160 * 1024) != cudaSuccess) return -2;
    flag_stats_kernel<uint8_t><<<grid, flag::kStatThreads, sh, st>>>(map, a);
  } else {
    static SmemAttrOnce attr;
    if (smem_attr_once(attr, flag_stats_kernel<float>, 160 * 1024) != cudaSuccess) return -2;
    flag_stats_kernel<float><<<grid, flag::kStatThreads, sh, st>>>(map, a);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// The statistics pass (which ends with the channel decisions and the total
// power), then the row-chunked apply pass (whose last CTA per beam makes the
// time-series decisions): two launches on one stream.
int launch_flag(const FlagArgs &a0, cudaStream_t st) {
  FlagArgs a = a0;
  if (a.nchan > flag::kMaxChan || a.ts_base < 1 || a.ts_base > flag::kMaxTsBase ||
      a.ts_base > a.ntime)
    return -1;
  if (!a.ctr) return -1;
  a.ts_mean = 0;
  a.decide = 1;
  a.nslab = (a.nchan + kFlagSlab - 1) / kFlagSlab;
  if (cudaMemsetAsync(a.ctr, 0, sizeof(int) * flag_ctr_ints(a.nbeam), st) != cudaSuccess) return -2;
  int rc = launch_flag_stats(a, st);
  if (rc != 0) return rc;
  const bool u8 = a.xu8 != nullptr;
  const int nch = a.nchan * (u8 ? 1 : 4) / 16;
  const size_t sh = sizeof(uint32_t) * nch + sizeof(float) * 2 * (size_t)a.ts_base;
  const dim3 grid((a.ntime + flag::kApplyRows - 1) / flag::kApplyRows, a.nbeam);
  if (u8)
    flag_apply_kernel<uint8_t><<<grid, flag::kApplyThreads, sh, st>>>(a);
  else
    flag_apply_kernel<float><<<grid, flag::kApplyThreads, sh, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_flag_baseline(const float *hist_spec, const float *hist_var, int naver, int nbeam,
                         int nchan, float *spec0, float *var0, cudaStream_t st) {
  const int bc = nbeam * nchan;
  flag_zspec_kernel<<<(bc + 255) / 256, 256, 0, st>>>(hist_spec, hist_var, naver, bc, spec0, var0);
  flag_medcalc_kernel<<<(nchan + 127) / 128, 128, 0, st>>>(spec0, var0, nbeam, nchan);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

namespace dsax {
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
  if (!a.pix_sum || a.tds < 1 || a.ntime % a.tds || a.nchan > flag::kLfMaxChan) return -1;
  const int H = a.ntime / a.tds;
  const size_t sh = sizeof(float) * (2 * a.nchan + (a.ts_base > a.nchan ? a.ts_base : a.nchan) +
                                     4 * a.nchan + a.ntime + 2 * H);
  if (sh > 200 * 1024) return -1;
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, lf_stat_features_kernel, 200 * 1024) != cudaSuccess) return -2;
  lf_stat_features_kernel<<<a.nbeam, 2 * flag::kDecThreads, sh, st>>>(a, F, Fbf);
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
  // spec, var, max, pp, ts, the two flag counts, the launches' completion counters
  const long long need = 4 * nbc + nbt + 2 + (long long)flag_ctr_ints(B);
  if (need > kNoAllocScratchFloats) return DSAX_ERR_ARG;   // beyond the fixed 6 MiB
  if (C % 4 || (reinterpret_cast<uintptr_t>(x) & 15u)) return DSAX_ERR_ARG;
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
  a.ctr = a.counts + 2;
  // the counters accumulate with atomics: clear them (the array keeps the
  // previous call's values)
  if (cudaMemsetAsync(a.counts, 0, 2 * sizeof(int), st) != cudaSuccess) return DSAX_ERR_CUDA;
  if (launch_flag(a, st) != 0) return DSAX_ERR_CUDA;
  if (counts && cudaMemcpyAsync(counts, a.counts, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st) !=
                    cudaSuccess)
    return DSAX_ERR_CUDA;
  return DSAX_OK;
}

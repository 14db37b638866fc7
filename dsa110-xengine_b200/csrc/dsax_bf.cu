// dsax_bf.cu -- the Stokes-I beamformer on sm_100a tensor cores (BF16 in,
// FP32 accumulate in TMEM), with the 4-bit unpack fused into the operand
// staging and the detect + time/channel/pol sum + uint8 quantisation fused
// into the epilogue.
//
// Replaces src/dsaX_beamformer.cu promoter (:170-193), beamformer (:267-416,
// wmma m16n16k16 with FP16 accumulators), badder/adder (:79-158).
//
// Arithmetic.  For channel group g (8 fine channels), pol p and beam b, the
// beam voltage of sample s = (packet, chunnel = 2*chan + time) is
//     B[b][s] = sum_a w[g][p][b][a] * x[a][s]            (no conjugate)
// and the output is
//     P[t_out][b][g] = sum_{p} sum_{s in t_out} |B[b][s]|^2
// over ppo packets x 16 chunnels x 2 pols.
// As a real GEMM (K = 64 antennas x {re, im} = 128):
//     A row b      = [ wr_a, -wi_a ]_a   -> Re B
//     A row 64 + b = [ wi_a,  wr_a ]_a   -> Im B
//     B column s   = [ xr_a,  xi_a ]_a
// so one UMMA D[128 x 256] = A * B^T gives Re/Im of 64 beams x 256 samples.
//
// Tiling.  A CTA owns one beam tile of 64 beams and a range of (channel
// group g, packet group) pairs; the nbt CTAs of the beam tiles share the
// range and run it together, so L2 serves their common input.  A stage is
// 16 packets (256 samples) of one pol.  The weights of both pols (64 KB) of
// the current g stay resident; data stages are double buffered (64 KB
// each); the producers stage the next packet group's raw bytes (32 KB)
// with cp.async while they build the current one; TMEM holds two
// 256-column accumulators so the epilogue of stage i overlaps the MMAs of
// stage i+1.
//   warps 0-7 : producers (global 4-bit -> BF16 K-major swizzled tiles)
//   warps 8-11: epilogue (TMEM -> |.|^2 row sums -> outputs)
//   warp  12  : TMEM allocation, weight loader (bulk copy), single-thread
//               UMMA issuer
// This one-CTA form (bf_kernel) runs FP8 and odd beam-tile counts; BF16
// with an even count runs as CTA pairs (bf_pair_kernel, below), which
// halves the conversion and operand traffic per SM.
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "dsax_internal.h"
#include "dsax_ptx.cuh"

namespace dsax {

namespace bf {
constexpr int kPktPerStage = 16;                      // N = 16 packets x 16 chunnels = 256
constexpr int kN = 256;
constexpr int kKBlockBytes = 128;                     // one 128-byte K block per row
constexpr int kWTileBytes = 128 * kKBlockBytes;       // 128 rows x 128 B = 16 KB
constexpr int kDTileBytes = kN * kKBlockBytes;        // 256 rows x 128 B = 32 KB
constexpr int kProducers = 256;                       // 8 producer warps
constexpr int kRawRowBytes = kProducers * 16;         // one 16 B load per producer thread
constexpr int kRawBytes = 8 * kRawRowBytes;           // 32 KB: one packet group, both pols
// + 4 or 8 epilogue warps + the UMMA warp
constexpr int threads(int epi_warps) { return kProducers + 32 * epi_warps + 32; }
// Operand type: BF16 (K = 64 antennas x {re, im} = 128 elements in two
// 128-byte K blocks) or FP8 E4M3 (the same K in one 128-byte K block).
template <bool kFp8> struct T {
  static constexpr int kKB = kFp8 ? 1 : 2;            // K blocks per operand row
  static constexpr int kWBytes = 2 /*pol*/ * kKB * kWTileBytes;   // per (g, bt)
  static constexpr int kStageBytes = kKB * kDTileBytes;
  static constexpr int kStages = kFp8 ? 3 : 2;
  static constexpr int kSmemBytes = 1024 + kWBytes + kStages * kStageBytes + kRawBytes;
  // f8f6f4: E4M3 = 0 for A and B; f16: BF16 = 1
  static constexpr uint32_t kIdesc = kFp8 ? umma_idesc(1, 0, 0, 128, kN) : umma_idesc(1, 1, 1, 128, kN);
};
}  // namespace bf

// PTX prmt in its default mode: selector nibble bit 3 replicates the msb of
// the chosen byte over the result byte (CUDA's __byte_perm drops that bit).
__device__ __forceinline__ uint32_t prmt_sx(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// Two packed complex 4-bit samples (the low 16 bits of s: nibbles re0, im0,
// re1, im1, two's complement) -> their 4 E4M3 codes [re0 im0 re1 im1].  The
// nibbles are the PRMT selectors themselves.  A = table of e4m3(0..7)
// indexed by the nibble: negative nibbles (bit 3 set) replicate the msb of a
// positive code, 0.  B = table of |e4m3(-8..-1)| indexed by the nibble ^ 8:
// now the non-negative nibbles have bit 3 set and give 0.  B is nonzero
// exactly for the negative values, whose sign bit is then added.  Exact for
// all 16 values.
__device__ __forceinline__ uint32_t nib2_to_e4m3x4(uint32_t s) {
  const uint32_t A = prmt_sx(0x44403800u, 0x4e4c4a48u, s);            // 0 .. 7
  const uint32_t B = prmt_sx(0x4a4c4e50u, 0x38404448u, s ^ 0x8888u);  // |-8| .. |-1|
  return A | B | ((B + 0x7F7F7F7Fu) & 0x80808080u);
}

// As nib2_to_e4m3x4, each value times 2^d of its antenna: `add` holds 8d
// mod 128 per output byte ([d_a, d_a, d_b, d_b]), d in [-6, 5].  The
// exponent field of every nonzero code moves by d (the magnitude codes of
// 1..8 have exponents 7..10, so the result stays normal and below 0x7F);
// zero stays zero.  m + add stays below 0x100 in every byte, so no carry
// crosses bytes; the mask to 7 bits drops the mod-128 wrap of negative d.
__device__ __forceinline__ uint32_t nib2_to_e4m3x4_shift(uint32_t s, uint32_t add) {
  const uint32_t A = prmt_sx(0x44403800u, 0x4e4c4a48u, s);
  const uint32_t B = prmt_sx(0x4a4c4e50u, 0x38404448u, s ^ 0x8888u);
  const uint32_t m = A | B;                                        // |code|, 0 for 0
  const uint32_t nz = prmt_sx(m + 0x7F7F7F7Fu, 0u, 0xBA98u);        // 0xFF where nonzero
  const uint32_t r = m + (add & nz);
  return (r & 0x7F7F7F7Fu) | ((B + 0x7F7F7F7Fu) & 0x80808080u);
}

// acc + (x0^2, x1^2) for the FP32 bit patterns x0, x1, as one packed
// fma.rn.f32x2 (each lane rounds like fmaf).
__device__ __forceinline__ uint64_t sqacc_f32x2(uint32_t x0, uint32_t x1, uint64_t acc) {
  uint64_t x;
  asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "r"(x0), "r"(x1));
  asm("fma.rn.f32x2 %0, %1, %1, %0;" : "+l"(acc) : "l"(x));
  return acc;
}

// Sum of the two FP32 lanes of a packed pair.
__device__ __forceinline__ float hsum_f32x2(uint64_t v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return lo + hi;
}

// The units of a CTA's slot: they enumerate (channel group g, packet group
// pg, pol) g-major, and slot s of nslots takes a contiguous range of whole
// output times (align units).
struct BfRange {
  int u_lo, u_hi;
};
__device__ __forceinline__ BfRange bf_range(int slot, int nslots, int ngrp, int npg, int align) {
  const int nchunks = ngrp * npg * 2 / align;
  return {(int)((long long)slot * nchunks / nslots) * align,
          (int)((long long)(slot + 1) * nchunks / nslots) * align};
}
// Unit u: channel group g, packet group pg, pol = u % 2.
__device__ __forceinline__ void bf_decode(int u, int npg, int &g, int &pg, int &pol) {
  pol = u & 1;
  const int r = u >> 1;
  pg = r % npg;
  g = r / npg;
}

template <bool kFp8, int kEpiW>
__global__ void __launch_bounds__(bf::threads(kEpiW), 1) bf_kernel(BfArgs a) {
  using namespace bf;
  using TT = T<kFp8>;
  constexpr int kMmaWarp = 8 + kEpiW;                 // TMEM owner, weight loader, UMMA issuer
  constexpr int kEpiThreads = 32 * kEpiW;
  constexpr int kWBytes = TT::kWBytes, kStageBytes = TT::kStageBytes, kStages = TT::kStages;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar[2];
  __shared__ __align__(8) uint64_t tempty_bar[2];
  __shared__ __align__(8) uint64_t wload_bar;
  __shared__ __align__(8) uint64_t wdrain_bar;
  __shared__ __align__(8) uint64_t final_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ float red[kEpiW / 4][128];   // one output's row partials per column share

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t wsm = base;                  // weights [pol][kb][128 x 128 B]
  const uint32_t dsm = base + kWBytes;        // data stages [s][kb][256 x 128 B]
  const uint32_t raw = dsm + kStages * kStageBytes;   // producer staging [8][256][16 B]

  // Work split: the nbt CTAs of a slot (consecutive blockIdx) own the same
  // (g, pg) range, one beam tile each, and run it in lockstep, so each
  // input sector is fetched from HBM about once and then served by L2.
  // Ranges are whole output times (pgs_per_out packet groups).
  const int ngrp = a.nchan / 8, nbt = a.nbeam / 64, npg = a.npkt / kPktPerStage;
  const int align = 2 * (a.ppo > kPktPerStage ? a.ppo / kPktPerStage : 1);
  const int nslots = gridDim.x / nbt, slot = blockIdx.x / nbt, bt = blockIdx.x % nbt;
  const BfRange rg = bf_range(slot, nslots, ngrp, npg, align);
  const int u_lo = rg.u_lo, u_hi = rg.u_hi;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], kProducers);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], kEpiThreads);
    }
    mbar_init(&wload_bar, 1);
    mbar_init(&wdrain_bar, 1);
    mbar_init(&final_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(&tmem_base_sh, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if ((tmem & 0xFFFFu) != 0u) {
    if (tid == 0) atomicOr(a.err, DEV_ERR_TMEM);
    abort_sh = 1;
  }

  if (warp < 8) {
    // ------------------------------------------------------------ producers
    // Thread (kb, q, j): K block kb, packet q of the stage, antennas
    // 32 kb + 4j .. +3.  The 16 B loads of a (g, pg) carry both pols: they
    // are issued once, one packet group ahead (while the previous group's
    // two pol stages are built), and reused for the pol-1 stage.
    // FP8: thread (q, j, kh): antennas 8j .. 8j+7 (one 16-byte K chunk of
    // the single K block), channels 4kh .. 4kh+3 of the group.
    const int j = kFp8 ? (tid >> 1) & 7 : tid & 7;
    const int q = kFp8 ? tid >> 4 : (tid >> 3) & 15;   // packet within the stage
    const int kb = kFp8 ? 0 : tid >> 7;
    const int kh = kFp8 ? tid & 1 : 0;
    const int64_t ant_stride = (int64_t)a.nchan * 4;
    const int64_t pkt_stride = (int64_t)a.nant_in * ant_stride;
    // Each thread stages its own 8 loads of the next packet group in a
    // private slice of `raw` ([8][256 threads][16 B], conflict free) with
    // cp.async (zero fill for the padded antenna), and reads them back into
    // registers when that group starts, which frees the slice for the next
    // group's copies.
    const uint32_t myraw = raw + 16u * (uint32_t)tid;
    uint4 Ucur[8];
    // FP8: exponent offsets 8d of this thread's 8 antennas, one byte per
    // E4M3 output byte ([re, im] per antenna, two antennas per word)
    uint32_t shift_add[4] = {0u, 0u, 0u, 0u};
    if (kFp8 && a.e4m3_add) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t a0 = (uint32_t)a.e4m3_add[8 * j + 2 * e] & 0x7Fu;
        const uint32_t a1 = (uint32_t)a.e4m3_add[8 * j + 2 * e + 1] & 0x7Fu;
        shift_add[e] = a0 | (a0 << 8) | (a1 << 16) | (a1 << 24);
      }
    }
    auto stage_group = [&](int r) {
      const int g = r / npg, pg = r % npg;
      const int p = pg * kPktPerStage + q;
#pragma unroll
      for (int k8 = 0; k8 < 8; ++k8) {
        // BF16: k8 = (channel half h, antenna ii); FP8: k8 = antenna 8j + k8, half kh
        const int h = kFp8 ? kh : k8 >> 2;
        const int ant = kFp8 ? 8 * j + k8 : 32 * kb + 4 * j + (k8 & 3);
        const bool ok = ant < a.nant_in && p < a.npkt;
        const uint8_t *src = a.in + (ok ? p * pkt_stride + ant * ant_stride + (int64_t)(8 * g) * 4 +
                                              16 * h
                                        : 0);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                         myraw + (uint32_t)k8 * (kRawRowBytes)),
                     "l"(src), "r"(ok ? 16 : 0)
                     : "memory");
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (u_lo < u_hi) stage_group(u_lo >> 1);
    for (int u = u_lo, i = 0; u < u_hi && !abort_sh; ++u, ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      const int pol = u & 1;
      if (pol == 0) {
        asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
                       : "=r"(Ucur[k].x), "=r"(Ucur[k].y), "=r"(Ucur[k].z), "=r"(Ucur[k].w)
                       : "r"(myraw + (uint32_t)k * kRawRowBytes)
                       : "memory");
        }
        if (u + 2 < u_hi) stage_group((u >> 1) + 1);
      }
      if (!mbar_wait_bounded(&empty_bar[s], ph ^ 1u, &abort_sh, a.err, DEV_ERR_WAIT_EMPTY,
                             a.wait_limit_ns))
        break;
      const uint32_t sel = (uint32_t)pol | ((4u + pol) << 4) | ((2u + pol) << 8) | ((6u + pol) << 12);
      const uint32_t tile = dsm + (uint32_t)s * kStageBytes + (uint32_t)kb * kDTileBytes;
      if constexpr (kFp8) {
#pragma unroll
        for (int w = 0; w < 4; ++w) {                   // channel 4kh + w of the group
          // t[ag][pair]: antennas 8j + 4ag + 2pair, +1 at time 0 (bits 0-15)
          // and time 1 (bits 16-31)
          uint32_t t[2][2];
#pragma unroll
          for (int ag = 0; ag < 2; ++ag) {
            const uint4 *U = Ucur + 4 * ag;
            const uint32_t u0 = w == 0 ? U[0].x : w == 1 ? U[0].y : w == 2 ? U[0].z : U[0].w;
            const uint32_t u1 = w == 0 ? U[1].x : w == 1 ? U[1].y : w == 2 ? U[1].z : U[1].w;
            const uint32_t u2 = w == 0 ? U[2].x : w == 1 ? U[2].y : w == 2 ? U[2].z : U[2].w;
            const uint32_t u3 = w == 0 ? U[3].x : w == 1 ? U[3].y : w == 2 ? U[3].z : U[3].w;
            t[ag][0] = __byte_perm(u0, u1, sel);
            t[ag][1] = __byte_perm(u2, u3, sel);
          }
#pragma unroll
          for (int odd = 0; odd < 2; ++odd) {
            uint32_t o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const uint32_t sel2 = t[e >> 1][e & 1] >> (16 * odd);
              // per-antenna power-of-two scale only where the weights need it
              // (uniform branch)
              o[e] = a.e4m3_add ? nib2_to_e4m3x4_shift(sel2, shift_add[e]) : nib2_to_e4m3x4(sel2);
            }
            const int k = 8 * kh + 2 * w + odd;       // chunnel = 2*chan + time
            st_shared_v4(tile + sw128_offset((uint32_t)(16 * q + k), (uint32_t)j), o[0], o[1], o[2],
                         o[3]);
          }
        }
      } else {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const uint4 *U = Ucur + 4 * h;
          const uint32_t u0 = w == 0 ? U[0].x : w == 1 ? U[0].y : w == 2 ? U[0].z : U[0].w;
          const uint32_t u1 = w == 0 ? U[1].x : w == 1 ? U[1].y : w == 2 ? U[1].z : U[1].w;
          const uint32_t u2 = w == 0 ? U[2].x : w == 1 ? U[2].y : w == 2 ? U[2].z : U[2].w;
          const uint32_t u3 = w == 0 ? U[3].x : w == 1 ? U[3].y : w == 2 ? U[3].z : U[3].w;
          const uint32_t t01 = __byte_perm(u0, u1, sel);
          const uint32_t t23 = __byte_perm(u2, u3, sel);
#pragma unroll
          for (int odd = 0; odd < 2; ++odd) {
            const uint32_t x = __byte_perm(t01, t23, odd ? 0x7632u : 0x5410u);
            uint32_t o[4];
            nib8_to_bf16x8(x, o);
            const int k = 8 * h + 2 * w + odd;     // chunnel = 2*chan + time
            const uint32_t row = (uint32_t)(16 * q + k);
            st_shared_v4(tile + sw128_offset(row, (uint32_t)j), o[0], o[1], o[2], o[3]);
          }
        }
      }
      }
      fence_proxy_async_smem();
      mbar_arrive(&full_bar[s]);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");   // no copy outlives an aborted loop
  } else if (warp < kMmaWarp) {
    // ------------------------------------------------------------ epilogue
    // kEpiW / 4 warps per TMEM lane quarter (warp % 4), each taking an equal
    // share of the 256 accumulator columns.
    const int q = warp & 3;                          // TMEM lane quarter (warp % 4)
    const int half = (warp - 8) >> 2;                // column share
    constexpr int kCW = (kN / 32) / (kEpiW / 4);     // 32-column loads per warp
    const int m = 32 * q + lane;                     // accumulator row
    const int nsub = a.ppo < kPktPerStage ? kPktPerStage / a.ppo : 1;  // outputs per stage
    const int span = kN / nsub;                      // columns per output (>= 64)
    const int pgs_per_out = a.ppo > kPktPerStage ? a.ppo / kPktPerStage : 1;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    float bpow = 0.f;   // this CTA's share of the beam's total power (AGC)
    for (int u = u_lo, i = 0; u < u_hi; ++u, ++i) {
      const int b = i & 1;
      const uint32_t ph = (uint32_t)(i >> 1) & 1u;
      bool ok = mbar_wait_bounded(&tfull_bar[b], ph, &abort_sh, a.err, DEV_ERR_WAIT_ACCUM,
                                  a.wait_limit_ns);
      tc_fence_after();
      // The four epilogue warps never leave this loop early: they meet at the
      // named barriers below, which have no timeout.  After an abort they
      // skip the TMEM work (tcgen05.ld is .sync.aligned: warp-uniform test).
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)b * 256u;
      // squares summed in four independent chains: packed FP32x2 FMAs for
      // BF16 (measured 4.5 % faster), scalar FMAs for FP8 (there the packed
      // form measured 3 % slower)
#pragma unroll
      for (int cc = 0; cc < (ok ? kCW : 0); ++cc) {
        const int c = half * kCW + cc;
        uint32_t r0[32];
        tmem_ld32(taddr + 32u * c, r0);
        tmem_wait_ld();
        float sq;
        if constexpr (kFp8) {
          float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
          for (int e = 0; e < 32; e += 4) {
            const float v0 = __uint_as_float(r0[e]), v1 = __uint_as_float(r0[e + 1]);
            const float v2 = __uint_as_float(r0[e + 2]), v3 = __uint_as_float(r0[e + 3]);
            s0 = fmaf(v0, v0, s0);
            s1 = fmaf(v1, v1, s1);
            s2 = fmaf(v2, v2, s2);
            s3 = fmaf(v3, v3, s3);
          }
          sq = (s0 + s1) + (s2 + s3);
        } else {
          uint64_t s2[4] = {0ull, 0ull, 0ull, 0ull};     // (+0.0f, +0.0f) pairs
#pragma unroll
          for (int e = 0; e < 32; e += 8)
#pragma unroll
            for (int k = 0; k < 4; ++k) s2[k] = sqacc_f32x2(r0[e + 2 * k], r0[e + 2 * k + 1], s2[k]);
          sq = (hsum_f32x2(s2[0]) + hsum_f32x2(s2[1])) + (hsum_f32x2(s2[2]) + hsum_f32x2(s2[3]));
        }
        const int sub = (32 * c) / span;
        if (nsub == 1) acc[0] += sq;
        else if (sub == 0) acc[0] += sq;
        else if (sub == 1) acc[1] += sq;
        else if (sub == 2) acc[2] += sq;
        else acc[3] += sq;
      }
      tc_fence_before();
      mbar_arrive(&tempty_bar[b]);

      int g, pg, pol;
      bf_decode(u, npg, g, pg, pol);
      if (pol == 1 && ((pg + 1) % pgs_per_out) == 0) {
        // rows m and m + 64 hold Re and Im of the same beam; the column
        // shares of a row are summed through shared memory, one output at
        // a time (static shared memory is at its limit beside the stages)
        const int beam = 64 * bt + m;
#pragma unroll
        for (int sI = 0; sI < 4; ++sI) {
          if (sI >= nsub) break;
          red[half][m] = acc[sI];
          named_bar(1, kEpiThreads);
          if (half == 0 && m < 64 && !abort_sh) {
            float Ps = red[0][m] + red[0][m + 64];
#pragma unroll
            for (int h2 = 1; h2 < kEpiW / 4; ++h2) Ps += red[h2][m] + red[h2][m + 64];
            const float P = Ps * a.pscale;
            const int to = a.ppo <= kPktPerStage ? pg * nsub + sI : pg / pgs_per_out;
            const int64_t o = ((int64_t)to * a.nbeam + beam) * ngrp + g;
            if (a.out_f32) a.out_f32[o] = P;
            if (a.out_fb) a.out_fb[((int64_t)beam * (a.npkt / a.ppo) + to) * ngrp + g] = P;
            if (a.out_u8) {
              // AGC: rint(P * bp) / 2 as src/dsaX_beamformer.cu adder (:150-156),
              // saturated instead of wrapped
              int v = a.agc_scale ? __float2int_rn(P * __ldg(a.agc_scale + beam)) / 2
                                  : __float2int_rn(P * a.scale);
              a.out_u8[o] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
            bpow += P;
          }
          named_bar(1, kEpiThreads);
        }
        acc[0] = acc[1] = acc[2] = acc[3] = 0.f;
      }
    }
    if (a.beam_power && half == 0 && m < 64 && bpow != 0.f) atomicAdd(a.beam_power + 64 * bt + m, bpow);
  } else {
    // ------------------------------------------------------------ weights + UMMA
    if (lane == 0) {
      int cur_gb = -1;
      uint32_t nload = 0, ndrain = 0;
      for (int u = u_lo, i = 0; u < u_hi && !abort_sh; ++u, ++i) {
        int g, pg, pol;
        bf_decode(u, npg, g, pg, pol);
        const int gb = g * nbt + bt;
        if (gb != cur_gb) {
          if (i > 0) {  // no UMMA may still read the old weights
            umma_commit(&wdrain_bar);
            if (!mbar_wait_bounded(&wdrain_bar, ndrain & 1u, &abort_sh, a.err,
                                   DEV_ERR_WAIT_ACCUM, a.wait_limit_ns))
              break;
            ++ndrain;
          }
          mbar_arrive_expect_tx(&wload_bar, (uint32_t)kWBytes);
          const uint8_t *src = a.wimg + (int64_t)gb * kWBytes;
#pragma unroll
          for (int c = 0; c < kWBytes / 16384; ++c)
            bulk_g2s(wsm + 16384u * c, src + 16384 * c, 16384u, &wload_bar);
          if (!mbar_wait_bounded(&wload_bar, nload & 1u, &abort_sh, a.err, DEV_ERR_WAIT_FULL,
                                 a.wait_limit_ns)) {
            // the weight copies may still be landing: let them finish first
            volatile int no_abort = 0;
            mbar_wait_bounded(&wload_bar, nload & 1u, &no_abort, a.err, DEV_ERR_WAIT_FULL,
                              drain_limit(a.wait_limit_ns));
            break;
          }
          ++nload;
          cur_gb = gb;
        }
        const int s = i % kStages;
        const int b = i & 1;
        if (!mbar_wait_bounded(&full_bar[s], (uint32_t)(i / kStages) & 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_FULL, a.wait_limit_ns))
          break;
        if (!mbar_wait_bounded(&tempty_bar[b], ((uint32_t)(i >> 1) & 1u) ^ 1u, &abort_sh, a.err,
                               DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        tc_fence_after();
        const uint32_t wpol = wsm + (uint32_t)pol * (TT::kKB * kWTileBytes);
        const uint32_t stage = dsm + (uint32_t)s * kStageBytes;
#pragma unroll
        for (int kk = 0; kk < 4 * TT::kKB; ++kk) {   // 32-byte K steps (16 bf16 / 32 e4m3)
          const uint32_t kb = kk >> 2, koff = 32u * (kk & 3);
          const uint64_t ad = umma_desc_sw128(wpol + kb * kWTileBytes + koff, 1024u);
          const uint64_t bd = umma_desc_sw128(stage + kb * kDTileBytes + koff, 1024u);
          if constexpr (kFp8)
            umma_f8(tmem + (uint32_t)b * 256u, ad, bd, TT::kIdesc, kk > 0);
          else
            umma_f16(tmem + (uint32_t)b * 256u, ad, bd, TT::kIdesc, kk > 0);
        }
        umma_commit(&empty_bar[s]);
        umma_commit(&tfull_bar[b]);
      }
      umma_commit(&final_bar);
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM,
                        drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------- CTA pairs
// bf_pair_kernel: the beamformer (BF16 or FP8 E4M3 operands) with the two
// beam tiles of a 2-CTA cluster sharing each data stage through one
// cta_group::2 MMA (M = 256: 2 x 64 beams x re/im, N = 256 samples,
// K = 128).  Each CTA converts
// only its half of a stage's packets (8 of 16) into its own shared memory,
// and the pair's MMA reads both halves, so the 4-bit -> BF16 conversion,
// the staging copies and the shared-memory operand reads per SM drop from
// (A + B + B) to (A + B/2 + B/2) of a stage while the tensor work per SM
// stays the same.  The even CTA issues the MMAs; D lanes 0-127 (its beam
// tile) land in its TMEM, lanes 128-255 (the odd CTA's tile) in the odd
// CTA's TMEM, and each CTA's epilogue reduces its own tile as bf_kernel
// does, with two warps per TMEM lane quarter (eight in all: with the
// producers' work halved, the epilogue sets the pace; 4 and 16 measured
// slower) and kLdG 32-column TMEM loads in flight per wait.
//   warps 0-7 : producers; each warp's lane 0 arrives on the even CTA's
//               stage barrier (8 + 8 warp arrivals complete a stage)
//   warps 8-15: epilogue; each warp's lane 0 frees the accumulator on the
//               even CTA's barrier (8 + 8 arrivals)
//   warp  16  : TMEM allocation (both CTAs), own weight tile (both CTAs),
//               MMA issue (even CTA); stage / accumulator / weight-drain
//               releases are multicast commits to both CTAs
// Cross-CTA arrivals use the default release-at-CTA-scope form (the form
// of the CUDA templates' CTA-pair pipelines); release at cluster scope
// cost a memory barrier per arrival and measured about 25 % slower.
namespace bfp {
constexpr int kPktPerCta = 8;                        // packets of a 16-packet stage per CTA
constexpr int kDHalfBytes = 128 * bf::kKBlockBytes;  // 128 B rows x 128 B = 16 KB per K block
constexpr int kRawBytes = 16384;                     // 8 packets x 64 ant x 32 B
constexpr int threads(int epi_warps) { return bf::kProducers + 32 * epi_warps + 32; }
constexpr uint16_t kBoth = 0x3;                      // CTA mask of the pair
// BF16: two 128-byte K blocks per operand row; FP8 E4M3: one.  kRD raw
// staging slots (packet groups of loads in flight ahead of the one being
// converted).
template <bool kFp8, int kRD> struct T {
  static constexpr int kKB = kFp8 ? 1 : 2;
  static constexpr int kStageBytes = kKB * kDHalfBytes;
  static constexpr int kStages = kFp8 ? 6 : (kRD > 1 ? 3 : 4);
  static constexpr int kWBytes = 2 /*pol*/ * kKB * bf::kWTileBytes;   // own beam tile
  // raw staging per thread: BF16 four 16 B loads (4 antennas x 4 channels),
  // FP8 eight 8 B loads (8 antennas x 2 channels)
  static constexpr int kRawLoads = kFp8 ? 8 : 4;
  static constexpr int kRawLoadBytes = kFp8 ? 8 : 16;
  static constexpr int kRawRowBytes = bf::kProducers * kRawLoadBytes;
  static constexpr int kSmemBytes = 1024 + kWBytes + kStages * kStageBytes + kRD * kRawBytes;
  static constexpr uint32_t kIdesc =
      kFp8 ? umma_idesc(1, 0, 0, 256, bf::kN) : umma_idesc(1, 1, 1, 256, bf::kN);
};
}  // namespace bfp

template <bool kFp8, int kEpiW, int kLdG, int kRD>
__global__ void __launch_bounds__(bfp::threads(kEpiW), 1) bf_pair_kernel(BfArgs a) {
  using TT = bfp::T<kFp8, kRD>;
  constexpr int kMmaWarp = 8 + kEpiW;                 // TMEM, weights, MMA issue
  constexpr int kEpiThreads = 32 * kEpiW;
  using bf::kKBlockBytes;
  using bf::kN;
  using bf::kPktPerStage;
  using bf::kWTileBytes;
  constexpr int kStages = TT::kStages, kStageBytes = TT::kStageBytes;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages];   // even CTA: 16 producer-warp arrivals
  __shared__ __align__(8) uint64_t empty_bar[kStages];  // both: one commit
  __shared__ __align__(8) uint64_t tfull_bar[2];        // both: one commit
  __shared__ __align__(8) uint64_t tempty_bar[2];       // even CTA: 2 x kEpiW epilogue-warp arrivals
  __shared__ __align__(8) uint64_t wload_bar;           // own weight copy landed
  __shared__ __align__(8) uint64_t wpeer_bar;           // even CTA: the odd CTA's weights landed
  __shared__ __align__(8) uint64_t wdrain_bar;          // both: MMAs on the old weights done
  __shared__ __align__(8) uint64_t final_bar;           // both: every MMA done
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ float red[kEpiW / 4][128];   // one output's row partials per column share

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  // identical offsets in both CTAs (same kernel, same static shared memory)
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  const uint32_t wsm = base;                          // own A tile [pol][kb][128 x 128 B]
  const uint32_t dsm = base + TT::kWBytes;            // B halves [s][kb][128 x 128 B]
  const uint32_t raw = dsm + kStages * kStageBytes;   // producer staging [4][256][16 B]

  // Work split as bf_kernel: the nbt CTAs of a slot share a (g, pg) range;
  // nbt is even and a cluster is two consecutive blockIdx, so the beam
  // tile's parity is the CTA's rank in the pair.
  const int ngrp = a.nchan / 8, nbt = a.nbeam / 64, npg = a.npkt / kPktPerStage;
  const int align = 2 * (a.ppo > kPktPerStage ? a.ppo / kPktPerStage : 1);
  const int nslots = gridDim.x / nbt, slot = blockIdx.x / nbt, bt = blockIdx.x % nbt;
  const BfRange rg = bf_range(slot, nslots, ngrp, npg, align);
  const int u_lo = rg.u_lo, u_hi = rg.u_hi;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 16);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 2 * kEpiW);
    }
    mbar_init(&wload_bar, 1);
    mbar_init(&wpeer_bar, 1);
    mbar_init(&wdrain_bar, 1);
    mbar_init(&final_bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc_pair(&tmem_base_sh, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_barrier();      // both CTAs' barriers exist before any remote arrival
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if ((tmem & 0xFFFFu) != 0u) {
    if (tid == 0) atomicOr(a.err, DEV_ERR_TMEM);
    abort_sh = 1;
  }
  // the even CTA's barriers, in the cluster window (also for the even CTA)
  const uint32_t full0 = cluster_map(&full_bar[0], 0);
  const uint32_t tempty0 = cluster_map(&tempty_bar[0], 0);
  const uint32_t wpeer0 = cluster_map(&wpeer_bar, 0);

  if (warp < 8) {
    // ------------------------------------------------------------ producers
    // BF16: thread (kb, q8, j, h): K block kb, packet 8 rank + q8 of the
    // stage, antennas 32 kb + 4j .. +3, channels 4h .. 4h+3 of the group:
    // four 16 B loads per packet group (both pols), eight 16 B stores per
    // stage.  FP8: thread (q8, j, kh, w2): packet 8 rank + q8, antennas
    // 8j .. 8j+7 (one 16-byte K chunk of the single K block), channels
    // 4kh + 2w2 + {0, 1}: eight 8 B loads, four 16 B stores per stage.
    const int q8 = kFp8 ? tid >> 5 : (tid >> 4) & 7;
    const int j = kFp8 ? (tid >> 2) & 7 : (tid >> 1) & 7;
    const int h = kFp8 ? (tid >> 1) & 1 : tid & 1;     // channel half
    const int w2 = tid & 1;                            // FP8: channel pair of the half
    const int kb = kFp8 ? 0 : tid >> 7;
    const int q = bfp::kPktPerCta * (int)rank + q8;
    const int64_t ant_stride = (int64_t)a.nchan * 4;
    const int64_t pkt_stride = (int64_t)a.nant_in * ant_stride;
    const uint32_t myraw = raw + (uint32_t)TT::kRawLoadBytes * (uint32_t)tid;
    uint32_t U[TT::kRawLoads][TT::kRawLoadBytes / 4];
    // FP8: exponent offsets 8d of this thread's 8 antennas, one byte per
    // E4M3 output byte ([re, im] per antenna, two antennas per word)
    uint32_t shift_add[4] = {0u, 0u, 0u, 0u};
    if (kFp8 && a.e4m3_add) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t a0 = (uint32_t)a.e4m3_add[8 * j + 2 * e] & 0x7Fu;
        const uint32_t a1 = (uint32_t)a.e4m3_add[8 * j + 2 * e + 1] & 0x7Fu;
        shift_add[e] = a0 | (a0 << 8) | (a1 << 16) | (a1 << 24);
      }
    }
    auto stage_group = [&](int r) {
      const int g = r / npg, pg = r % npg;
      const int p = pg * kPktPerStage + q;
      const uint32_t slot = (uint32_t)(r % kRD) * bfp::kRawBytes;
#pragma unroll
      for (int ii = 0; ii < TT::kRawLoads; ++ii) {
        const int ant = kFp8 ? 8 * j + ii : 32 * kb + 4 * j + ii;
        const bool ok = ant < a.nant_in && p < a.npkt;
        const int chan = 8 * g + 4 * h + (kFp8 ? 2 * w2 : 0);
        const uint8_t *src = a.in + (ok ? p * pkt_stride + ant * ant_stride + (int64_t)chan * 4 : 0);
        const uint32_t dst = myraw + slot + (uint32_t)ii * TT::kRawRowBytes;
        if constexpr (kFp8)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src),
                       "r"(ok ? 8 : 0)
                       : "memory");
        else
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                       "r"(ok ? 16 : 0)
                       : "memory");
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // packet groups r = u / 2 of the range: the first kRD are staged now,
    // group r + kRD when group r is read (into the slot it frees)
#pragma unroll
    for (int d = 0; d < kRD; ++d)
      if (2 * ((u_lo >> 1) + d) < u_hi) stage_group((u_lo >> 1) + d);
    // every exit from this loop is warp-uniform (the warp meets in
    // __syncwarp / __all_sync below)
    for (int u = u_lo, i = 0; u < u_hi; ++u, ++i) {
      if (__any_sync(0xffffffffu, abort_sh != 0)) break;
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      const int pol = u & 1;
      if (pol == 0) {
        const int r = u >> 1;
        // group r's copies landed (with two slots the next group may still be in flight)
        if (kRD > 1 && 2 * (r + 1) < u_hi)
          asm volatile("cp.async.wait_group 1;" ::: "memory");
        else
          asm volatile("cp.async.wait_all;" ::: "memory");
        const uint32_t slot = (uint32_t)(r % kRD) * bfp::kRawBytes;
#pragma unroll
        for (int k = 0; k < TT::kRawLoads; ++k) {
          const uint32_t src = myraw + slot + (uint32_t)k * TT::kRawRowBytes;
          if constexpr (kFp8)
            asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];"
                         : "=r"(U[k][0]), "=r"(U[k][1])
                         : "r"(src)
                         : "memory");
          else
            asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
                         : "=r"(U[k][0]), "=r"(U[k][1]), "=r"(U[k][2]), "=r"(U[k][3])
                         : "r"(src)
                         : "memory");
        }
        if (2 * (r + kRD) < u_hi) stage_group(r + kRD);
      }
      const bool ok = mbar_wait_bounded(&empty_bar[s], ph ^ 1u, &abort_sh, a.err,
                                        DEV_ERR_WAIT_EMPTY, a.wait_limit_ns);
      if (!__all_sync(0xffffffffu, ok)) break;
      const uint32_t sel = (uint32_t)pol | ((4u + pol) << 4) | ((2u + pol) << 8) | ((6u + pol) << 12);
      const uint32_t tile = dsm + (uint32_t)s * kStageBytes + (uint32_t)kb * bfp::kDHalfBytes;
      if constexpr (kFp8) {
#pragma unroll
        for (int wl = 0; wl < 2; ++wl) {                // channel 4h + 2 w2 + wl of the group
          // t[ag][pair]: antennas 8j + 4ag + 2pair, +1 at time 0 (bits 0-15)
          // and time 1 (bits 16-31)
          uint32_t t[2][2];
#pragma unroll
          for (int ag = 0; ag < 2; ++ag) {
            t[ag][0] = __byte_perm(U[4 * ag][wl], U[4 * ag + 1][wl], sel);
            t[ag][1] = __byte_perm(U[4 * ag + 2][wl], U[4 * ag + 3][wl], sel);
          }
#pragma unroll
          for (int odd = 0; odd < 2; ++odd) {
            uint32_t o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const uint32_t sel2 = t[e >> 1][e & 1] >> (16 * odd);
              o[e] = a.e4m3_add ? nib2_to_e4m3x4_shift(sel2, shift_add[e]) : nib2_to_e4m3x4(sel2);
            }
            const int k = 8 * h + 2 * (2 * w2 + wl) + odd;   // chunnel = 2*chan + time
            const uint32_t row = (uint32_t)(16 * q8 + k);     // row of this CTA's B half
            st_shared_v4(tile + sw128_offset(row, (uint32_t)j), o[0], o[1], o[2], o[3]);
          }
        }
      } else {
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const uint32_t t01 = __byte_perm(U[0][w], U[1][w], sel);
          const uint32_t t23 = __byte_perm(U[2][w], U[3][w], sel);
#pragma unroll
          for (int odd = 0; odd < 2; ++odd) {
            const uint32_t x = __byte_perm(t01, t23, odd ? 0x7632u : 0x5410u);
            uint32_t o[4];
            nib8_to_bf16x8(x, o);
            const int k = 8 * h + 2 * w + odd;      // chunnel = 2*chan + time
            const uint32_t row = (uint32_t)(16 * q8 + k);   // row of this CTA's B half
            st_shared_v4(tile + sw128_offset(row, (uint32_t)j), o[0], o[1], o[2], o[3]);
          }
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(full0 + 8u * (uint32_t)s);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");   // no copy outlives an aborted loop
  } else if (warp < kMmaWarp) {
    // ------------------------------------------------------------ epilogue
    // kEpiW / 4 warps per TMEM lane quarter (warp % 4), each taking an equal
    // share of the 256 accumulator columns.
    const int qq = warp & 3;                         // TMEM lane quarter (warp % 4)
    const int half = (warp - 8) >> 2;                // column share
    constexpr int kCW = (kN / 32) / (kEpiW / 4);     // 32-column loads per warp
    const int m = 32 * qq + lane;                    // accumulator row of this CTA's tile
    const int nsub = a.ppo < kPktPerStage ? kPktPerStage / a.ppo : 1;
    const int span = kN / nsub;
    const int pgs_per_out = a.ppo > kPktPerStage ? a.ppo / kPktPerStage : 1;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    float bpow = 0.f;
    for (int u = u_lo, i = 0; u < u_hi; ++u, ++i) {
      const int b = i & 1;
      const uint32_t ph = (uint32_t)(i >> 1) & 1u;
      bool ok = mbar_wait_bounded(&tfull_bar[b], ph, &abort_sh, a.err, DEV_ERR_WAIT_ACCUM,
                                  a.wait_limit_ns);
      tc_fence_after();
      ok = __all_sync(0xffffffffu, ok && !abort_sh);
      const uint32_t taddr = tmem + ((uint32_t)(32 * qq) << 16) + (uint32_t)b * 256u;
#pragma unroll
      // kLdG 32-column TMEM loads in flight per wait
      for (int cc = 0; cc < (ok ? kCW : 0); cc += kLdG) {
        uint32_t r0[kLdG][32];
#pragma unroll
        for (int gi = 0; gi < kLdG; ++gi) tmem_ld32(taddr + 32u * (half * kCW + cc + gi), r0[gi]);
        tmem_wait_ld();
#pragma unroll
        for (int gi = 0; gi < kLdG; ++gi) {
          const int c = half * kCW + cc + gi;
          float sq;
          if constexpr (kFp8) {   // scalar chains (the packed form measured slower for FP8)
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
            for (int e = 0; e < 32; e += 4) {
              const float v0 = __uint_as_float(r0[gi][e]), v1 = __uint_as_float(r0[gi][e + 1]);
              const float v2 = __uint_as_float(r0[gi][e + 2]), v3 = __uint_as_float(r0[gi][e + 3]);
              s0 = fmaf(v0, v0, s0);
              s1 = fmaf(v1, v1, s1);
              s2 = fmaf(v2, v2, s2);
              s3 = fmaf(v3, v3, s3);
            }
            sq = (s0 + s1) + (s2 + s3);
          } else {
            uint64_t s2[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
            for (int e = 0; e < 32; e += 8)
#pragma unroll
              for (int k = 0; k < 4; ++k)
                s2[k] = sqacc_f32x2(r0[gi][e + 2 * k], r0[gi][e + 2 * k + 1], s2[k]);
            sq = (hsum_f32x2(s2[0]) + hsum_f32x2(s2[1])) + (hsum_f32x2(s2[2]) + hsum_f32x2(s2[3]));
          }
          const int sub = (32 * c) / span;
          if (nsub == 1) acc[0] += sq;
          else if (sub == 0) acc[0] += sq;
          else if (sub == 1) acc[1] += sq;
          else if (sub == 2) acc[2] += sq;
          else acc[3] += sq;
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(tempty0 + 8u * (uint32_t)b);

      int g, pg, pol;
      bf_decode(u, npg, g, pg, pol);
      if (pol == 1 && ((pg + 1) % pgs_per_out) == 0) {
        // rows m and m + 64 hold Re and Im of the same beam; the column
        // shares of a row are summed through shared memory, one output at
        // a time
        const int beam = 64 * bt + m;
#pragma unroll
        for (int sI = 0; sI < 4; ++sI) {
          if (sI >= nsub) break;
          red[half][m] = acc[sI];
          named_bar(1, kEpiThreads);
          if (half == 0 && m < 64 && !abort_sh) {
            float Ps = red[0][m] + red[0][m + 64];
#pragma unroll
            for (int h2 = 1; h2 < kEpiW / 4; ++h2) Ps += red[h2][m] + red[h2][m + 64];
            const float P = Ps * a.pscale;
            const int to = a.ppo <= kPktPerStage ? pg * nsub + sI : pg / pgs_per_out;
            const int64_t o = ((int64_t)to * a.nbeam + beam) * ngrp + g;
            if (a.out_f32) a.out_f32[o] = P;
            if (a.out_fb) a.out_fb[((int64_t)beam * (a.npkt / a.ppo) + to) * ngrp + g] = P;
            if (a.out_u8) {
              int v = a.agc_scale ? __float2int_rn(P * __ldg(a.agc_scale + beam)) / 2
                                  : __float2int_rn(P * a.scale);
              a.out_u8[o] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
            bpow += P;
          }
          named_bar(1, kEpiThreads);
        }
        acc[0] = acc[1] = acc[2] = acc[3] = 0.f;
      }
    }
    if (a.beam_power && half == 0 && m < 64 && bpow != 0.f)
      atomicAdd(a.beam_power + 64 * bt + m, bpow);
  } else {
    // ------------------------------------------------------------ weights + MMA
    if (lane == 0) {
      int cur_g = -1;
      uint32_t nload = 0, ndrain = 0;
      for (int u = u_lo, i = 0; u < u_hi && !abort_sh; ++u, ++i) {
        int g, pg, pol;
        bf_decode(u, npg, g, pg, pol);
        if (g != cur_g) {
          if (i > 0) {  // no MMA may still read either CTA's old weights
            if (leader) umma_commit_pair(&wdrain_bar, bfp::kBoth);
            if (!mbar_wait_bounded<true>(&wdrain_bar, ndrain & 1u, &abort_sh, a.err,
                                         DEV_ERR_WAIT_ACCUM, a.wait_limit_ns))
              break;
            ++ndrain;
          }
          mbar_arrive_expect_tx(&wload_bar, (uint32_t)TT::kWBytes);
          const uint8_t *src = a.wimg + (int64_t)(g * nbt + bt) * TT::kWBytes;
#pragma unroll
          for (int c = 0; c < TT::kWBytes / 16384; ++c)
            bulk_g2s(wsm + 16384u * c, src + 16384 * c, 16384u, &wload_bar);
          if (!mbar_wait_bounded(&wload_bar, nload & 1u, &abort_sh, a.err, DEV_ERR_WAIT_FULL,
                                 a.wait_limit_ns)) {
            volatile int no_abort = 0;
            mbar_wait_bounded(&wload_bar, nload & 1u, &no_abort, a.err, DEV_ERR_WAIT_FULL,
                              drain_limit(a.wait_limit_ns));
            break;
          }
          if (!leader) {
            mbar_arrive_cluster(wpeer0);
          } else if (!mbar_wait_bounded<true>(&wpeer_bar, nload & 1u, &abort_sh, a.err,
                                              DEV_ERR_WAIT_FULL, a.wait_limit_ns)) {
            break;
          }
          ++nload;
          cur_g = g;
        }
        if (!leader) continue;
        const int s = i % kStages;
        const int b = i & 1;
        if (!mbar_wait_bounded(&full_bar[s], (uint32_t)(i / kStages) & 1u, &abort_sh, a.err,
                                     DEV_ERR_WAIT_FULL, a.wait_limit_ns))
          break;
        if (!mbar_wait_bounded(&tempty_bar[b], ((uint32_t)(i >> 1) & 1u) ^ 1u, &abort_sh,
                                     a.err, DEV_ERR_WAIT_EMPTY, a.wait_limit_ns))
          break;
        tc_fence_after();
        const uint32_t wpol = wsm + (uint32_t)pol * (uint32_t)(TT::kKB * kWTileBytes);
        const uint32_t stage = dsm + (uint32_t)s * kStageBytes;
#pragma unroll
        for (int kk = 0; kk < 4 * TT::kKB; ++kk) {   // 32-byte K steps (16 bf16 / 32 e4m3)
          const uint32_t kb = kk >> 2, koff = 32u * (kk & 3);
          const uint64_t ad = umma_desc_sw128(wpol + kb * kWTileBytes + koff, 1024u);
          const uint64_t bd = umma_desc_sw128(stage + kb * bfp::kDHalfBytes + koff, 1024u);
          if constexpr (kFp8)
            umma_f8_pair(tmem + (uint32_t)b * 256u, ad, bd, TT::kIdesc, kk > 0);
          else
            umma_f16_pair(tmem + (uint32_t)b * 256u, ad, bd, TT::kIdesc, kk > 0);
        }
        umma_commit_pair(&empty_bar[s], bfp::kBoth);
        umma_commit_pair(&tfull_bar[b], bfp::kBoth);
      }
      if (leader) umma_commit_pair(&final_bar, bfp::kBoth);
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    if (lane == 0) {
      volatile int no_abort = 0;
      mbar_wait_bounded<true>(&final_bar, 0u, &no_abort, a.err, DEV_ERR_WAIT_ACCUM,
                              drain_limit(a.wait_limit_ns));
    }
    __syncwarp();
  }
  tc_fence_before();
  cluster_barrier();      // both CTAs past their last TMEM read and remote arrival
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc_pair(tmem, 512);
}

// Slots of a launch: at most one per pair of units of whole output times.
static int bf_slots(const BfArgs &a, int nslots) {
  const int ngrp = a.nchan / 8, npg = a.npkt / bf::kPktPerStage;
  const int align = 2 * (a.ppo > bf::kPktPerStage ? a.ppo / bf::kPktPerStage : 1);
  const int nchunks = ngrp * npg * 2 / align;
  if (nslots < 1) nslots = 1;
  return nslots > nchunks ? nchunks : nslots;
}

template <bool kFp8, int kEpiW, int kLdG, int kRD>
static int launch_bf_pair(const BfArgs &a, int num_sms, cudaStream_t st) {
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, bf_pair_kernel<kFp8, kEpiW, kLdG, kRD>, bfp::T<kFp8, kRD>::kSmemBytes) != cudaSuccess) return -2;
  const int nbt = a.nbeam / 64;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(bfp::threads(kEpiW), 1, 1);
  cfg.dynamicSmemBytes = bfp::T<kFp8, kRD>::kSmemBytes;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  // One wave: as many slots as pairs of SMs can hold clusters at once (an
  // SM left without a partner in its GPC takes none), per device.
  static std::atomic<int> max_clusters[64];   // per kernel instantiation and device
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -2;
  int maxc = dev >= 0 && dev < 64 ? max_clusters[dev].load(std::memory_order_relaxed) : 0;
  if (maxc <= 0) {
    cfg.gridDim = dim3((unsigned)(2 * num_sms), 1, 1);
    if (cudaOccupancyMaxActiveClusters(&maxc, bf_pair_kernel<kFp8, kEpiW, kLdG, kRD>, &cfg) != cudaSuccess ||
        maxc < 1)
      maxc = num_sms / 2;
    if (dev >= 0 && dev < 64) max_clusters[dev].store(maxc, std::memory_order_relaxed);
  }
  const int nslots = bf_slots(a, maxc / (nbt / 2));
  cfg.gridDim = dim3((unsigned)(nslots * nbt), 1, 1);
  return cudaLaunchKernelEx(&cfg, bf_pair_kernel<kFp8, kEpiW, kLdG, kRD>, a) == cudaSuccess ? 0 : -2;
}

bool beamform_pair_ok(const BfArgs &a) { return a.nbeam % 128 == 0; }

template <bool kFp8, int kEpiW>
static int launch_bf(const BfArgs &a, int num_sms, cudaStream_t st) {
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, bf_kernel<kFp8, kEpiW>, bf::T<kFp8>::kSmemBytes) != cudaSuccess)
    return -2;
  const int nbt = a.nbeam / 64;
  const int nslots = bf_slots(a, num_sms / nbt);
  const int grid = nslots * nbt;
  void *args[] = {(void *)&a};
  return cudaLaunchKernel((const void *)bf_kernel<kFp8, kEpiW>, dim3(grid),
                          dim3(bf::threads(kEpiW)), args, bf::T<kFp8>::kSmemBytes,
                          st) == cudaSuccess
             ? 0
             : -2;
}

int launch_beamform(const BfArgs &a, int num_sms, cudaStream_t st) {
  // default and 2: CTA pairs where they apply (BF16, an even number of
  // 64-beam tiles); 1, FP8 and the rest: one CTA per beam tile
  // FP8 epilogues keep two TMEM loads in flight (2.4 % faster; BF16 1 % slower)
  // FP8: two raw staging slots beside its six 16 KB stages (1 % faster);
  // BF16 keeps one slot and four 32 KB stages (three stages and two slots
  // measured 4 % slower)
  if (a.path != 1 && beamform_pair_ok(a)) {
    // variant: (TMEM loads per wait, raw staging slots) = 1 (1,1), 2 (2,1),
    // 3 (1,2), 4 (2,2); 0 = the default above per operand type
    const int v = a.variant ? a.variant : (a.fp8 ? 4 : 1);
    if (a.fp8) {
      switch (v) {
        case 1: return launch_bf_pair<true, 8, 1, 1>(a, num_sms, st);
        case 2: return launch_bf_pair<true, 8, 2, 1>(a, num_sms, st);
        case 3: return launch_bf_pair<true, 8, 1, 2>(a, num_sms, st);
        default: return launch_bf_pair<true, 8, 2, 2>(a, num_sms, st);
      }
    }
    switch (v) {
      case 2: return launch_bf_pair<false, 8, 2, 1>(a, num_sms, st);
      case 3: return launch_bf_pair<false, 8, 1, 2>(a, num_sms, st);
      case 4: return launch_bf_pair<false, 8, 2, 2>(a, num_sms, st);
      default: return launch_bf_pair<false, 8, 1, 1>(a, num_sms, st);
    }
  }
  return a.fp8 ? launch_bf<true, 4>(a, num_sms, st) : launch_bf<false, 4>(a, num_sms, st);
}

}  // namespace dsax

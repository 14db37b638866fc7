// dsax_internal.h -- launch-argument structs shared between the kernels and
// the C-ABI layer (not installed; the public interface is include/dsax.h).
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace dsax {

// Per-device "max dynamic shared memory" attribute of one kernel.
// cudaFuncSetAttribute applies to the current device only, so the set-once
// state is one bit per device (devices 0..63; higher ordinals set it on
// every launch), kept in an atomic so that host threads driving different
// contexts may launch concurrently.  Two threads racing on a device's first
// launch both set the same value, which is harmless.
struct SmemAttrOnce {
  std::atomic<unsigned long long> done{0ull};
};
template <typename Kernel>
inline cudaError_t smem_attr_once(SmemAttrOnce &once, Kernel kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
  if (bit && (once.done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel),
                           cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) once.done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

// ---- error codes written to the device error word (bit flags) ----
enum : int {
  DEV_ERR_WAIT_FULL = 1 << 0,    // consumer gave up waiting for a filled stage
  DEV_ERR_WAIT_EMPTY = 1 << 1,   // producer gave up waiting for a free stage
  DEV_ERR_WAIT_ACCUM = 1 << 2,   // epilogue gave up waiting for the accumulator
  DEV_ERR_TMEM = 1 << 3,         // TMEM allocation returned an unusable address
  DEV_ERR_BOUNDS = 1 << 4,       // an index check failed (access skipped)
};

// Input formats accepted by the correlator.
enum {
  FMT_CAPTURED = 0,   // [pkt][nant_in][nchan][2 t][2 pol] 4+4-bit (CAPTURED key)
  FMT_REORDERED = 1,  // [pkt][2 nchan][64][2 pol] 4+4-bit (REORDER key, massage())
  FMT_XGPU_INT8 = 2,  // [pkt][2 nchan][64][2 pol][re,im] int8 (xGPU ComplexInput)
};

struct CorrArgs {
  const uint8_t *in;       // device input block
  float *vis;              // device output [2 nchan][2080][4][re,im]
  int *err;                // device error word (bit flags, dsax_ptx.cuh)
  int npkt;                // packets (xGPU time samples) per block
  int nant_in;             // antennas present in the captured block (<= 64)
  int nchan;               // channels (= CTAs); frequencies = 2 * nchan
  int accumulate;          // 1: vis += block's products (xGPU integration buffer)
  unsigned long long wait_limit_ns;  // bound on every pipeline wait
};

int launch_correlate(const CorrArgs &a, int fmt, cudaStream_t st);

}  // namespace dsax

namespace dsax {

struct BfArgs {
  const uint8_t *in;       // captured block [npkt][nant_in][nchan][2 t][2 pol]
  const uint8_t *wimg;     // weight operand image [ngrp][nbeam/64][2 pol][2 kb][16 KB]
  uint8_t *out_u8;         // [npkt/ppo][nbeam][nchan/8] Stokes-I uint8 (or null)
  float *out_f32;          // same layout, FP32 power before scaling (or null)
  float *out_fb;           // [nbeam][npkt/ppo][nchan/8] FP32 power (filterbank order, or null)
  float pscale = 1.0f;     // power scale: 1 (BF16); FP8 2^-2E undoes the operands' 2^E
  const signed char *e4m3_add;  // FP8: per-antenna data exponent 8d (64 entries) or null
  int fp8;                 // operands: 0 BF16 (kind::f16), 1 FP8 E4M3 (kind::f8f6f4)
  const float *agc_scale;  // per-beam AGC scale: u8 = rint(P * s) / 2 (or null: fixed scale)
  float *beam_power;       // per-beam total power of the block, accumulated (or null)
  int *err;
  int npkt, nant_in, nchan, nbeam, ppo;
  float scale;
  unsigned long long wait_limit_ns;
};

int launch_beamform(const BfArgs &a, int num_sms, cudaStream_t st);

// AGC bandpass state (dsax_agc.cu): per-beam scale for the next block from
// this block's per-beam power.
constexpr int kAgcNbp = 8;   // blocks averaged once the history is full
int launch_agc_update(void *state, int nbeam, int ngrp, int nints, cudaStream_t st);
size_t agc_state_bytes(int nbeam);
float *agc_scale_ptr(void *state, int nbeam);
float *agc_power_ptr(void *state, int nbeam);

}  // namespace dsax

namespace dsax {

struct FlagArgs {
  const float *x;          // filterbank [nbeam][ntime][nchan] FP32 (device)
  const float *oldspec;    // previous block's spec [nbeam][nchan] or null
  float *spec, *var, *maxs, *pp, *ts;   // statistics (device)
  uint8_t *chanmask;       // [nbeam][nchan]
  uint8_t *tsmask;         // [nbeam][ntime]
  int *counts;             // [2]: flagged (beam, chan) columns, (beam, t) rows
  int nbeam, ntime, nchan, guard, filt, tbin, fbin, ts_base, tsflag, parity;
  float thresh, var_add, ts_thresh;
  int nperm;
  int perm[8];
  // optional downsampled spectrogram (staged statistics kernel only; needs
  // tbin % tds == 0): per (beam, pixel row of tds samples, chan) sum and max
  float *pix_sum = nullptr, *pix_max = nullptr;
  int tds = 0;
};

int launch_flag(const FlagArgs &a, cudaStream_t st);
// Statistics pass only (spec, var, max, pp, ts and the optional pixel sums);
// returns -1 when the staged kernel cannot take the shape.
int launch_flag_stats(const FlagArgs &a, cudaStream_t st);
bool flag_stats_staged_ok(const FlagArgs &a);
// Learned-flagger features F[B][T/tds][C][8] from a finished statistics pass
// (spec, var, maxs, pp, ts, pix_sum, pix_max of `a`).
// F (FP32, may be null) and / or Fbf (BF16, may be null).
int launch_lf_stat_features(const FlagArgs &a, float *F, uint16_t *Fbf, cudaStream_t st);

}  // namespace dsax

namespace dsax {
int launch_reorder(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                   cudaStream_t st);
}  // namespace dsax

namespace dsax {
// Channel-major corner turn: [nchan][npkt][64][4 B] (internal layout).
int launch_reorder_chanmajor(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                             cudaStream_t st);
// bulk_fed: the operand feed is one cp.async.bulk per 64-packet stage (true)
// or direct coalesced loads into registers (false).
int launch_correlate_chanmajor(const CorrArgs &a, cudaStream_t st, bool bulk_fed);
}  // namespace dsax

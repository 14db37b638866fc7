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
  int path;                // kernel form (dsax_config.bf_path)
  int variant;             // CTA-pair stage parameters (dsax_config.bf_variant)
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
  const float *x = nullptr;      // filterbank [nbeam][ntime][nchan] FP32 (device), or
  const uint8_t *xu8 = nullptr;  // the same as uint8 (the reference's type)
  float *xw = nullptr;           // where scaled / replaced FP32 data go (clean mode; may be x)
  uint8_t *xw8 = nullptr;        // the same for uint8
  const float *oldspec = nullptr;  // previous block's spec [nbeam][nchan] or null
  float *spec = nullptr, *var = nullptr, *maxs = nullptr, *pp = nullptr;  // [nbeam][nchan]
  float *ts = nullptr;           // [nbeam][ntime] channel-mean series (after replacement)
  float *rowsum = nullptr;       // [nbeam][nslab][ntime] raw row sums when nslab > 1
  uint8_t *chanmask = nullptr;   // [nbeam][nchan]
  uint8_t *tsmask = nullptr;     // [nbeam][ntime]
  int *counts = nullptr;         // [2]: flagged (beam, chan) columns, (beam, t) rows
  int nbeam = 0, ntime = 0, nchan = 0, guard = 0, filt = 0, tbin = 0, fbin = 0, ts_base = 0;
  int tsflag = 0, parity = 0;
  float thresh = 0.f, var_add = 0.f, ts_thresh = 0.f;
  int nperm = 0;
  int perm[8] = {};
  // optional downsampled spectrogram (FP32, one channel slab; needs
  // tbin % tds == 0): per (beam, pixel row of tds samples, chan) sum and max
  float *pix_sum = nullptr, *pix_max = nullptr;
  int tds = 0;
  // statistics-pass geometry, set by the launcher
  int nslab = 1;                 // channel slabs of kFlagSlab channels (CTAs per beam)
  int rs = 0;                    // rows per pipeline stage (divides tbin)
  int ts_mean = 0;               // 1: the statistics pass writes ts = row mean (no apply pass)
  // data path (src/gpu_flagger.cu:1290-1410)
  int clean = 0;                 // 1: replace flagged columns / rows in xw / xw8
  float mn = 48.0f;              // MN: replacement level (x bpwr[beam])
  float sig = 6.0f;              // SIG: scaley target standard deviation
  const float *spec0 = nullptr, *var0 = nullptr;  // scaley baseline [nbeam][nchan] (null: none)
  float *bpwr = nullptr;         // per-beam level [nbeam] (null: 1)
  int pwr = 0;                   // 1: bpwr from this block's spectrum (calc_bpwr)
  int modcheck = 0;              // 1: total-power modulation check against *prev_tpwr
  float mod_thresh = 0.0005f;
  const double *prev_tpwr = nullptr;  // previous flagged block's total power (0: none)
  double *tpwr_out = nullptr;    // this block's total power
  int *status = nullptr;         // [0] = 1 when the block was replaced by noise
  const void *noise = nullptr;   // replacement block [ntime][nchan] (element type of x)
  // completion counters, [2 nbeam + 2] ints zeroed by launch_flag: per-beam
  // slab CTAs done, per-beam apply CTAs done, CTAs of the statistics grid
  // done (the last arrival of each does the next step; nothing spins)
  int *ctr = nullptr;
  int decide = 0;                // statistics pass also makes the channel decisions
  // bounded waits of the statistics pass (TMA stages): where a wait that
  // ran out is recorded (a context's error word; null: a library-wide word)
  // and the bound (0: 1 s)
  int *err = nullptr;
  unsigned long long wait_limit_ns = 0;
};

// ints of FlagArgs::ctr for nbeam beams
inline size_t flag_ctr_ints(int nbeam) { return 2 * (size_t)nbeam + 2; }

constexpr int kFlagSlab = 128;   // channels per statistics CTA

int launch_flag(const FlagArgs &a, cudaStream_t st);
// Statistics pass only (spec, var, max, pp, ts and the optional pixel sums).
// With a.ts_mean the series is the plain row mean.  Returns -1 when the
// shape is not supported.
int launch_flag_stats(FlagArgs a, cudaStream_t st);
bool flag_shape_ok(const FlagArgs &a);
// Learned-flagger features F[B][T/tds][C][8] from a finished statistics pass
// (spec, var, maxs, pp, ts, pix_sum, pix_max of `a`).
// F (FP32, may be null) and / or Fbf (BF16, may be null).
int launch_lf_stat_features(const FlagArgs &a, float *F, uint16_t *Fbf, cudaStream_t st);
// Scaley baseline from naver blocks of history (fix_zspec, then median_calc
// across beams): hist_spec / hist_var [naver][nbeam][nchan] -> spec0 / var0.
int launch_flag_baseline(const float *hist_spec, const float *hist_var, int naver, int nbeam,
                         int nchan, float *spec0, float *var0, cudaStream_t st);

}  // namespace dsax

namespace dsax {
int launch_reorder(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                   cudaStream_t st);
}  // namespace dsax

namespace dsax {
// Channel-major corner turn: [nchan][npkt][64][4 B] (internal layout).
int launch_reorder_chanmajor(const uint8_t *in, uint8_t *out, int npkt, int nant_in, int nchan,
                             cudaStream_t st);
// corr_path selects the operand feed: 3 direct coalesced loads into
// registers, 5 and 7 one cp.async.bulk per 64-packet stage unpacked by 16
// warps, anything else (4, 6) the same bulk feed unpacked by 8 warps.
int launch_correlate_chanmajor(const CorrArgs &a, cudaStream_t st, int corr_path);
// The captured block [npkt][nant_in][nchan][4 B] correlated directly (no
// corner turn): clusters of four channel CTAs, TMA boxes split across the
// cluster through distributed shared memory.  Needs nchan % 4 == 0 and a
// 16-byte aligned block; returns -1 otherwise.
bool captured_cluster_ok(const CorrArgs &a);
int launch_correlate_captured_cluster(const CorrArgs &a, cudaStream_t st, int unpack_warps);
// corr_path 6 (8 unpack warps) and 7 (16) select the captured-block feed.
inline bool corr_path_fused(int corr_path) { return corr_path == 6 || corr_path == 7; }
inline int corr_path_unpack_warps(int corr_path) { return corr_path == 7 ? 16 : 8; }
}  // namespace dsax

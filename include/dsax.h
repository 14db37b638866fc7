/*
 * dsax.h -- C ABI of the B200 (sm_100a) DSA-110 X-engine hot path.
 *
 * One library, libdsax.so, replaces the GPU stages of the reference
 * pipeline behind plain C calls (pointers, sizes, int status codes):
 *
 *   dsax_correlate  <- src/dsaX_reorder_raw.c massage() (:99-219)
 *                      + src/dsaX_xgpu.cu promoter (:67-77)
 *                      + xgpuCudaXengine / xgpuClearDeviceIntegrationBuffer
 *                        (:318, :336)
 *   dsax_beamform   <- src/dsaX_beamformer.cu promoter/beamformer/adder
 *                      (:121-416) with calc_weights (:421-449)
 *   dsax_flag       <- src/gpu_flagger.cu statistics kernels (:175-494)
 *                      + host flagging (:534-798, :1340-1398)
 *
 * The xGPU call shapes used at src/dsaX_xgpu.cu:253-287 are also exported
 * with their original names by include/xgpu_dsax.h, so a caller written
 * against xGPU can relink without source changes.
 *
 * Conventions
 *  - Every function returns an int status: DSAX_OK (0) or a negative
 *    DSAX_ERR_* code.  The library never exits the process.
 *  - A context owns one CUDA device, one stream and its device scratch.
 *    Calls on one context are serialised by the caller (a context is not
 *    thread-safe); several contexts may be used concurrently.
 *  - mem = DSAX_MEM_HOST: input and output pointers are host memory; the
 *    call copies in, computes, copies out and synchronises before
 *    returning.  Pinned host memory (dsax_host_alloc) makes the copies
 *    asynchronous DMA transfers.
 *    mem = DSAX_MEM_DEVICE: pointers are device memory on the context's
 *    device; the work is enqueued on the context stream and the call
 *    returns without waiting.  dsax_sync() waits and reports any
 *    device-side error.
 */
#ifndef DSAX_H
#define DSAX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define DSAX_OK 0
#define DSAX_ERR_ARG (-1)         /* bad argument, size, alignment or layout */
#define DSAX_ERR_CUDA (-2)        /* CUDA runtime error; see dsax_last_error */
#define DSAX_ERR_TIMEOUT (-3)     /* a bounded device-side wait expired */
#define DSAX_ERR_NOMEM (-4)       /* device or host allocation failed */
#define DSAX_ERR_UNSUPPORTED (-5) /* device is not a compute-capability 10.0 GPU */
#define DSAX_ERR_DEVICE (-6)      /* a device-side check failed */

/* ---- memory kinds ---- */
#define DSAX_MEM_HOST 0
#define DSAX_MEM_DEVICE 1

/* ---- correlator input formats ---- */
#define DSAX_FMT_CAPTURED 0  /* [pkt][nant_in][nchan][2 t][2 pol], 4+4-bit   */
#define DSAX_FMT_REORDERED 1 /* [pkt][2*nchan][64][2 pol], 4+4-bit (REORDER key) */
#define DSAX_FMT_XGPU_INT8 2 /* [pkt][2*nchan][64][2 pol][re,im] int8         */
#define DSAX_FMT_CHANMAJOR 3 /* [nchan][pkt][64][2 t][2 pol], 4+4-bit (corner-turned) */

typedef struct dsax_config {
    int npkt;            /* packets per block = xGPU NTIME (2048)                 */
    int nant_in;         /* antennas present in the captured block (63, <= 64)     */
    int nchan;           /* channels per packet (384); frequencies = 2*nchan      */
    int nbeam;           /* beams formed (256; multiple of 64)                     */
    int bf_pkt_per_out;  /* packets per Stokes-I output sample (16 = 32 times)    */
    float bf_scale;      /* fixed scale before the uint8 quantisation             */
    unsigned long long wait_limit_ns; /* bound on device waits (0 = 1 s)          */
    int corr_path;       /* captured-block correlation: 0 = default (= 4),
                            1 = one fused kernel reading the captured layout,
                            2 = corner turn to the REORDER layout + correlate,
                            3 = corner turn to channel-major streams + correlate
                                fed by direct coalesced loads,
                            4 = as 3, fed by one bulk copy per 64-packet stage,
                            5 = as 4, unpacked by 16 warps instead of 8,
                            6 = no corner turn: the correlator reads the
                                captured block in clusters of four channel
                                CTAs (TMA boxes split through distributed
                                shared memory; needs nchan % 4 == 0, else 4),
                            7 = as 6, unpacked by 16 warps.
                            3 to 7 also select the feed for
                            DSAX_FMT_CHANMAJOR (6 as 4, 7 as 5) */
    int bf_fp8;          /* beamformer operands: 0 BF16 (tcgen05 kind::f16), 1 FP8
                            E4M3 with a per-antenna power-of-two scale
                            (kind::f8f6f4; the 4-bit data, shifted by the
                            antenna's exponent, are exact in E4M3) */
    int bf_path;         /* beamformer kernel form: 0 = default (2 where it
                            applies, else 1), 1 = one CTA per 64-beam tile,
                            2 = CTA pairs: the two beam tiles of a 2-CTA
                                cluster share each data stage through one
                                cta_group::2 MMA of M = 256 (BF16 or
                                FP8, nbeam % 128 == 0; else as 1) */
    int bf_variant;      /* CTA-pair beamformer stage parameters: 0 = the
                            default for the operand type (BF16 1, FP8 4);
                            1..4 = (TMEM loads in flight per epilogue wait,
                            raw staging slots of packet groups in flight) =
                            (1, 1), (2, 1), (1, 2), (2, 2); two slots cost
                            BF16 one of its four operand stages.  All give
                            the same beams; dsax_autotune_beamformer picks */
} dsax_config;

typedef struct dsax_ctx dsax_ctx;

/* Fills cfg with the reference block geometry (src/dsaX_def.h:72-81,
 * README.md:34-62): npkt 2048, nant_in 63, nchan 384, nbeam 256,
 * bf_pkt_per_out 16. */
void dsax_default_config(dsax_config *cfg);

/* Sizes in bytes of the block layouts for a configuration. */
size_t dsax_block_bytes(const dsax_config *cfg, int fmt);
size_t dsax_vis_bytes(const dsax_config *cfg);   /* 2*nchan*2080*4 complex float */
size_t dsax_beam_bytes(const dsax_config *cfg);  /* (npkt/bf_pkt_per_out)*nbeam*(nchan/8) */

int dsax_create(dsax_ctx **ctx, const dsax_config *cfg, int device);
void dsax_destroy(dsax_ctx *ctx);
const char *dsax_strerror(int status);
const char *dsax_last_error(const dsax_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that enqueue
 * their own work around DSAX_MEM_DEVICE calls. */
void *dsax_stream(dsax_ctx *ctx);

/* Waits for all work on the context stream; returns DSAX_ERR_TIMEOUT or
 * DSAX_ERR_DEVICE if a kernel recorded a device-side error since the last
 * check (and clears it). */
int dsax_sync(dsax_ctx *ctx);

/* Pins caller-owned host memory (e.g. a shared-memory ring buffer) for
 * asynchronous DMA, as src/dsaX_bfCorr.cu:86-114 does with
 * cudaHostRegister; undo with dsax_unregister_host before freeing it. */
int dsax_register_host(dsax_ctx *ctx, void *p, size_t n);
int dsax_unregister_host(dsax_ctx *ctx, void *p);

/* Pinned host memory for fast transfers (cudaHostAlloc / cudaFreeHost). */
int dsax_host_alloc(dsax_ctx *ctx, size_t nbytes, void **ptr);
int dsax_host_free(dsax_ctx *ctx, void *ptr);

/* ---- correlator ----
 * Replaces massage() + promoter + xgpuCudaXengine(ctx, in, SYNCOP_DUMP)
 * (src/dsaX_reorder_raw.c:153-169, src/dsaX_xgpu.cu:312-340).
 * in  : one block in format `fmt` (dsax_block_bytes(cfg, fmt) bytes,
 *       16-byte aligned).
 * vis : xGPU triangular visibilities, MATRIX_ORDER_TRIANGULAR:
 *       vis[((f*2080 + i*(i+1)/2 + j)*4 + 2*pol_i + pol_j)] = {re, im}
 *       (float), f = 2*chan + time, j <= i, value sum_t x_i conj(x_j).
 *       Bit-exact to an FP32 accumulation (all sums are integers < 2^24).
 * accumulate = 0 overwrites vis; 1 adds the block's products to vis (the
 * xGPU device integration buffer semantics).  Host-memory calls always
 * overwrite. */
int dsax_correlate(dsax_ctx *ctx, const void *in, void *vis, int mem);

/* nblk CAPTURED blocks -> nblk xGPU triangular visibility buffers.  With
 * mem = DSAX_MEM_HOST the stages of consecutive blocks overlap: block i+1's
 * copy in and corner turn run on side streams while block i is correlated
 * and block i-1 copied out (pinned host buffers give asynchronous DMA).  In
 * device mode block i+1's corner turn runs on a side stream beside block
 * i's correlation, on the SMs the correlator's CTAs free as they finish.
 * Replaces the per-block loop of src/dsaX_xgpu.cu:300-357 (H2D,
 * promoter, xgpuCudaXengine, matrix copy-out, one block at a time).  Device
 * mode enqueues (ordered on the context stream); host mode returns when all
 * visibilities are in the host buffers.  Output always overwrites.  Uses
 * the channel-major path (corr_path 3 or 4 selects the correlator feed). */
int dsax_correlate_many(dsax_ctx *ctx, const void *const *blocks, void *const *vis, int nblk,
                        int mem);

/* Packet capture -> block assembly (src/dsaX_capture.c receive_obs
 * :870-960) for npk packets in device memory, `stride` bytes apart: an
 * 8-byte header (35-bit sequence number in bytes 0-4, 16-bit antenna id in
 * bytes 6-7, big-endian) and `payload` bytes (multiple of 8) at offset 8.
 * Slot act = seq * slots_per_seq + ant_lookup[ant_id] (ant_lookup: device
 * int[nlookup], -1 = unknown) goes to block slot act - act0 when below
 * nslots, else to next_block (may be NULL) when below 2 nslots; earlier
 * slots are late.  counts (device, 4 x uint64, accumulated): placed,
 * placed in the next block, late, dropped (beyond / unknown antenna).
 * Enqueued on the context stream. */
int dsax_place_packets(dsax_ctx *ctx, const void *pkts, int npk, int stride, int payload,
                       const int *ant_lookup, int nlookup, unsigned long long act0,
                       unsigned long long nslots, int slots_per_seq, void *block, void *next_block,
                       unsigned long long *counts);

/* simple_extract of src/dsaX_writevis.c:55-74 on the GPU: XX and YY
 * (pol-products 0 and 3) averaged over the two time slots of each channel,
 * xGPU triangular visibilities -> [2080 baselines][nchan][2 pol][re, im]
 * float (dsax_extract_bytes).  dsax_correlate_extract correlates a
 * CAPTURED block and extracts on the device, so only the product is copied
 * out in host mode. */
size_t dsax_extract_bytes(const dsax_config *cfg);
int dsax_extract(dsax_ctx *ctx, const void *vis, void *out, int mem);
int dsax_correlate_extract(dsax_ctx *ctx, const void *in, void *out, int mem);

/* The same with the options of the visibility writers:
 * order = DSAX_BL_XGPU keeps xGPU's baseline order; DSAX_BL_GREG writes the
 *   baselines in the "Greg" order of src/dsaX_wrangleAndWrite.c gen_lookup /
 *   reorder_gh (:46-93): antenna pairs (i, j >= i), i major, so output
 *   baseline k holds xGPU baseline lookup[k].
 * autos (may be NULL): [nant_in][nchan] float spectra to which auto_extract
 *   (src/dsaX_wrangle.c:47-70) adds, per antenna and channel, the real part
 *   of the time-slot-averaged XX and then YY autocorrelation (accumulated
 *   across calls, as the reference sums N_INTS blocks before writing).
 * out may be NULL when autos is given.  Pointers follow `mem`. */
#define DSAX_BL_XGPU 0
#define DSAX_BL_GREG 1
int dsax_extract_ex(dsax_ctx *ctx, const void *vis, void *out, int order, float *autos, int mem);
int dsax_correlate_extract_ex(dsax_ctx *ctx, const void *in, void *out, int order, float *autos,
                              int mem);

/* Autotuner: times the captured-block correlator variants (corr_path 1 to
 * 7) on a synthetic block of the context's geometry (reps launches each),
 * sets the context's corr_path to the fastest, and returns the per-variant
 * milliseconds (times_ms[0..6] for paths 1..7, up to ntimes) and the choice. */
int dsax_autotune(dsax_ctx *ctx, int reps, float *times_ms, int ntimes, int *best_path);

/* Beamformer autotuner: times, with the context's weights (dsax_set_weights
 * first) on a synthetic block of its geometry, five candidates: (1) the
 * one-CTA form (bf_path 1) and (2-5) the CTA-pair form (bf_path 2) with
 * bf_variant 1-4; keeps the fastest in the context's bf_path / bf_variant,
 * and returns the milliseconds (times_ms[0..4], up to ntimes) and the
 * candidate number (1-5).  Every candidate computes the same beams (FP32
 * power within 1e-5 relative). */
int dsax_autotune_beamformer(dsax_ctx *ctx, int reps, float *times_ms, int ntimes,
                             int *best_path);

/* Measured dense tensor-core throughput of the context's GPU (ops/s, best
 * of reps): every SM issues back-to-back tcgen05.mma M=128 N=256 from shared
 * memory.  kind 0: int8 (kind::i8, as the correlator), 1: BF16 (kind::f16,
 * as the beamformer), 2: FP8 E4M3 (kind::f8f6f4).  No reference
 * counterpart: the denominator for the int8 and FP8 roofline fractions. */
int dsax_probe_tensor_peak(dsax_ctx *ctx, int kind, int reps, double *ops_per_s);

/* Failure detection check (no reference counterpart): one kernel waits on a
 * barrier that nothing completes, with the same bounded wait the pipelines
 * use, limited to limit_ns (<= 10 s).  Returns DSAX_ERR_TIMEOUT from the
 * device error word, as any kernel whose wait expired does; the context
 * stays usable. */
int dsax_check_wait_limit(dsax_ctx *ctx, unsigned long long limit_ns);

/* massage() on the GPU (src/dsaX_reorder_raw.c:153-169): captured block ->
 * REORDER-key layout [pkt][2*nchan][64][2 pol] (4+4-bit kept packed, padded
 * antennas zero).  dsax_block_bytes(cfg, DSAX_FMT_REORDERED) bytes out. */
int dsax_reorder(dsax_ctx *ctx, const void *captured, void *reordered, int mem);

/* Corner turn of a captured block into out_fmt = DSAX_FMT_REORDERED (as
 * dsax_reorder) or DSAX_FMT_CHANMAJOR (one contiguous stream per channel,
 * the layout the default correlator path reads). */
int dsax_corner_turn(dsax_ctx *ctx, const void *captured, void *out, int out_fmt, int mem);
int dsax_correlate_fmt(dsax_ctx *ctx, int fmt, const void *in, void *vis, int mem,
                       int accumulate);

/* ---- beamformer ----
 * Replaces the promoter/beamformer/adder chain of src/dsaX_beamformer.cu
 * (:121-416) and the weight upload of calc_weights (:421-449).
 *
 * dsax_set_weights: complex weights in FP64, host memory, layout
 *   [nchan/8 groups][2 pol][nbeam][64 antennas] (re and im arrays), the
 *   product of the geometric phase and the calibration as calc_weights
 *   forms it.  Converted once (round-to-nearest-even) to the BF16 operand
 *   image kept on the device; FP64 is used only here.
 * dsax_beamform: one captured block -> Stokes-I
 *   out[t][beam][group] = sum over 2 pols x bf_pkt_per_out packets x
 *   8 channels x 2 times of |sum_a w * x|^2 (no conjugate on w, as
 *   src/dsaX_beamformer.cu:376-378), t = packet / bf_pkt_per_out.
 *   out_u8  : saturate(rint(P * bf_scale)) in [0, 255] (the reference wraps
 *             modulo 256 instead, src/dsaX_beamformer.cu:150-156), or NULL;
 *   out_f32 : P itself (FP32), or NULL.  At least one must be given.
 *   Requires nchan % 8 == 0, nbeam % 64 == 0, npkt % 16 == 0 and
 *   bf_pkt_per_out in {4, 8, 16, 32, ...} dividing npkt. */

/* Geometric fan-beam weights computed in FP64 from the array description
 * (src/dsaX_beamformer.cu calc_weights :421-449, init_weights :559-602):
 * antpos[64] antenna eastings (m), cal[64][nchan/8][2 pol][re, im]
 * calibration gains (weights use cal / |cal|^2), flagged[64] (nonzero:
 * antenna zeroed; may be NULL), fch1_mhz (first channel), sep_arcmin (beam
 * separation; beam b points at sep x (127 - b)).  Group g's frequency is
 * fch1 - (8g + 4) x 250/8192 MHz.  Replaces dsax_set_weights' input. */
int dsax_set_geometric_weights(dsax_ctx *ctx, const double *antpos, const double *cal,
                               const int *flagged, double fch1_mhz, double sep_arcmin);
int dsax_set_weights(dsax_ctx *ctx, const double *wre, const double *wim);

/* Two-arm weights with a declination term, the cuBLAS beamformer's
 * populate_weights_matrix (src/dsaX_bfCorr.cu:815-863, calc_weights
 * :869-928): beams [0, nbeam/2) are formed from the E-W arm (arm[a] == 0,
 * phase from antpos_e), beams [nbeam/2, nbeam) from the N-S arm (arm[a] ==
 * 1, phase from antpos_n, the beam angle offset by -dec_deg degrees; the
 * reference passes 37.23 - its observation declination); an antenna only
 * contributes to its own arm's beams (arm[a] = -1: to none).  Beam b of an
 * arm points at sep x (nbeam/4 - 1 - b) arcmin (127 - b for 256 beams per
 * arm); group g's frequency is sfreq - g x 250/1024 MHz (:1131); gains are
 * cal / |cal| (:891-895), zero for flagged antennas.  Computed in FP64,
 * then converted as dsax_set_weights.  Needs nbeam % 128 == 0. */
int dsax_set_two_arm_weights(dsax_ctx *ctx, const double *antpos_e, const double *antpos_n,
                             const int *arm, const double *cal, const int *flagged,
                             double sfreq_mhz, double sep_arcmin, double dec_deg);
int dsax_beamform(dsax_ctx *ctx, const void *blk, void *out_u8, void *out_f32, int mem);

/* Automatic gain control of the uint8 beams (src/dsaX_beamformer.cu badder
 * :79-112, calc_allbp :482-494, ret_med_bp :506-513, ret_many_bp :515-530,
 * per-block update :1017-1062).  mode 1: adaptive (the default of the
 * reference), 2: frozen at the first block's median (-g), 0: off (fixed
 * bf_scale).  Enabling resets the state.  While on, every dsax_beamform
 * quantises u8 = rint(P * bp[beam]) / 2 (saturated) with bp from the
 * previous blocks (0 for the first block, whose beams are zero) and then
 * updates bp on the GPU from this block's per-beam power: median over beams
 * for the first 8 blocks, then the mean of the last 8 with beams more than
 * 10 % off the first median reset to it; bp = 2.5 * 128 / (power / (nchan/8
 * x npkt/16)). */
int dsax_agc_enable(dsax_ctx *ctx, int mode);
/* Current per-beam scale [nbeam] (may be NULL), state (0 before the first
 * block, 1 median phase, 2 history phase) and blocks seen; synchronises. */
int dsax_agc_state(dsax_ctx *ctx, float *scale, int *started, int *blocks);

/* ---- plain RFI flagger ----
 * Replaces src/gpu_flagger.cu: the statistics kernels (:175-494) and the
 * host decisions run per block (:1340-1398) -- channflag on spec-oldspec
 * (Thr), on var (Thr + 0.5), on max (Thr), simple_channflag on the
 * peak-to-peak of TBIN-sample means (Thr / sqrt(FBIN)), simple_tsflag on
 * the channel-mean time series (TsThr), all with lower medians (medval,
 * :534-556) and MADs -- on the GPU.  The shapes the reference hard-codes
 * are parameters here. */
typedef struct dsax_flag_params {
    int nbeam, ntime, nchan; /* filterbank [nbeam][ntime][nchan], 4 <= nchan <= 1024;
                                nchan a multiple of 4 (FP32) or 16 (uint8); uint8
                                ntime <= 262,144 (exact 32-bit partial sums)      */
    int guard;     /* ZeroChannels guard band at each edge (128 of 1024)           */
    int filt;      /* nFiltSize forward median window (21)                          */
    int tbin;      /* TBIN samples per peak-to-peak bin (128)                       */
    int fbin;      /* FBIN channels of the simple_channflag boxcar (8)              */
    int ts_base;   /* samples of the time-series median/MAD baseline (ntime/16)    */
    int tsflag;    /* 1: time-series flagging (-s)                                  */
    int parity;    /* 1: reproduce the reference as written: max spectrum = mean
                      spectrum (:1334) and the FBIN boxcar reads spec[j] (:594)     */
    float thresh;  /* Thr (-t, 5.0)                                                 */
    float var_add; /* variance threshold = Thr + var_add (0.5)                      */
    float ts_thresh; /* TsThr (-s, 10.0)                                            */
    int nperm;     /* permanent flag channels (flagchannels[], :95)                 */
    int perm[8];
} dsax_flag_params;

void dsax_default_flag_params(dsax_flag_params *p, int nbeam, int ntime, int nchan);

/* x: filterbank [nbeam][ntime][nchan] float32.  oldspec: previous block's
 * mean spectrum [nbeam][nchan] or NULL (zeros).  Outputs: chanmask
 * [nbeam][nchan] and tsmask [nbeam][ntime] (0/1 bytes); stats (optional)
 * [spec | var | max | pp] each [nbeam][nchan] then ts [nbeam][ntime];
 * counts (optional) = {flagged (beam, chan) columns, flagged (beam, t) rows}.
 * The time series is the channel mean after the flagged columns are set to
 * MN = 48 (the reference replaces them before make_ts, :1379-1386); x itself
 * is not modified.  ts_base <= 4096.
 * With DSAX_MEM_DEVICE every pointer is device memory. */
int dsax_flag(dsax_ctx *ctx, const dsax_flag_params *p, const float *x, const float *oldspec,
              uint8_t *chanmask, uint8_t *tsmask, float *stats, int *counts, int mem);

/* ---- plain flagger, data path ----
 * The per-block processing of src/gpu_flagger.cu's main loop (:1260-1487)
 * on a filterbank block that is cleaned in place: once a baseline exists,
 * scaley (:1296-1297) normalises the block with the baseline spectrum and
 * variance; the total-power modulation check (:1313-1330) replaces the whole
 * block with a fixed noise block when the summed spectrum changed by
 * mod_thresh or more since the previous flagged block; otherwise the
 * channel tests run, flagged columns are set to MN x bpwr[beam] (flag,
 * :459-474), the time series is formed from that data and flagged rows are
 * set to the same level inside the guard band (flagts, :479-494).  The first
 * naver blocks are only measured (no flagging, data unchanged): their
 * spectra and variances give the baseline by a per-(beam, channel) median
 * over the naver blocks (fix_zspec, :114-170) and then the median over
 * beams broadcast to every beam (median_calc, :771-798) -- the state that
 * the reference also reloads from specvar0.dat.
 * Deviations: the reference compares its first flagged block with a
 * pre-start noise block (:1276-1282), which in practice replaces it; here
 * the first flagged block has no previous total power and is not checked.
 * The noise block is a seeded Box-Muller block [ntime][nchan] (uniforms
 * from SplitMix64 quantised to 1/16384 as genrand does, :500-516, with u1 in
 * (0, 1] so that no sample is infinite), the same for every beam as in
 * :1323-1324. */
typedef struct dsax_flag_clean_params {
    float mn;           /* MN, replacement level (48)                                */
    float sig;          /* SIG, scaley target standard deviation (6)                 */
    float mod_thresh;   /* -q, total-power modulation threshold (0.0005)             */
    int naver;          /* blocks in the baseline median (5)                         */
    int scale;          /* 1: scaley once the baseline exists (the reference: always) */
    int pwr;            /* 1: level from this block's spectrum (calc_bpwr, -p); 0: 1  */
    int modcheck;       /* 1: total-power modulation check (the reference: always)   */
    unsigned long long seed; /* noise block                                         */
} dsax_flag_clean_params;

#define DSAX_DTYPE_F32 0
#define DSAX_DTYPE_U8 1

typedef struct dsax_flag_block_info {
    int blocks;          /* blocks processed by this state                             */
    int started;         /* 1 once the baseline exists (flagging on)                   */
    int flagged;         /* the last block went through the flagging branch            */
    int replaced;        /* the last block was replaced by noise (modulation check)    */
    int nchan_flagged;   /* flagged (beam, channel) columns of the last block          */
    int nts_flagged;     /* flagged (beam, time) rows of the last block                */
    double tpwr;         /* the last flagged block's total power (sum of spec)         */
    double prev_tpwr;    /* the total power it was compared with (0: none)             */
} dsax_flag_block_info;

typedef struct dsax_flag_state dsax_flag_state;

void dsax_default_flag_clean_params(dsax_flag_clean_params *cp);
/* A state for blocks of p's shape and element type dtype (DSAX_DTYPE_F32
 * or DSAX_DTYPE_U8) on the context's device; p and cp are copied. */
int dsax_flag_state_create(dsax_ctx *ctx, const dsax_flag_params *p,
                           const dsax_flag_clean_params *cp, int dtype, dsax_flag_state **st);
void dsax_flag_state_destroy(dsax_flag_state *st);
/* One block: data [nbeam][ntime][nchan] of the state's type, cleaned in
 * place; chanmask [nbeam][nchan], tsmask [nbeam][ntime] (0/1; NULL to skip
 * in host mode).  mem = DSAX_MEM_DEVICE enqueues on the context stream.
 * Calls on one state are serialised by the caller. */
int dsax_flag_clean(dsax_ctx *ctx, dsax_flag_state *st, void *data, uint8_t *chanmask,
                    uint8_t *tsmask, int mem);
/* Waits for the context stream and reports the last block. */
int dsax_flag_state_info(dsax_ctx *ctx, dsax_flag_state *st, dsax_flag_block_info *info);
/* The baseline spectrum and variance [nbeam][nchan] (host memory; either may
 * be NULL); get waits for the stream.  set loads a saved baseline and turns
 * flagging on (the reference's specvar0.dat, :1430-1441). */
int dsax_flag_state_get_baseline(dsax_ctx *ctx, dsax_flag_state *st, float *spec0, float *var0);
int dsax_flag_state_set_baseline(dsax_ctx *ctx, dsax_flag_state *st, const float *spec0,
                                 const float *var0);
/* The noise block [ntime][nchan] of the state's type (host memory). */
int dsax_flag_state_noise(dsax_ctx *ctx, dsax_flag_state *st, void *noise);

/* Allocation-free plain flagger.  No counterpart in the reference: it is for
 * callers that cannot call cudaMalloc -- a process whose device memory is
 * owned by another runtime's pool, a real-time thread that must not enter
 * the allocator, or code running while someone else records a CUDA graph.
 * Same computation and outputs as dsax_flag, without a context: it runs on
 * the current device and the given cudaStream_t (NULL = default stream),
 * and every pointer (x, oldspec, chanmask, tsmask, counts) is device memory.
 * The statistics use a fixed 6 MiB device array compiled into the library
 * (held on every GPU that loads it until the process exits), so
 * 4*nbeam*nchan + nbeam*ntime + 2*nbeam + 4 must not exceed 1,572,864 floats
 * (nchan <= 128, a multiple of 4; x 16-byte aligned); larger
 * sizes return DSAX_ERR_ARG.  The first call on a device looks up that
 * array's address; make it before any stream capture.  All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  Nothing is allocated or freed. */
int dsax_flag_noalloc(const dsax_flag_params *p, const float *x, const float *oldspec,
                      uint8_t *chanmask, uint8_t *tsmask, int *counts, void *stream);

/* ---- beam corner turn (beamformer -> search-side flagger) ----
 * The socket corner turn of src/dsaX_dbnic.c:84-152 and
 * src/dsaX_nicdb.c:180-196 as two device reorders around one all-to-all
 * (NCCL over NVLink; the caller's collective, e.g. torch.distributed).
 * dsax_ct_pack: this subband's beams [nt][nb][nc] (the beamformer's uint8
 *   output layout) -> send [ndest][nb/ndest][nt][nc], one contiguous chunk
 *   per destination (dbnic's per-search-node transpose).
 * dsax_ct_unpack: the chunks received from nsrc subbands,
 *   recv [nsrc][nbl][nt][nc] -> fil[nbl][t0 + t][ch0 + s nc + k] of a
 *   [nbl][fil_nt][fil_nc] uint8 filterbank (nicdb's placement; the
 *   reference uses fil_nc = 1024, ch0 = CHOFF/8 = 128, 16 subbands of 48
 *   channels, so the unfilled channels are the flagger's guard bands).
 * Device pointers; enqueued on the context stream. */
int dsax_ct_pack(dsax_ctx *ctx, const uint8_t *beams, int nt, int nb, int nc, int ndest,
                 uint8_t *send);
int dsax_ct_unpack(dsax_ctx *ctx, const uint8_t *recv, int nsrc, int nbl, int nt, int nc,
                   uint8_t *fil, int fil_nt, int fil_nc, int t0, int ch0);

/* ---- batches of blocks ----
 * Many consecutive capture blocks in one submission, each with its own
 * subband width (nchan, a multiple of 8, at most the nchan the context
 * and its weights were set up with).  Per block: corner turn + correlate
 * (if vis), beamform (if beams or chanmask), plain flagger on the block's
 * beam filterbank [nbeam][npkt/bf_pkt_per_out][nchan/8] (if chanmask; the
 * ts mask too if tsmask).  Device pointers only.  use_graph = 1 captures
 * the whole batch into a CUDA graph on the first call and replays it while
 * the descriptors stay the same.  Enqueued on the context stream. */
typedef struct dsax_block_desc {
    const void *blk;      /* captured block [npkt][nant_in][nchan][2][2]      */
    int nchan;            /* subband width of this block                       */
    float *vis;           /* [2*nchan][2080][4][re,im] or NULL                 */
    uint8_t *beams;       /* [npkt/ppo][nbeam][nchan/8] uint8 or NULL          */
    uint8_t *chanmask;    /* [nbeam][nchan/8] or NULL                          */
    uint8_t *tsmask;      /* [nbeam][npkt/ppo] or NULL                         */
} dsax_block_desc;

int dsax_run_batch(dsax_ctx *ctx, const dsax_block_desc *blocks, int nblk, int use_graph);

/* ---- learned RFI flagger (no reference counterpart) ----
 * A 4-layer 3x3 conv net (8 -> 32 -> 64 -> 64 -> 1 channels, ReLU,
 * 58,337 FP32 parameters) over the filterbank downsampled by tds samples,
 * with eight features per pixel (log-compressed z-scores of the pixel mean
 * and max, the row channel-mean, the max of the channel-mean series inside
 * the pixel, and the column mean, max, variance and peak-to-peak of
 * 128-sample means -- the statistics the plain flagger thresholds).  It is
 * trained on the
 * plain flagger's masks and predicts the pixel mask the plain flagger
 * applies: (chanmask[b][c]) or (tsmask in the pixel's samples and inside
 * the guard band).  The plain flagger (dsax_flag) stays the fallback and
 * the judge.  Parameter vector: for each layer W[co][3][3][ci] then b[co].
 * Filterbank, masks and feature pointers of dsax_lf_features and
 * dsax_lf_train_step are device memory. */
int dsax_lf_nparams(void);
int dsax_lf_init(dsax_ctx *ctx, unsigned long long seed);
int dsax_lf_set_params(dsax_ctx *ctx, const float *params, int n);
int dsax_lf_get_params(dsax_ctx *ctx, float *params, int n);
/* features [nbeam][ntime/tds][nchan][8] float32 */
int dsax_lf_features(dsax_ctx *ctx, const float *x, const dsax_flag_params *p, int tds, float *F);
/* One training step on p->nbeam beams: weighted BCE-with-logits (positive
 * pixels weighted by pos_weight, guard band excluded) on the plain
 * flagger's masks, then Adam (lr) if update != 0.  loss (host, optional):
 * mean loss; grads (host, optional): the flat gradient vector. */
int dsax_lf_train_step(dsax_ctx *ctx, const float *x, const uint8_t *chanmask,
                       const uint8_t *tsmask, const dsax_flag_params *p, int tds, float lr,
                       float pos_weight, int update, float *loss, float *grads);
/* Inference: mask [nbeam][ntime/tds][nchan] (0/1, guard band 0) and
 * optionally the logits (float32, same layout). */
int dsax_flag_learned(dsax_ctx *ctx, const float *x, const dsax_flag_params *p, int tds,
                      uint8_t *mask, float *logits, int mem);

#ifdef __cplusplus
}
#endif
#endif /* DSAX_H */

#!/usr/bin/env python
"""X-engine benchmark: full-size correlator blocks per second on B200.

Workload (one step = one block through the hot path): the full capture block
[2048 packets][63 antennas -> 64][384 channels][2 times][2 pols] of 4+4-bit
complex voltages (198,180,864 B), Gaussian sigma 2.5 quantised and clipped
to [-8, 7], correlated to the xGPU triangular visibilities
(768 freqs x 2080 baselines x 4 pol products, complex FP32, 51,118,080 B).

  value : blocks/s with the blocks already resident in HBM (device-timed with
          CUDA events on the library's stream, three resident blocks rotated
          so every step reads 198 MB that is not in the 126 MB L2).
  e2e   : the same metric through the public C-ABI call with host buffers
          (dsax_correlate, DSAX_MEM_HOST): pinned host block -> device,
          correlate, visibilities -> pinned host, every step.
  --impl reference : the reference path's CPU arithmetic (the oracle port of
          the xGPU CPU X-engine, all host threads) on a bounded sample.

Multi-GPU (torchrun, N > 1): blocks are independent, so every rank
correlates its own blocks (weak scaling, no collective on the data path);
the timed region is bracketed by a barrier and the max over ranks is used.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dsa110-xengine_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

REALTIME_S = 0.134217728          # one block of 4096 x 32.768 us samples
BLOCK_IN = 198_180_864
VIS_OUT = 51_118_080
ALG_OPS = 8 * 2080 * 4 * 768 * 2048   # one complex MAC = 8 integer ops
MMA_OPS = 2 * 128 * 256 * 4096 * 768  # executed tensor-core ops
METRIC = "X-engine blocks/s (full 198 MB block, bit-exact correlate)"
UNIT = "blocks/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_from_profiles(kernel: str):
    """Per-launch DRAM bytes of `kernel` from its committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_full_block.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    except Exception:
        pass
    return None


class ClockSampler:
    """SM clocks and clock-event reasons sampled DURING the timed region.

    NVML is read (never set) from a thread every ~2 ms, so even a timed
    region of a few milliseconds gets samples; nvidia-smi at 100 ms is the
    fallback when the NVML bindings are missing."""

    NAMES = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
             ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
             ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
             ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.smax = None
        self._stop = threading.Event()
        self._thr = None
        self._nv = None

    def _handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def _run(self, nv, h):
        bits = [(name, getattr(nv, const, 0)) for name, const in self.NAMES]
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, [n for n, b in bits if b and (r & b)]))
            except Exception:
                break
            time.sleep(0.002)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._nv = nv
            self._thr = threading.Thread(target=self._run, args=(nv, h), daemon=True)
            self._thr.start()
        except Exception:
            self._thr = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thr is not None:
            self._thr.join(timeout=5)
        if self._nv is not None:
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if self._thr is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no NVML"], "samples": 0}
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"], "samples": 0}
        sm = [r[0] for r in self.rows]
        reasons = sorted({n for r in self.rows for n in r[1]})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(self.rows), "source": "NVML, ~2 ms period"}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _has_avx512bw() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " avx512bw" in f.read()
    except Exception:
        return False


def _time_reorders(oracle, blk, nthr: int):
    """The reference's own CPU corner turns on one full block, from
    oracle/_ref (lifted from the reference tree): massage()
    (src/dsaX_reorder_raw.c:153-169, byte reorder) and the AVX-512 fluff +
    transpose (src/dsaX_reorder_raw.c.bak:184-258), at 1 and nthr threads.
    Returns {name: seconds per block} or {"unavailable": why}."""
    import ctypes
    try:
        ref = oracle.ref_lib()
    except Exception as exc:
        return {"unavailable": f"oracle/_ref: {type(exc).__name__}: {exc}"}
    src = np.ascontiguousarray(blk)
    out = {}
    nts = sorted({1, max(1, min(16, nthr))})
    for name, fn, nbytes in (("massage", ref.ref_massage_raw, 2048 * 768 * 64 * 2),
                             ("fluff_avx512", ref.ref_massage_bak, 2048 * 768 * 64 * 4)):
        if name == "fluff_avx512" and not _has_avx512bw():
            out[name] = "host CPU has no AVX-512BW"
            continue
        buf = np.zeros(nbytes, np.uint8)
        for nt in nts:
            while 2048 % nt:
                nt -= 1
            fn(src.ctypes.data_as(ctypes.c_void_p), buf.ctypes.data_as(ctypes.c_void_p), nt)
            t0 = time.perf_counter()
            fn(src.ctypes.data_as(ctypes.c_void_p), buf.ctypes.data_as(ctypes.c_void_p), nt)
            out[f"{name}_{nt}t_s"] = time.perf_counter() - t0
    return out


def run_reference(args):
    """The reference's CPU path for one full block on the host cores: its
    own massage() corner turn (oracle/_ref, all threads up to its 16-thread
    limit) plus the CPU X-engine of the oracle port (xGPU, whose CPU
    X-engine the reference calls xgpuOmpXengine, is not in the reference
    tree), every step a whole block unless --steps would take too long."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import ctypes
    import oracle
    oracle.build()
    nthr = oracle.nthreads()
    blk = oracle.gen_block(12345, 2048, 63, 384, "gauss")
    try:
        ref = oracle.ref_lib()
        mthr = max(1, min(16, nthr))
        while 2048 % mthr:
            mthr -= 1
        reo = np.zeros(2048 * 768 * 64 * 2, np.uint8)

        def massage():
            ref.ref_massage_raw(blk.ctypes.data_as(ctypes.c_void_p),
                                reo.ctypes.data_as(ctypes.c_void_p), mthr)
        kind = "reference"
    except Exception:
        massage, mthr = (lambda: oracle.massage(blk)), nthr
        kind = "port"
    t0 = time.perf_counter()
    massage()
    oracle.correlate(blk)
    full_s = time.perf_counter() - t0
    # a whole block per step when the run stays within ~3 minutes, else a
    # channel sample of the X-engine per step, scaled to a block
    nch = 384 if (args.steps + 1) * full_s <= 180 else \
        max(8, int(384 * 180 / ((args.steps + 1) * full_s)))
    for _ in range(max(0, min(args.warmup, 1))):
        massage()
        oracle.correlate(blk, ch0=0, nch=nch)
    times = []
    for s in range(args.steps):
        ch0 = (s * nch) % (384 - nch + 1)
        t0 = time.perf_counter()
        massage()
        t1 = time.perf_counter()
        oracle.correlate(blk, ch0=ch0, nch=nch)
        t2 = time.perf_counter()
        times.append((t1 - t0) + (t2 - t1) * 384.0 / nch)
    per_block = statistics.mean(times)
    v = 1.0 / per_block
    sample = ("one full block per step" if nch == 384 else
              f"massage on the full block + X-engine on {nch} of 384 channels per step, scaled")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_block * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic seeded Gaussian sigma 2.5, 4+4-bit",
        "config": {"workload": "full-size correlator block [2048][63][384][2][2] -> 768x2080x4 vis",
                   "sample": sample},
        "same_config": nch == 384,
        "realtime_factor": v * REALTIME_S,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthr, "kind": kind,
                         "sample": sample,
                         "parts": f"massage() from the reference source ({mthr} threads) + "
                                  f"oracle X-engine ({nthr} threads)"},
        "reorders_s_per_block": _time_reorders(oracle, blk, nthr),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's X-engine is the un-vendored xGPU library; its CPU arithmetic "
                "is the oracle port (OpenMP); the corner turn is the reference's own code",
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(budget_s: float = 12.0):
    """Oracle X-engine on the host cores over a bounded channel sample."""
    import oracle
    oracle.build()
    blk = oracle.gen_block(777, 2048, 63, 384, "gauss")
    nch, done, t_total = 4, 0, 0.0
    oracle.correlate(blk, ch0=0, nch=1)
    while t_total < budget_s and done + nch <= 384:
        t0 = time.perf_counter()
        oracle.correlate(blk, ch0=done, nch=nch)
        t_total += time.perf_counter() - t0
        done += nch
    per_block = t_total * 384.0 / done
    return {"value": 1.0 / per_block, "unit": UNIT, "cores": oracle.nthreads(), "kind": "port",
            "sample": f"{done} of 384 channels of one full block ({t_total:.1f} s), scaled"}


BF_FLOPS = 8 * 256 * 64 * 2 * 384 * 4096      # 256-beam beamformer, FLOP per full block


def _bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured"
    except Exception:
        return 1590.0, 1400.0, "fallback"


def _time_loop(stream, fn, steps, warm=3):
    import torch
    for i in range(warm):
        fn(i)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        fn(i)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_beamformer(dsax, synth, dev, blk_dev, steps, peaks=None):
    """Beamformer workload: 256 beams, 32 t x 8 ch Stokes-I from a full block
    (BF16, and FP8 E4M3): device-timed, end to end with host buffers, error
    of every output of two channel groups against the FP64 oracle, and the
    oracle's FP64 beamformer on the host cores as the CPU baseline."""
    import ctypes
    import torch
    import oracle
    scale = 128.0 / (512 * 64 * 2 * 6.25)
    cfg = dsax.default_config(bf_scale=scale)
    wre, wim = synth.random_phase_weights(9, 48, 256)
    blk_host = synth.gen_block(4242, 2048, 63, 384, "gauss")
    nout = 128 * 256 * 48
    with dsax.Context(cfg, device=dev) as ctx:
        ctx.set_weights(wre, wim)
        out = torch.empty(nout, dtype=torch.uint8, device=f"cuda:{dev}")
        f32 = torch.empty(nout, dtype=torch.float32, device=f"cuda:{dev}")
        st = torch.cuda.ExternalStream(ctx.stream)
        ms = _time_loop(st, lambda i: ctx.beamform(blk_dev[i % len(blk_dev)], out), steps)
        # error against FP64 on two channel groups of the first block
        ctx.beamform(blk_dev[0], out, f32)
        ctx.sync()
        got = f32.cpu().numpy().reshape(128, 256, 48).astype(np.float64)
        gu8 = out.cpu().numpy().reshape(128, 256, 48)
        # end to end: pinned host block in, uint8 beams out, every step
        lib = dsax.lib()
        p_in, p_out = ctypes.c_void_p(), ctypes.c_void_p()
        assert lib.dsax_host_alloc(ctx.handle, BLOCK_IN, ctypes.byref(p_in)) == 0
        assert lib.dsax_host_alloc(ctx.handle, nout, ctypes.byref(p_out)) == 0
        ctypes.memmove(p_in.value, blk_host.ctypes.data, BLOCK_IN)
        for _ in range(2):
            ctx.beamform(p_in.value, p_out.value, None, dsax.MEM_HOST)
        e_steps = 10
        t0 = time.perf_counter()
        for _ in range(e_steps):
            ctx.beamform(p_in.value, p_out.value, None, dsax.MEM_HOST)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / e_steps
        lib.dsax_host_free(ctx.handle, p_in)
        lib.dsax_host_free(ctx.handle, p_out)
    # the autotuner's candidates on this GPU: the one-CTA form and the CTA
    # pairs with each stage-parameter variant
    with dsax.Context(dsax.default_config(bf_scale=scale), device=dev) as ctx:
        ctx.set_weights(wre, wim)
        tune_ms, tune_best = ctx.autotune_beamformer(reps=5)
    # the one-CTA-per-beam-tile form (bf_path 1), for comparison with the
    # default CTA pairs
    cfg1 = dsax.default_config(bf_scale=scale, bf_path=1)
    with dsax.Context(cfg1, device=dev) as ctx:
        ctx.set_weights(wre, wim)
        st = torch.cuda.ExternalStream(ctx.stream)
        ms1 = _time_loop(st, lambda i: ctx.beamform(blk_dev[i % len(blk_dev)], out), steps)
        ctx.sync()
    # the FP8 E4M3 operands (per-antenna power-of-two weight scale)
    cfg8 = dsax.default_config(bf_scale=scale, bf_fp8=1)
    with dsax.Context(cfg8, device=dev) as ctx:
        ctx.set_weights(wre, wim)
        st = torch.cuda.ExternalStream(ctx.stream)
        ms8 = _time_loop(st, lambda i: ctx.beamform(blk_dev[i % len(blk_dev)], out), steps)
        ctx.beamform(blk_dev[0], out, f32)
        ctx.sync()
        got8 = f32.cpu().numpy().reshape(128, 256, 48).astype(np.float64)
        gu8_8 = out.cpu().numpy().reshape(128, 256, 48)
    # per-output error on groups 0 and 47 against the FP64 oracle (unrounded
    # weights) on the same block, for the BF16 and the FP8 operands
    blk0 = blk_dev[0].cpu().numpy().reshape(2048, 63, 384, 2, 2)
    refs = {g: oracle.beamform_power(blk0, wre, wim, 16, g0=g, ng=1)[:, :, 0] for g in (0, 47)}

    def _err(gp, gu):
        rel_all, lsb_all = [], []
        for g, ref in refs.items():
            rel = np.abs(gp[:, :, g] - ref) / np.maximum(ref, 1e-30)
            lsb = np.abs(gu[:, :, g].astype(int) - oracle.quantize_u8(ref, scale).astype(int))
            rel_all.append(rel.reshape(-1))
            lsb_all.append(lsb.reshape(-1))
        rel_all = np.concatenate(rel_all)
        lsb_all = np.concatenate(lsb_all)
        return {"outputs_checked": int(rel_all.size), "groups": [0, 47],
                "fp32_rel_max": float(rel_all.max()), "fp32_rel_mean": float(rel_all.mean()),
                "u8_max_lsb": int(lsb_all.max()),
                "u8_frac_off_by_1": float((lsb_all == 1).mean())}
    err = _err(got, gu8)
    err8 = _err(got8, gu8_8)
    # CPU baseline: the oracle's FP64 beamformer on the host cores, a sample
    # of channel groups scaled to the block
    t0 = time.perf_counter()
    ng = 0
    while ng < 48 and time.perf_counter() - t0 < 8.0:
        oracle.beamform_power(blk_host, wre, wim, 16, g0=ng, ng=2)
        ng += 2
    cpu_s = (time.perf_counter() - t0) * 48.0 / ng
    burst, sust, kind = _bf16_peak()
    tf = BF_FLOPS / (ms * 1e-3) / 1e12
    tf8 = BF_FLOPS / (ms8 * 1e-3) / 1e12
    fp8_peak = (peaks or {}).get("fp8_tops")
    res = {"workload": "64 ant x 2 pol x 384 ch x 4096 t -> 128 x 256 x 48 uint8, 256 beams, BF16",
           "blocks_per_s": 1e3 / ms, "ms_per_block": ms, "realtime_factor": 1e3 / ms * REALTIME_S,
           "gpu_launches_per_block": 1,
           "kernel_form": "CTA pairs: two 64-beam tiles share each data stage through one "
                          "tcgen05.mma.cta_group::2 (M = 256)",
           "one_cta_form": {"ms_per_block": ms1, "achieved_tflops": BF_FLOPS / (ms1 * 1e-3) / 1e12,
                            "kernel": "bf_kernel (bf_path 1)"},
           "autotune": {"candidates_ms": {("one CTA" if k == 1 else f"pairs, variant {k - 1}"): v
                                          for k, v in tune_ms.items()},
                        "chosen": "one CTA" if tune_best == 1 else f"pairs, variant {tune_best - 1}",
                        "call": "dsax_autotune_beamformer (BF16)"},
           "roofline": {"bound": "tensor", "kernel": "bf_pair_kernel", "achieved": tf,
                        "peak": burst, "unit": "TFLOP/s", "frac": tf / burst,
                        "frac_of_sustained": tf / sust, "peak_kind": f"{kind} BF16 dense (cuBLAS)"},
           "error_vs_fp64": err,
           "e2e": {"value": 1e3 / e2e_ms, "unit": "blocks/s", "ms_per_step": e2e_ms,
                   "h2d_bytes_per_step": BLOCK_IN, "d2h_bytes_per_step": nout,
                   "call": "dsax_beamform, DSAX_MEM_HOST (pinned)"},
           "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "blocks/s", "kind": "port",
                            "cores": oracle.nthreads(),
                            "sample": f"FP64 oracle beamformer on {ng} of 48 channel groups of one "
                                      f"block, scaled"},
           "fp8": {"ms_per_block": ms8, "blocks_per_s": 1e3 / ms8, "achieved_tflops": tf8,
                   "frac_of_2x_bf16_peak": tf8 / (2 * burst),
                   "peak_kind": "E4M3 dense taken as 2x the measured BF16 burst",
                   "error_vs_fp64": err8}}
    if fp8_peak:
        res["fp8"]["frac_of_probe"] = tf8 / fp8_peak
        res["fp8"]["probe_tflops"] = fp8_peak
    return res


def bench_flaggers(dsax, synth, dev, steps, train_steps=2000):
    """Flagger workload: plain vs learned flagger on [256][4096][48] FP32
    (chi2(2) + RFI), plus the plain flagger's data path (dsax_flag_clean) on
    that block and on a reference-shaped uint8 block [64][16384][1024].
    The learned net is trained here first (outside the timed regions)."""
    import torch
    import oracle
    from dsax import lflag
    x, _ = synth.gen_filterbank(4040)
    xd = torch.from_numpy(x).to(f"cuda:{dev}")
    B, T, C = x.shape
    tds = 32
    p = dsax.flag_params(B, T, C)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8), device=dev) as ctx:
        st = torch.cuda.ExternalStream(ctx.stream)
        cm = torch.zeros(B * C, dtype=torch.uint8, device=xd.device)
        tm = torch.zeros(B * T, dtype=torch.uint8, device=xd.device)
        plain_ms = _time_loop(st, lambda i: ctx.flag(p, xd, cm, tm), steps)
        # the data path: measured blocks build the baseline (naver = 1), then
        # flagged + cleaned blocks in place (the modulation check on)
        clean = {}
        for name, arr, dt, fp in (
                ("fp32_256x4096x48", x, dsax.DTYPE_F32, p),
                ("u8_64x16384x1024", None, dsax.DTYPE_U8,
                 dsax.flag_params(64, 16384, 1024, guard=128, ts_base=1024))):
            if arr is None:
                g = torch.Generator(device=xd.device)
                g.manual_seed(9)
                d = torch.randint(40, 80, (64 * 16384 * 1024,), dtype=torch.uint8,
                                  device=xd.device, generator=g)
            else:
                d = torch.from_numpy(arr.copy()).to(xd.device).reshape(-1)
            fs = ctx.flag_state(fp, dsax.flag_clean_params(naver=1, mod_thresh=1.0), dt)
            fs.clean(d)
            nbytes = d.numel() * d.element_size()
            cms = _time_loop(st, lambda i: fs.clean(d), steps)
            inf = fs.info()
            fs.close()
            clean[name] = {"ms_per_block": cms, "gbytes_per_s": nbytes / (cms * 1e-3) / 1e9,
                           "block_bytes": nbytes, "flagged": bool(inf.flagged),
                           "gpu_launches_per_block": 4}
            del d
        train = [torch.from_numpy(synth.gen_filterbank(5000 + k, nbeam=64)[0]).to(xd.device)
                 for k in range(4)]
        ctx.lf_init(11)
        t0 = time.perf_counter()
        lflag.train(ctx, train, steps=train_steps, beams_per_step=16, tds=tds)
        ctx.sync()
        train_s = time.perf_counter() - t0
        mask = torch.zeros(B * (T // tds) * C, dtype=torch.uint8, device=xd.device)
        learned_ms = _time_loop(st, lambda i: ctx.flag_learned(p, xd, mask, tds=tds), steps)
        ctx.sync()
        pred, ref = lflag.evaluate(ctx, xd, tds)
    P, R, F1 = lflag.prf1(pred, ref)
    npx = B * T * C
    peak, peak_kind = _peaks()
    alg = npx * 4 + B * C + B * T          # filterbank read once, masks written
    # CPU baseline: the oracle's plain flagger (statistics + decisions) on a
    # sample of beams, scaled to the block
    nb = 32
    po = oracle.flag_params(nb, T, C)
    xs = np.ascontiguousarray(x[:nb])
    oracle.plain_flag(xs, po)
    t0 = time.perf_counter()
    reps = 0
    while reps < 20 and (reps == 0 or time.perf_counter() - t0 < 6.0):
        oracle.plain_flag(xs, po)
        reps += 1
    cpu_s = (time.perf_counter() - t0) / reps * B / nb
    return {"workload": "256 beams x 4096 t x 48 ch FP32 chi2(2) + tones/bursts/drifts",
            "plain": {"ms_per_block": plain_ms, "samples_per_s": npx / (plain_ms * 1e-3),
                      "gpu_launches_per_block": 4,
                      "roofline": {"bound": "hbm", "kernel": "plain flagger (4 launches)",
                                   "achieved": alg / (plain_ms * 1e-3) / 1e9, "peak": peak,
                                   "unit": "GB/s", "frac": alg / (plain_ms * 1e-3) / 1e9 / peak,
                                   "alg_bytes_per_block": alg,
                                   "peak_kind": f"{peak_kind} (HBM copy bandwidth)"},
                      "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "blocks/s", "kind": "port",
                                       "cores": oracle.nthreads(),
                                       "sample": f"oracle plain flagger on {nb} of {B} beams, "
                                                 f"scaled"}},
            "clean": clean,
            "learned": {"ms_per_block": learned_ms, "samples_per_s": npx / (learned_ms * 1e-3),
                        "precision": P, "recall": R, "f1": F1, "train_s": train_s,
                        "train_steps": train_steps, "params": dsax.lib().dsax_lf_nparams(),
                        "gpu_launches_per_block": 9},
            "learned_vs_plain_speed": plain_ms / learned_ms}


def bench_config1(dsax, synth, dev, steps):
    """The small correlator case: 64 antennas x 48 channels x 2048 packets,
    samples uniform on [-8, 7] (bit-exact in the tests), device-timed."""
    import torch
    blk = synth.gen_block(101, 2048, 64, 48, "uniform")
    cfg = dsax.default_config(npkt=2048, nant_in=64, nchan=48)
    with dsax.Context(cfg, device=dev) as ctx:
        d = torch.from_numpy(blk.reshape(-1)).to(f"cuda:{dev}")
        vis = torch.empty(96 * 2080 * 8, dtype=torch.float32, device=f"cuda:{dev}")
        st = torch.cuda.ExternalStream(ctx.stream)
        ms = _time_loop(st, lambda i: ctx.correlate(d, vis), steps)
        ctx.sync()
    ops = 8 * 2080 * 4 * 96 * 2048
    return {"workload": "64 ant x 48 ch x 2048 pkt x 2 t, uniform [-8, 7] -> 96 x 2080 x 4 vis",
            "blocks_per_s": 1e3 / ms, "ms_per_block": ms,
            "int8_alg_tops": ops / (ms * 1e-3) / 1e12, "gpu_launches_per_block": 2,
            "note": "L2-resident (25 MB input); latency-bound at this size"}


def bench_batch(dsax, synth, dev, steps):
    """Batch workload: 16 blocks, widths from {192, 384, 768}, corner turn +
    correlate + beamform + flag each, one CUDA graph vs per-block launches."""
    import torch
    rng = np.random.default_rng(55)
    widths = [int(w) for w in rng.choice([192, 384, 768], size=16)]
    cfg = dsax.default_config(nchan=768, bf_scale=128.0 / (512 * 64 * 2 * 6.25))
    base = synth.gen_block(5150, 2048, 63, 768, "gauss")
    with dsax.Context(cfg, device=dev) as ctx:
        wre, wim = synth.random_phase_weights(5, 96, 256)
        ctx.set_weights(wre, wim)
        descs = []
        for k, w in enumerate(widths):
            blk = np.ascontiguousarray(base[:, :, (7 * k) % (768 - w + 1):][:, :, :w])
            descs.append({"blk": torch.from_numpy(blk.reshape(-1)).to(f"cuda:{dev}"), "nchan": w,
                          "vis": torch.empty(2 * w * 2080 * 8, dtype=torch.float32, device=f"cuda:{dev}"),
                          "beams": torch.empty(128 * 256 * (w // 8), dtype=torch.uint8, device=f"cuda:{dev}"),
                          "chanmask": torch.empty(256 * (w // 8), dtype=torch.uint8, device=f"cuda:{dev}"),
                          "tsmask": torch.empty(256 * 128, dtype=torch.uint8, device=f"cuda:{dev}")})
        st = torch.cuda.ExternalStream(ctx.stream)
        graph_ms = _time_loop(st, lambda i: ctx.run_batch(descs, use_graph=True), steps)
        eager_ms = _time_loop(st, lambda i: ctx.run_batch(descs, use_graph=False), steps)
        ctx.sync()
    # the same batch with the one-CTA-per-beam-tile beamformer (bf_path 1)
    cfg1 = dsax.default_config(nchan=768, bf_scale=128.0 / (512 * 64 * 2 * 6.25), bf_path=1)
    with dsax.Context(cfg1, device=dev) as ctx:
        ctx.set_weights(wre, wim)
        st = torch.cuda.ExternalStream(ctx.stream)
        graph1_ms = _time_loop(st, lambda i: ctx.run_batch(descs, use_graph=True), steps)
        ctx.sync()
    nb = len(widths)
    # work of the batch, and its rate over the whole batch time (the stages
    # share that time on two streams, so these are lower bounds per stage)
    bf_flop = BF_FLOPS * sum(widths) / 384.0
    corr_bytes = sum(2048 * 63 * w * 4 + 2 * w * 2080 * 8 for w in widths)
    burst, _, kind = _bf16_peak()
    hbm = _peaks()[0]
    return {"workload": "16 blocks x 2048 pkt x 63 ant, widths " + ",".join(map(str, widths)),
            "widths": widths,
            "graph": {"blocks_per_s": nb * 1e3 / graph_ms, "ms_per_batch": graph_ms},
            "per_block_launches": {"blocks_per_s": nb * 1e3 / eager_ms, "ms_per_batch": eager_ms},
            "graph_one_cta_beamformer": {"blocks_per_s": nb * 1e3 / graph1_ms,
                                         "ms_per_batch": graph1_ms},
            "realtime_factor_graph": nb * 1e3 / graph_ms * REALTIME_S * 384.0 / np.mean(widths),
            "over_batch_time": {
                "beamformer_tflops": bf_flop / (graph_ms * 1e-3) / 1e12,
                "beamformer_frac_of_bf16_burst": bf_flop / (graph_ms * 1e-3) / 1e12 / burst,
                "correlation_alg_gbs": corr_bytes / (graph_ms * 1e-3) / 1e9,
                "correlation_frac_of_hbm": corr_bytes / (graph_ms * 1e-3) / 1e9 / hbm,
                "note": "each stage's work over the whole batch time (lower bounds): the "
                        "beamformer takes about 60 % of it, the correlation chain 30 %"},
            "gpu_launches_per_batch": 5 * nb}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="dsax", choices=["dsax", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=60)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", choices=["beamformer", "flagger", "batch", "config1"], default=None,
                    help="run one side workload alone (profiling); prints its JSON")
    ap.add_argument("--serial", action="store_true",
                    help="one dsax_correlate call per block (no cross-block overlap)")
    ap.add_argument("--lf-train-steps", type=int, default=2000,
                    help="training steps of the learned flagger before it is timed")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the beamformer / flagger / batch side measurements")
    ap.add_argument("--corr-path", type=int, default=0,
                    help="0 default (=4), 1 fused kernel, 2 REORDER-layout corner turn, "
                         "3 channel-major corner turn + directly fed correlator, "
                         "4 the same, bulk-copy fed, 5 as 4 with 16 unpack warps, "
                         "6 captured block read directly by 4-CTA clusters, 7 as 6 with 16 unpack warps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch

    import dsax

    ws, rank, local = _dist()
    if args.only:
        from dsax import synth
        torch.cuda.set_device(local)
        ins = None
        if args.only == "beamformer":
            blk = synth.gen_block(4242, 2048, 63, 384, "gauss")
            ins = [torch.from_numpy(blk.reshape(-1)).to(f"cuda:{local}")]
            res = bench_beamformer(dsax, synth, local, ins, args.steps)
        elif args.only == "config1":
            res = bench_config1(dsax, synth, local, args.steps)
        elif args.only == "flagger":
            res = bench_flaggers(dsax, synth, local, args.steps, args.lf_train_steps)
        else:
            res = bench_batch(dsax, synth, local, args.steps)
        print(json.dumps({"only": args.only, **res}), flush=True)
        return 0
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)

    from dsax import synth
    blk = synth.gen_block(4242 + rank, 2048, 63, 384, "gauss")
    cfg = dsax.default_config(corr_path=args.corr_path)
    ctx = dsax.Context(cfg, device=dev)
    nbuf = 3
    d_in0 = torch.from_numpy(blk.reshape(-1)).to(f"cuda:{dev}")
    ins = [d_in0] + [torch.roll(d_in0.view(2048, -1), shifts=97 * (k + 1), dims=0).reshape(-1)
                     for k in range(nbuf - 1)]
    vis = torch.empty(VIS_OUT // 4, dtype=torch.float32, device=f"cuda:{dev}")
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)

    for w in range(args.warmup):
        ctx.correlate(ins[w % nbuf], vis)
    ctx.sync()

    # measured tensor-pipe peaks of this GPU (the pool measures HBM and
    # cuBLAS BF16 only): int8, BF16 and FP8 E4M3 tcgen05.mma from shared memory
    probes = {}
    if rank == 0:
        for kname, kind in (("int8_tops", 0), ("bf16_tflops", 1), ("fp8_tops", 2)):
            try:
                probes[kname] = ctx.probe_tensor_peak(kind, 3) / 1e12
            except Exception as exc:
                probes[kname] = None
                probes[kname + "_error"] = str(exc)

    # ---------------------------------------------------------- device-timed
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # The K blocks through one dsax_correlate_many call: each block's corner
    # turn runs on a side stream beside the previous block's (persistent)
    # correlation.  --serial: one dsax_correlate call per block (corner turn
    # then correlate on the library stream), also timed below as
    # serial_ms_per_step.  The end-to-end leg uses dsax_correlate_many with
    # host buffers, which also overlaps the PCIe copies.
    pipelined = cfg.corr_path in (0, 3, 4, 5, 6, 7) and not args.serial
    step_blocks = [ins[s % nbuf] for s in range(args.steps)]
    if pipelined:
        ctx.correlate_many(step_blocks[:min(args.steps, 4)], [vis] * min(args.steps, 4))
        ctx.sync()
        torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        if pipelined:
            ctx.correlate_many(step_blocks, [vis] * args.steps)
        else:
            for s in range(args.steps):
                ctx.correlate(ins[s % nbuf], vis)
        ev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    # one call per block, for comparison
    serial_ms = None
    if pipelined:
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for s in range(args.steps):
            ctx.correlate(ins[s % nbuf], vis)
        s1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
        serial_ms = s0.elapsed_time(s1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_per_step = ms / args.steps
    value = ws * 1e3 / ms_per_step
    clocks = clk.summary()

    # ---------------------------------------------------------- per kernel
    # The same work split into its two launches, timed separately on the
    # library stream: the corner turn (captured -> REORDER layout) and the
    # tcgen05 correlator on the corner-turned block.
    kernel_ms = {}
    if cfg.corr_path != 1:
        reo = torch.empty(2048 * 768 * 64 * 2, dtype=torch.uint8, device=f"cuda:{dev}")
        tfmt = dsax.FMT_REORDERED if cfg.corr_path == 2 else dsax.FMT_CHANMAJOR
        names = (("reorder_kernel", "corr_kernel") if cfg.corr_path == 2
                 else ("reorder_cm_kernel", "corr_cm_kernel"))
        for name, fn in ((names[0], lambda s: ctx.corner_turn(ins[s % nbuf], reo, tfmt)),
                         (names[1], lambda s: ctx.correlate(reo, vis, fmt=tfmt))):
            for s in range(3):
                fn(s)
            ctx.sync()
            k0 = torch.cuda.Event(enable_timing=True)
            k1 = torch.cuda.Event(enable_timing=True)
            k0.record(stream)
            for s in range(args.steps):
                fn(s)
            k1.record(stream)
            ctx.sync()
            torch.cuda.synchronize()
            kernel_ms[name] = k0.elapsed_time(k1) / args.steps
        del reo
    else:
        kernel_ms["corr_kernel"] = ms_per_step

    # ---------------------------------------------------------- end to end
    h_in = ctx_host = None
    e2e_steps = max(3, args.e2e_steps)
    import ctypes
    p_in, p_vis = ctypes.c_void_p(), ctypes.c_void_p()
    lib = dsax.lib()
    assert lib.dsax_host_alloc(ctx.handle, BLOCK_IN, ctypes.byref(p_in)) == 0
    assert lib.dsax_host_alloc(ctx.handle, VIS_OUT, ctypes.byref(p_vis)) == 0
    ctypes.memmove(p_in.value, blk.ctypes.data, BLOCK_IN)
    for _ in range(3):
        ctx.correlate(p_in.value, p_vis.value, dsax.MEM_HOST)
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if pipelined:
        ctx.correlate_many([p_in.value] * 3, [p_vis.value] * 3, dsax.MEM_HOST)
    e0.record(stream)
    if pipelined:
        # host buffers in and out through the pipelined call: PCIe copies in,
        # out and the device work of consecutive blocks overlap
        ctx.correlate_many([p_in.value] * e2e_steps, [p_vis.value] * e2e_steps, dsax.MEM_HOST)
    else:
        for _ in range(e2e_steps):
            ctx.correlate(p_in.value, p_vis.value, dsax.MEM_HOST)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms_e2e], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = ws * 1e3 * e2e_steps / ms_e2e
    # spot-check the e2e output against the device result of the same block
    host_vis = np.ctypeslib.as_array((ctypes.c_float * (VIS_OUT // 4)).from_address(p_vis.value))
    ctx.correlate(ins[0], vis)
    ctx.sync()
    assert np.array_equal(host_vis, vis.cpu().numpy()), "e2e output differs from device output"
    lib.dsax_host_free(ctx.handle, p_in)
    lib.dsax_host_free(ctx.handle, p_vis)

    if rank == 0:
        peak, peak_kind = _peaks()
        # dominant kernel of the step and its algorithmic bytes per launch
        dom = max(kernel_ms, key=kernel_ms.get)
        corr_ms = [v for k, v in kernel_ms.items() if k.startswith("corr")][0]
        dom_ms = kernel_ms[dom]
        reo_bytes = 2048 * 768 * 64 * 2
        if dom.startswith("reorder"):
            alg = BLOCK_IN + reo_bytes
        elif cfg.corr_path != 1:
            alg = reo_bytes + VIS_OUT
        else:
            alg = BLOCK_IN + VIS_OUT
        achieved = alg / (dom_ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8 in / int32 accumulate (tcgen05 kind::i8)",
            "data": "synthetic seeded Gaussian sigma 2.5 quantised to 4+4-bit",
            "config": {"workload": "full-size correlator block [2048][63->64][384][2][2] "
                                   "-> xGPU triangular 768x2080x4 complex FP32",
                       "block_bytes": BLOCK_IN, "vis_bytes": VIS_OUT,
                       "corr_path": ["channel-major corner turn + bulk-fed correlate", "fused",
                                     "REORDER-layout corner turn + correlate",
                                     "channel-major corner turn + directly fed correlate",
                                     "channel-major corner turn + bulk-fed correlate",
                                     "channel-major corner turn + bulk-fed correlate, 16 unpack warps",
                                     "captured block read directly (4-CTA clusters, no corner turn)",
                                     "captured block read directly (4-CTA clusters), 16 unpack warps"
                                     ][cfg.corr_path],
                       "l2": "inputs larger than L2: 3 resident 198 MB blocks rotated",
                       "step": ("K blocks in one dsax_correlate_many call (each corner turn on a "
                                "side stream beside the previous block's correlation)"
                                if pipelined else "one dsax_correlate call per block"),
                       "parallelism": f"blocks independent per GPU x{ws}"},
            "realtime_factor": value / ws * REALTIME_S,
            "e2e_pipelined": pipelined,
            "pipelined": pipelined,
            "serial_ms_per_step": serial_ms,
            "gpu_launches": args.steps * (1 if cfg.corr_path == 1 else 2),
            "kernel_ms": kernel_ms,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": _traffic_from_profiles(dom),
                         "peak_kind": f"{peak_kind} (HBM copy bandwidth)",
                         "alg_bytes_per_launch": alg,
                         "int8_alg_tops": ALG_OPS / (corr_ms * 1e-3) / 1e12,
                         "int8_mma_tops": MMA_OPS / (corr_ms * 1e-3) / 1e12,
                         "int8_peak_probe_tops": probes.get("int8_tops"),
                         "int8_alg_frac_of_probe": (ALG_OPS / (corr_ms * 1e-3) / 1e12 /
                                                    probes["int8_tops"]
                                                    if probes.get("int8_tops") else None),
                         "int8_mma_frac_of_probe": (MMA_OPS / (corr_ms * 1e-3) / 1e12 /
                                                    probes["int8_tops"]
                                                    if probes.get("int8_tops") else None)},
            "tensor_peaks_probe": dict(probes, how="dsax_probe_tensor_peak: every SM issues "
                                       "back-to-back tcgen05.mma M128 N256 from shared memory "
                                       "(builder-measured, not the pool's peak file)"),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": BLOCK_IN,
                    "d2h_bytes_per_step": VIS_OUT, "steps": e2e_steps,
                    "ms_per_step": ms_e2e / e2e_steps},
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and ws == 1:
            line["cpu_baseline"] = cpu_baseline_sample()
        if not args.no_extras and ws == 1:
            for key, fn in (("config1", lambda: bench_config1(dsax, synth, dev, 50)),
                            ("beamformer", lambda: bench_beamformer(dsax, synth, dev, ins, 20,
                                                                    probes)),
                            ("flagger", lambda: bench_flaggers(dsax, synth, dev, 20,
                                                               args.lf_train_steps)),
                            ("batch", lambda: bench_batch(dsax, synth, dev, 5))):
                try:
                    line[key] = fn()
                except Exception as exc:  # reported, never silently dropped
                    line[key] = {"error": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

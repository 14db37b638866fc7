"""ctypes wrapper around oracle/liboracle.so -- the CPU restatement of the
DSA-110 X-engine hot path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker; the product path
(libdsax.so and its C-ABI) never loads it.

Each function cites the reference code it restates; the C source carries
the details.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

# Seeded input generators live with the package (they are not part of the
# oracle); re-exported here for the tests.
from dsax.synth import gen_block, gen_filterbank, random_phase_weights  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

NST = 64
NBL = NST * (NST + 1) // 2  # 2080 baselines


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    srcs = [os.path.join(_HERE, f) for f in ("dsax_oracle.c", "dsax_oracle_flag.c")]
    if force or not os.path.exists(_LIB_PATH) or any(
            os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in srcs):
        subprocess.check_call(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i32, i64, f32, f64 = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double
        L.oracle_promote.argtypes = [P, P, i64]
        L.oracle_massage.argtypes = [P, P, i32, i32, i32]
        L.oracle_fluff_reorder.argtypes = [P, P, i32, i32, i32]
        L.oracle_correlate.argtypes = [P, i32, i32, i32, i32, i32, P]
        L.oracle_correlate.restype = i32
        L.oracle_xengine_int8.argtypes = [P, i32, i32, P]
        L.oracle_xengine_int8.restype = i32
        L.oracle_simple_extract.argtypes = [P, i32, P]
        L.oracle_beamform.argtypes = [P, i32, i32, i32, P, P, i32, i32, i32, i32, P]
        L.oracle_beamform.restype = i32
        L.oracle_geometric_weights.argtypes = [P, P, P, i32, i32, f64, f64, P, P]
        L.oracle_plain_flag.argtypes = [P, P, P, P, P, P, P, P]
        L.oracle_plain_flag.restype = i32
        L.oracle_nthreads.restype = i32
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def nthreads() -> int:
    return int(lib().oracle_nthreads())


# --------------------------------------------------------------------------
# seeded synthetic capture blocks
# --------------------------------------------------------------------------
def pack4(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    """4+4-bit two's complement byte: real in the low nibble, imag in the
    high nibble (src/dsaX_xgpu.cu:74-75, utils/gen_packet.py:137-147)."""
    return ((re.astype(np.int16) & 0xF) | ((im.astype(np.int16) & 0xF) << 4)).astype(np.uint8)


def unpack4(b: np.ndarray):
    b = b.astype(np.int16)
    re = ((b & 0xF) ^ 0x8) - 8
    im = (((b >> 4) & 0xF) ^ 0x8) - 8
    return re.astype(np.int8), im.astype(np.int8)




# --------------------------------------------------------------------------
# correlator
# --------------------------------------------------------------------------
def correlate(blk: np.ndarray, ch0: int = 0, nch: int | None = None) -> np.ndarray:
    """X-engine on a captured block; returns vis[2*nch][2080][4][2] float32
    (xGPU triangular order, f' = 2*chan + time).  See oracle_correlate."""
    npkt, nant_in, nchan = blk.shape[:3]
    nch = nchan - ch0 if nch is None else nch
    blk = np.ascontiguousarray(blk)
    vis = np.zeros((2 * nch, NBL, 4, 2), dtype=np.float32)
    rc = lib().oracle_correlate(_ptr(blk), npkt, nant_in, nchan, ch0, nch, _ptr(vis))
    if rc != 0:
        raise RuntimeError(f"oracle_correlate failed: {rc}")
    return vis


def massage(blk: np.ndarray) -> np.ndarray:
    """dsaX_reorder_raw massage(): -> [pkt][2*nchan][64][2 pol] packed bytes."""
    npkt, nant_in, nchan = blk.shape[:3]
    out = np.empty((npkt, 2 * nchan, NST, 2), dtype=np.uint8)
    lib().oracle_massage(_ptr(np.ascontiguousarray(blk)), _ptr(out), npkt, nant_in, nchan)
    return out


def fluff_reorder(blk: np.ndarray) -> np.ndarray:
    """AVX-512 fluff + transpose: -> [pkt][2*nchan][64][2 pol][re,im] int8."""
    npkt, nant_in, nchan = blk.shape[:3]
    out = np.empty((npkt, 2 * nchan, NST, 2, 2), dtype=np.int8)
    lib().oracle_fluff_reorder(_ptr(np.ascontiguousarray(blk)), _ptr(out), npkt, nant_in, nchan)
    return out


def promote(packed: np.ndarray) -> np.ndarray:
    out = np.empty(packed.size * 2, dtype=np.int8)
    lib().oracle_promote(_ptr(np.ascontiguousarray(packed).reshape(-1)), _ptr(out), packed.size)
    return out


def xengine_int8(xin: np.ndarray) -> np.ndarray:
    """X-engine on xGPU's 8-bit input [ntime][nfreq][64][2][2]."""
    ntime, nfreq = xin.shape[:2]
    vis = np.zeros((nfreq, NBL, 4, 2), dtype=np.float32)
    rc = lib().oracle_xengine_int8(_ptr(np.ascontiguousarray(xin)), ntime, nfreq, _ptr(vis))
    if rc != 0:
        raise RuntimeError(f"oracle_xengine_int8 failed: {rc}")
    return vis


def simple_extract(vis: np.ndarray) -> np.ndarray:
    nchan = vis.shape[0] // 2
    out = np.empty((NBL, nchan, 2, 2), dtype=np.float32)
    lib().oracle_simple_extract(_ptr(np.ascontiguousarray(vis)), nchan, _ptr(out))
    return out


# --------------------------------------------------------------------------
# beamformer
# --------------------------------------------------------------------------


def geometric_weights(antpos, cal, flagged, ngrp: int, nbeam: int,
                      fch1_mhz: float = 1530.0, sep_arcmin: float = 1.0):
    """calc_weights/init_weights restated in FP64 (see C source)."""
    antpos = np.ascontiguousarray(antpos, dtype=np.float64)
    cal = np.ascontiguousarray(cal, dtype=np.float64)
    fl = np.ascontiguousarray(flagged, dtype=np.int32)
    wre = np.empty((ngrp, 2, nbeam, NST))
    wim = np.empty_like(wre)
    lib().oracle_geometric_weights(_ptr(antpos), _ptr(cal), _ptr(fl), ngrp, nbeam,
                                   float(fch1_mhz), float(sep_arcmin), _ptr(wre), _ptr(wim))
    return wre, wim


def beamform_power(blk: np.ndarray, wre: np.ndarray, wim: np.ndarray,
                   pkt_per_out: int = 16, g0: int = 0, ng: int | None = None) -> np.ndarray:
    """FP64 Stokes-I power [npkt/pkt_per_out][nbeam][ng]."""
    npkt, nant_in, nchan = blk.shape[:3]
    nbeam = wre.shape[2]
    ng = nchan // 8 - g0 if ng is None else ng
    pw = np.empty((npkt // pkt_per_out, nbeam, ng), dtype=np.float64)
    rc = lib().oracle_beamform(_ptr(np.ascontiguousarray(blk)), npkt, nant_in, nchan,
                               _ptr(np.ascontiguousarray(wre)), _ptr(np.ascontiguousarray(wim)),
                               nbeam, pkt_per_out, g0, ng, _ptr(pw))
    if rc != 0:
        raise RuntimeError(f"oracle_beamform failed: {rc}")
    return pw


def quantize_u8(power: np.ndarray, scale: float) -> np.ndarray:
    """Fixed scaling to uint8: saturate(rint(P * scale)) to [0, 255]."""
    return np.clip(np.rint(power * scale), 0, 255).astype(np.uint8)


def e4m3(x: np.ndarray) -> np.ndarray:
    """Values of FP32(x) rounded to FP8 E4M3 (3 mantissa bits, exponent
    -6..8, subnormal step 2^-9, round to nearest even, saturating at 448)."""
    x32 = np.asarray(x, np.float32).astype(np.float64)
    a = np.abs(x32)
    out = np.zeros_like(a)
    nz = a > 0
    e = np.maximum(np.floor(np.log2(a[nz])), -6.0)
    step = np.ldexp(1.0, (e - 3).astype(np.int64))
    out[nz] = np.minimum(np.rint(a[nz] / step) * step, 448.0)
    return np.copysign(out, x32)


def fp8_weights(wre: np.ndarray, wim: np.ndarray):
    """The FP8 beamformer's effective weights with a per-antenna
    power-of-two scale.  Antenna a's ideal exponent e_a puts its largest
    |coefficient| times 2^e_a in [128, 256); E = max(min e, max e - 6),
    at most min e + 5; the
    data shift d_a = clip(E - e_a, -6, 5); the stored weight is
    q = e4m3(2^(E - d_a) w), so the effective weight is 2^-(E - d_a) q.
    wre, wim: [ngrp][2][nbeam][64].  Returns (wre_q, wim_q, d, E)."""
    mx = np.maximum(np.abs(wre), np.abs(wim)).max(axis=(0, 1, 2))
    live = mx > 0
    ea = np.zeros(64, np.int64)
    ea[live] = np.clip(7 - np.floor(np.log2(mx[live])), -50, 50).astype(np.int64)
    E = int(min(ea[live].min() + 5, max(ea[live].min(), ea[live].max() - 6))) if live.any() else 0
    d = np.where(live, np.clip(E - ea, -6, 5), 0)
    sc = np.ldexp(1.0, E - d)
    return e4m3(wre * sc) / sc, e4m3(wim * sc) / sc, d, E


def quantize_u8_agc(power: np.ndarray, bp: np.ndarray) -> np.ndarray:
    """AGC requantisation of src/dsaX_beamformer.cu adder (:150-156):
    rint(P * bp[beam]) / 2 (integer division), saturated to [0, 255]
    (the reference wraps).  power [t][beam][g], bp [beam]."""
    v = np.rint(power * bp[None, :, None].astype(np.float64)).astype(np.int64)
    v = np.where(v >= 0, v // 2, -((-v) // 2))   # C division truncates toward zero
    return np.clip(v, 0, 255).astype(np.uint8)


class AgcOracle:
    """Beamformer automatic gain control, restated from the host code of
    src/dsaX_beamformer.cu: per-block per-beam power (badder :79-112 summed
    over channels by calc_allbp :482-494) enters a history of NBP = 8 blocks
    (:1022-1024); for the first 8 blocks every beam gets the median over
    beams, 0.5 (sorted[n/2-1] + sorted[n/2]) (ret_med_bp :506-513), and the
    first block's median is frozen as medbp (:1030-1036); afterwards the
    mean over the history, with beams more than 10 % off medbp reset to it
    (ret_many_bp :515-530); AGC off uses medbp throughout (:1055-1056);
    bp = 2.5 * 128 / (bp / (48 * nints)) (:1057-1062).  float32 arithmetic
    where the reference uses float, double where it promotes."""
    NBP = 8

    def __init__(self, nbeam: int, ngrp: int, nints: int, agc: bool = True):
        self.nbeam, self.ngrp, self.nints, self.agc = nbeam, ngrp, nints, agc
        self.started, self.bpctr = 0, 0
        self.medbp = np.float32(0.0)
        self.hist = np.zeros((self.NBP, nbeam), np.float32)
        self.scale = np.zeros(nbeam, np.float32)

    def update(self, power: np.ndarray) -> np.ndarray:
        p = np.asarray(power, np.float32)
        self.hist[self.bpctr % self.NBP] = p
        f32 = np.float32
        if self.started == 0 or self.bpctr < self.NBP:
            srt = np.sort(p)
            med = f32(f32(0.5) * f32(srt[self.nbeam // 2 - 1] + srt[self.nbeam // 2]))
            if self.started == 0:
                self.medbp = med
            bp = np.full(self.nbeam, med, np.float32)
            self.started = max(self.started, 1)
        else:
            acc = np.zeros(self.nbeam, np.float32)
            for j in range(self.NBP):
                acc = (acc + self.hist[j]).astype(np.float32)
            bp = (acc.astype(np.float64) / self.NBP).astype(np.float32)
            off = np.abs((bp - self.medbp).astype(np.float32)).astype(np.float64) / float(self.medbp) > 0.1
            bp[off] = self.medbp
            self.started = 2
        if not self.agc:
            bp = np.full(self.nbeam, self.medbp, np.float32)
        out = np.zeros(self.nbeam, np.float32)
        nz = bp != 0
        v = (bp[nz].astype(np.float64) / (float(self.ngrp) * self.nints)).astype(np.float32)
        out[nz] = (2.5 * 128.0 / v.astype(np.float64)).astype(np.float32)
        self.scale = out
        self.bpctr += 1
        return out


# --------------------------------------------------------------------------
# packet capture -> block assembly
# --------------------------------------------------------------------------
def packet_header(seq: int, ch_id: int, ant_id: int) -> bytes:
    """8-byte header as decoded by src/dsaX_capture.c:872-891: 35-bit seq in
    bytes 0-4 (its low 3 bits in the top of byte 4), 13-bit ch_id in the low
    5 bits of byte 4 and byte 5, 16-bit ant_id in bytes 6-7 (big-endian)."""
    h = bytearray(8)
    h[0] = (seq >> 27) & 0xFF
    h[1] = (seq >> 19) & 0xFF
    h[2] = (seq >> 11) & 0xFF
    h[3] = (seq >> 3) & 0xFF
    h[4] = ((seq & 7) << 5) | ((ch_id >> 8) & 0x1F)
    h[5] = ch_id & 0xFF
    h[6] = (ant_id >> 8) & 0xFF
    h[7] = ant_id & 0xFF
    return bytes(h)


def place_packets(pkts: bytes, stride: int, payload: int, ant_lookup, act0: int, nslots: int,
                  slots_per_seq: int, with_next: bool = True):
    """Placement of receive_obs (src/dsaX_capture.c:870-960): returns
    (block, next_block, counts[placed, next, late, dropped])."""
    block = bytearray(nslots * payload)
    nxt = bytearray(nslots * payload)
    counts = [0, 0, 0, 0]
    for k in range(len(pkts) // stride):
        p = pkts[k * stride:(k + 1) * stride]
        seq = ((p[4] & 0xE0) >> 5) | (p[3] << 3) | (p[2] << 11) | (p[1] << 19) | (p[0] << 27)
        ant_id = (p[6] << 8) | p[7]
        aid = ant_lookup[ant_id] if ant_id < len(ant_lookup) else -1
        if aid < 0:
            counts[3] += 1
            continue
        act = seq * slots_per_seq + aid
        if act < act0:
            counts[2] += 1
        elif act - act0 < nslots:
            o = (act - act0) * payload
            block[o:o + payload] = p[8:8 + payload]
            counts[0] += 1
        elif with_next and act - act0 < 2 * nslots:
            o = (act - act0 - nslots) * payload
            nxt[o:o + payload] = p[8:8 + payload]
            counts[1] += 1
        else:
            counts[3] += 1
    return bytes(block), bytes(nxt), counts


# --------------------------------------------------------------------------
# plain flagger
# --------------------------------------------------------------------------
class FlagParams(ctypes.Structure):
    _fields_ = [("nbeam", ctypes.c_int), ("ntime", ctypes.c_int), ("nchan", ctypes.c_int),
                ("guard", ctypes.c_int), ("filt", ctypes.c_int), ("tbin", ctypes.c_int),
                ("fbin", ctypes.c_int), ("ts_base", ctypes.c_int), ("tsflag", ctypes.c_int),
                ("parity", ctypes.c_int), ("thresh", ctypes.c_float),
                ("var_add", ctypes.c_float), ("ts_thresh", ctypes.c_float),
                ("nperm", ctypes.c_int), ("perm", ctypes.c_int * 8)]


def flag_params(nbeam, ntime, nchan, guard=None, filt=21, tbin=128, fbin=8,
                ts_base=None, tsflag=1, parity=0, thresh=5.0, var_add=0.5,
                ts_thresh=10.0, perm=()):
    p = FlagParams()
    p.nbeam, p.ntime, p.nchan = nbeam, ntime, nchan
    p.guard = int(round(nchan * 128 / 1024)) if guard is None else guard
    p.filt, p.tbin, p.fbin = filt, tbin, fbin
    p.ts_base = ntime // 16 if ts_base is None else ts_base
    p.tsflag, p.parity = tsflag, parity
    p.thresh, p.var_add, p.ts_thresh = thresh, var_add, ts_thresh
    p.nperm = len(perm)
    for i, c in enumerate(perm):
        p.perm[i] = c
    return p


def plain_flag(x: np.ndarray, params: FlagParams, oldspec=None):
    """Returns (chanmask[B][C] int32, tsmask[B][T] int32, chan_margin,
    ts_margin, stats) for a float32 filterbank x[B][T][C]."""
    B, T, C = x.shape
    x = np.ascontiguousarray(x, dtype=np.float32)
    cm = np.zeros((B, C), np.int32)
    tm = np.zeros((B, T), np.int32)
    cmg = np.zeros((B, C), np.float32)
    tmg = np.zeros((B, T), np.float32)
    st = np.zeros(5 * B * C + B * T, np.float32)
    old = None if oldspec is None else np.ascontiguousarray(oldspec, dtype=np.float32)
    lib().oracle_plain_flag(_ptr(x), ctypes.byref(params),
                            None if old is None else _ptr(old),
                            _ptr(cm), _ptr(tm), _ptr(cmg), _ptr(tmg), _ptr(st))
    stats = {
        "spec": st[0:B * C].reshape(B, C), "var": st[B * C:2 * B * C].reshape(B, C),
        "max": st[2 * B * C:3 * B * C].reshape(B, C), "pp": st[3 * B * C:4 * B * C].reshape(B, C),
        "sub": st[4 * B * C:5 * B * C].reshape(B, C), "ts": st[5 * B * C:].reshape(B, T),
    }
    return cm, tm, cmg, tmg, stats



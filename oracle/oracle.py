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
        L.oracle_plain_flag.argtypes = [P, P, P, P, P, P, P, P, f32]
        L.oracle_plain_flag.restype = i32
        L.oracle_flag_stats.argtypes = [P, P, P, P, P, P, P]
        L.oracle_flag_stats.restype = None
        L.oracle_chan_flags.argtypes = [P, P, P, P, P, P, P, P]
        L.oracle_chan_flags.restype = None
        L.oracle_simple_tsflag.argtypes = [P, f32, P, P, P]
        L.oracle_simple_tsflag.restype = None
        L.oracle_channflag.argtypes = [P, f32, P, P, P]
        L.oracle_channflag.restype = None
        L.oracle_simple_channflag.argtypes = [P, f32, P, P, P]
        L.oracle_simple_channflag.restype = None
        L.oracle_ts_replaced.argtypes = [P, P, P, P, P]
        L.oracle_ts_replaced.restype = None
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


def auto_extract(extracted: np.ndarray, specs: np.ndarray | None = None,
                 nant: int = 63) -> np.ndarray:
    """auto_extract (src/dsaX_wrangle.c:47-70): adds the real parts of both
    polarisations of every autocorrelation (baseline i(i+1)/2 + i, i < nant)
    of a simple_extract product [2080][nchan][2][2] into specs[nant][nchan]."""
    nchan = extracted.shape[1]
    if specs is None:
        specs = np.zeros((nant, nchan), np.float32)
    for i in range(nant):
        bl = i * (i + 1) // 2 + i
        specs[i] = (specs[i] + extracted[bl, :, 0, 0]).astype(np.float32)
        specs[i] = (specs[i] + extracted[bl, :, 1, 0]).astype(np.float32)
    return specs


def greg_order() -> np.ndarray:
    """gen_lookup (src/dsaX_wrangleAndWrite.c:46-80): for each baseline of
    the "Greg" order -- antenna pairs (i, j >= i), i major -- its index in
    xGPU's triangular order (pair (j, i) with j <= i at i(i+1)/2 + j)."""
    idx = []
    for i in range(NST):
        for j in range(i, NST):
            idx.append(j * (j + 1) // 2 + i)
    return np.asarray(idx, np.int32)


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


def two_arm_weights(antpos_e, antpos_n, arm, cal, flagged, ngrp: int, nbeam: int,
                    sfreq_mhz: float, sep_arcmin: float, dec_deg: float, pi: float = np.pi):
    """populate_weights_matrix (src/dsaX_bfCorr.cu:815-863) with the gain
    normalisation of its calc_weights (:869-928), in FP64: beams [0, nbeam/2)
    from arm 0 (phase from antpos_e), [nbeam/2, nbeam) from arm 1 (antpos_n,
    beam angle offset by -dec_deg degrees); gains cal / |cal|, zero for
    flagged antennas and for antennas of the other arm.  Returns wre, wim
    [ngrp][2 pol][nbeam][nant] (nant = len(antpos_e))."""
    antpos_e = np.asarray(antpos_e, np.float64)
    antpos_n = np.asarray(antpos_n, np.float64)
    arm = np.asarray(arm)
    nant = antpos_e.size
    cal = np.asarray(cal, np.float64).reshape(nant, ngrp, 2, 2)
    cr, ci = cal[..., 0], cal[..., 1]
    n = np.sqrt(cr * cr + ci * ci)
    n = np.where(n == 0, 1.0, n)
    g_ = (cr + 1j * ci) / n                                   # [a][g][pol]
    if flagged is not None:
        g_ = np.where(np.asarray(flagged)[:, None, None] != 0, 0, g_)
    nb_arm = nbeam // 2
    w = np.zeros((ngrp, 2, nbeam, nant), np.complex128)
    for A in (0, 1):
        pos = antpos_e if A == 0 else antpos_n
        bb = np.arange(nb_arm)
        theta = sep_arcmin * ((nb_arm // 2 - 1) - bb) * pi / 10800.0
        if A == 1:
            theta = theta - dec_deg * pi / 180.0
        for g in range(ngrp):
            nu = (sfreq_mhz - g * 250.0 / 1024.0) * 1e6
            afac = -2.0 * pi * nu * theta / 299792458.0        # [bb]
            ph = np.exp(1j * afac[:, None] * pos[None, :])      # [bb][a]
            ph = np.where((arm == A)[None, :], ph, 0)
            for pol in range(2):
                w[g, pol, A * nb_arm:(A + 1) * nb_arm] = ph * g_[None, :, g, pol]
    return w.real.copy(), w.imag.copy()


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


def plain_flag(x: np.ndarray, params: FlagParams, oldspec=None, level: float = 48.0):
    """Returns (chanmask[B][C] int32, tsmask[B][T] int32, chan_margin,
    ts_margin, stats) for a float32 filterbank x[B][T][C].  The time series
    is formed after the flagged columns are set to `level` (MN)."""
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
                            _ptr(cm), _ptr(tm), _ptr(cmg), _ptr(tmg), _ptr(st), float(level))
    stats = {
        "spec": st[0:B * C].reshape(B, C), "var": st[B * C:2 * B * C].reshape(B, C),
        "max": st[2 * B * C:3 * B * C].reshape(B, C), "pp": st[3 * B * C:4 * B * C].reshape(B, C),
        "sub": st[4 * B * C:5 * B * C].reshape(B, C), "ts": st[5 * B * C:].reshape(B, T),
    }
    return cm, tm, cmg, tmg, stats




# --------------------------------------------------------------------------
# plain flagger: the per-block data path of src/gpu_flagger.cu:1260-1487
# --------------------------------------------------------------------------
def flag_stats(x: np.ndarray, params: FlagParams):
    """spec, var, max, pp [B][C] (float32) of a filterbank (any real dtype,
    converted to float32 exactly for uint8)."""
    B, T, C = x.shape
    xf = np.ascontiguousarray(x, dtype=np.float32)
    out = [np.zeros((B, C), np.float32) for _ in range(4)]
    ts = np.zeros((B, T), np.float32)
    lib().oracle_flag_stats(_ptr(xf), ctypes.byref(params), *[_ptr(o) for o in out], _ptr(ts))
    return out


def chan_flags(spec, var, mx, pp, params: FlagParams, oldspec=None):
    """chanmask [B][C] int32 and its decision margins (channflag x3 +
    simple_channflag + permanent channels, :1340-1347)."""
    B, C = spec.shape
    cm = np.zeros((B, C), np.int32)
    mg = np.zeros((B, C), np.float32)
    arr = [np.ascontiguousarray(a, dtype=np.float32) for a in (spec, var, mx, pp)]
    old = None if oldspec is None else np.ascontiguousarray(oldspec, dtype=np.float32)
    lib().oracle_chan_flags(*[_ptr(a) for a in arr], None if old is None else _ptr(old),
                            ctypes.byref(params), _ptr(cm), _ptr(mg))
    return cm, mg


def ts_flags(ts, params: FlagParams):
    """simple_tsflag (:612-653): tsmask [B][T] int32 and margins."""
    B, T = ts.shape
    tm = np.zeros((B, T), np.int32)
    mg = np.full((B, T), np.inf, np.float32)
    t = np.ascontiguousarray(ts, dtype=np.float32)
    lib().oracle_simple_tsflag(_ptr(t), float(params.ts_thresh), ctypes.byref(params), _ptr(tm),
                               _ptr(mg))
    return tm, mg


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser of x + golden gamma (uint64 arrays)."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def noise_block(seed: int, ntime: int, nchan: int, sig: float = 6.0, mn: float = 48.0,
                dtype=np.float32) -> np.ndarray:
    """The replacement noise block [ntime][nchan]: genrand's Box-Muller
    (src/gpu_flagger.cu:500-516) on uniforms quantised to 1/16384 (RMAX),
    drawn from SplitMix64 with u1 in (0, 1]; uint8 requantised as
    (unsigned char)(rint(2 v) / 2)."""
    n = ntime * nchan
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64(seed) * np.uint64(0x100000001B3)
        r1 = splitmix64(base + np.uint64(2) * i)
        r2 = splitmix64(base + np.uint64(2) * i + np.uint64(1))
    u1 = ((r1 % np.uint64(16384)).astype(np.float64) + 1.0) / 16384.0
    u2 = (r2 % np.uint64(16384)).astype(np.float64) / 16384.0
    va = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    v = (va * float(sig) + float(mn)).astype(np.float32)
    if dtype == np.uint8:
        w = np.rint(2.0 * v.astype(np.float64))
        u = np.clip(w, 0, 4294967295).astype(np.uint64)
        return ((u // np.uint64(2)) & np.uint64(255)).astype(np.uint8).reshape(ntime, nchan)
    return v.reshape(ntime, nchan)


def scaley(x: np.ndarray, spec0: np.ndarray, var0: np.ndarray, sig: float = 6.0,
           mn: float = 48.0) -> np.ndarray:
    """scaley (:382-394): (x - spec0) * (SIG / sqrtf(var0)) + MN with the
    reference's float / double evaluation; uint8 requantised as
    (unsigned char)(__float2uint_rn(2 val) / 2) (wraps modulo 256)."""
    B, T, C = x.shape
    xf = x.astype(np.float32)
    d = (xf - spec0.astype(np.float32)[:, None, :]).astype(np.float32)
    k = np.float64(sig) / np.sqrt(var0.astype(np.float32)).astype(np.float64)
    val = (d.astype(np.float64) * k[:, None, :] + np.float64(mn)).astype(np.float32)
    if x.dtype == np.uint8:
        w = np.rint(2.0 * val.astype(np.float64))
        w = np.where(np.isnan(w), 0.0, w)
        u = np.clip(w, 0, 4294967295).astype(np.uint64)
        return ((u // np.uint64(2)) & np.uint64(255)).astype(np.uint8)
    return val


def calc_bpwr(spec: np.ndarray, guard: int, mn: float = 48.0) -> np.ndarray:
    """calc_bpwr (:759-769): float sum of every channel in order, divided by
    the channels inside the guard band, then by MN."""
    B, C = spec.shape
    acc = np.zeros(B, np.float32)
    for c in range(C):
        acc = (acc + spec[:, c].astype(np.float32)).astype(np.float32)
    return ((acc.astype(np.float64) / float(C - 2 * guard)) / float(mn)).astype(np.float32)


def zspec_median(hist: np.ndarray) -> np.ndarray:
    """fix_zspec (:114-170) over hist[naver][...]: the value whose count of
    other values <= it is naver // 2; the first block's value if none."""
    n = hist.shape[0]
    out = hist[0].copy()
    for k in range(n):
        ct = np.zeros(hist.shape[1:], np.int64)
        for j in range(n):
            if j != k:
                ct += hist[j] <= hist[k]
        out = np.where(ct == n // 2, hist[k], out)
    return out


def median_calc(arr: np.ndarray) -> np.ndarray:
    """median_calc (:771-798): per channel the lower median over beams,
    broadcast to every beam."""
    B = arr.shape[0]
    med = np.sort(arr, axis=0)[(B + 1) // 2 - 1]
    return np.broadcast_to(med, arr.shape).astype(np.float32).copy()


def repl_level(level: np.ndarray, dtype) -> np.ndarray:
    """MN x bpwr as the element type: uint8 truncates toward zero, clamped."""
    if dtype == np.uint8:
        return np.clip(np.trunc(np.minimum(level, 255.0)), 0, 255).astype(np.uint8)
    return level.astype(np.float32)


class CleanOracle:
    """The per-block data path of dsax_flag_clean, restated: measure the
    first naver blocks, then scaley + modulation check + channel flags +
    column replacement + time-series flags + row replacement per block."""

    def __init__(self, params: FlagParams, dtype=np.float32, mn=48.0, sig=6.0, mod_thresh=5e-4,
                 naver=5, scale=True, pwr=False, modcheck=True, seed=1):
        self.p = params
        self.dtype = np.dtype(dtype).type
        self.mn, self.sig, self.mod_thresh = mn, sig, mod_thresh
        self.naver, self.scale, self.pwr, self.modcheck = naver, scale, pwr, modcheck
        B, T, C = params.nbeam, params.ntime, params.nchan
        self.noise = noise_block(seed, T, C, sig, mn, self.dtype)
        self.hist = []
        self.started = False
        self.spec0 = self.var0 = None
        self.oldspec = np.zeros((B, C), np.float32)
        self.prev_tpwr = 0.0
        self.bpwr = np.ones(B, np.float32)

    def step(self, data: np.ndarray):
        """Returns (cleaned data, chanmask, tsmask, info dict, margins)."""
        p = self.p
        B, T, C, G = p.nbeam, p.ntime, p.nchan, p.guard
        x = np.array(data, copy=True)
        cm = np.zeros((B, C), np.uint8)
        tm = np.zeros((B, T), np.uint8)
        info = {"flagged": False, "replaced": False, "tpwr": 0.0, "prev_tpwr": 0.0}
        cmg = np.full((B, C), np.inf, np.float32)
        tmg = np.full((B, T), np.inf, np.float32)
        if not self.started:
            spec, var, mx, pp = flag_stats(x, p)
            self.hist.append((spec, var))
            if len(self.hist) >= self.naver:
                hs = np.stack([h[0] for h in self.hist])
                hv = np.stack([h[1] for h in self.hist])
                self.spec0 = median_calc(zspec_median(hs))
                self.var0 = median_calc(zspec_median(hv))
                self.started = True
        else:
            if self.scale:
                x = scaley(x, self.spec0, self.var0, self.sig, self.mn)
            spec, var, mx, pp = flag_stats(x, p)
            tpwr = float(np.sum(spec.astype(np.float64)))
            info.update(flagged=True, tpwr=tpwr, prev_tpwr=self.prev_tpwr)
            replaced = (self.modcheck and self.prev_tpwr > 0 and
                        abs(tpwr - self.prev_tpwr) / self.prev_tpwr >= self.mod_thresh)
            info["mod_index"] = (abs(tpwr - self.prev_tpwr) / self.prev_tpwr
                                 if self.prev_tpwr > 0 else None)
            if replaced:
                x[:] = self.noise[None, :, :]
                info["replaced"] = True
            else:
                cmi, cmg = chan_flags(spec, var, mx, pp, p, self.oldspec)
                cm = cmi.astype(np.uint8)
                if self.pwr:
                    self.bpwr = calc_bpwr(spec, G, self.mn)
                lev = repl_level(self.mn * self.bpwr.astype(np.float32), self.dtype)
                for b in range(B):
                    cols = np.nonzero(cm[b])[0]
                    if cols.size:
                        x[b][:, cols] = lev[b]
                ts = (x.astype(np.float64).sum(axis=2) / C).astype(np.float32)
                if p.tsflag:
                    tmi, tmg = ts_flags(ts, p)
                    tm = tmi.astype(np.uint8)
                    for b in range(B):
                        rows = np.nonzero(tm[b])[0]
                        if rows.size:
                            x[b][rows, G:C - G] = lev[b]
                info["ts"] = ts
            self.prev_tpwr = tpwr
        self.oldspec = spec
        info["spec"] = spec
        return x, cm, tm, info, (cmg, tmg)


# --------------------------------------------------------------------------
# oracle/_ref: the reference's own functions (built by make_ref.py)
# --------------------------------------------------------------------------
_ref_libs = {}


def ref_lib(small: bool = False):
    """oracle/_ref/libref.so (or the 64-packet build), built from the
    reference tree when missing.  Raises FileNotFoundError when neither the
    library nor the reference tree is present."""
    key = "small" if small else "full"
    if key in _ref_libs:
        return _ref_libs[key]
    path = os.path.join(_HERE, "_ref", "libref_small.so" if small else "libref.so")
    if not os.path.exists(path):
        import make_ref  # noqa: E402  (oracle/ is on sys.path)
        make_ref.build()
    L = ctypes.CDLL(path)
    P, i32, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.ref_flag_shape.argtypes = [P, P, P]
    L.ref_medval.argtypes = [P, i32]
    L.ref_medval.restype = f32
    for n in ("ref_channflag", "ref_simple_channflag", "ref_simple_tsflag"):
        getattr(L, n).argtypes = [P, f32, P]
    for n in ("ref_gather_mask", "ref_gather_tsmask"):
        getattr(L, n).argtypes = [P, P, P]
    L.ref_calc_bpwr.argtypes = [P, P]
    L.ref_median_calc.argtypes = [P]
    L.ref_scaley.argtypes = [P, P, P]
    L.ref_flag.argtypes = [P, P, i32, P]
    L.ref_flagts.argtypes = [P, P, i32, P]
    L.ref_auto_extract.argtypes = [P, P]
    L.ref_simple_extract.argtypes = [P, P]
    L.ref_gen_lookup.argtypes = [P]
    L.ref_reorder_gh.argtypes = [P, P, P]
    L.ref_bfcorr_shape.argtypes = [P, P, P]
    L.ref_populate_weights.argtypes = [P, P, P, P, P, P, f32]
    L.ref_massage_raw.argtypes = [P, P, i32]
    L.ref_massage_raw.restype = i32
    L.ref_massage_bak.argtypes = [P, P, i32]
    L.ref_massage_bak.restype = i32
    L.ref_npackets.restype = i32
    L.ref_nants.restype = i32
    _ref_libs[key] = L
    return L


def ref_available() -> bool:
    if os.path.exists(os.path.join(_HERE, "_ref", "libref.so")):
        return True
    return os.path.isdir(os.environ.get("DSAX_REFERENCE", "/root/reference"))


# --------------------------------------------------------------------------
# beam corner turn (src/dsaX_dbnic.c:84-152, src/dsaX_nicdb.c:180-196)
# --------------------------------------------------------------------------
def ct_pack(beams: np.ndarray, ndest: int) -> np.ndarray:
    """dbnic's per-search-node transpose: beams [T][NB][C] ->
    [ndest][NB/ndest][T][C] (op[j][i][k] = output[i][d*nbl + j][k])."""
    T, NB, C = beams.shape
    return np.ascontiguousarray(beams.reshape(T, ndest, NB // ndest, C).transpose(1, 2, 0, 3))


def ct_unpack(recv: np.ndarray, fil: np.ndarray, t0: int, ch0: int) -> np.ndarray:
    """nicdb's placement: recv [nsrc][nbl][T][C] into fil[nbl][t0 + t]
    [ch0 + src C + k]."""
    S, nbl, T, C = recv.shape
    for s in range(S):
        fil[:, t0:t0 + T, ch0 + s * C:ch0 + (s + 1) * C] = recv[s]
    return fil

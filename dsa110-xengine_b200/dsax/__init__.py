"""Python binding of libdsax.so (include/dsax.h) through ctypes.

This is a thin host-side mirror of the C ABI for tests, the benchmark and
Python callers.  Device buffers are passed as raw pointers (torch tensors'
data_ptr() or any CUDA allocation); the library itself holds no torch types.

There is no fallback: if libdsax.so is missing or cannot be loaded, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "libdsax.so")
HEADER_DIR = os.path.join(os.path.dirname(_PKG_DIR), "include")

DSAX_OK = 0
DSAX_ERR_ARG = -1
DSAX_ERR_CUDA = -2
DSAX_ERR_TIMEOUT = -3
DSAX_ERR_NOMEM = -4
DSAX_ERR_UNSUPPORTED = -5
DSAX_ERR_DEVICE = -6

MEM_HOST = 0
MEM_DEVICE = 1

FMT_CAPTURED = 0
FMT_REORDERED = 1
FMT_XGPU_INT8 = 2
FMT_CHANMAJOR = 3

NBL = 2080


class DsaxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"dsax status {status}: {msg}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [
        ("npkt", ctypes.c_int),
        ("nant_in", ctypes.c_int),
        ("nchan", ctypes.c_int),
        ("nbeam", ctypes.c_int),
        ("bf_pkt_per_out", ctypes.c_int),
        ("bf_scale", ctypes.c_float),
        ("wait_limit_ns", ctypes.c_ulonglong),
        ("corr_path", ctypes.c_int),
        ("bf_fp8", ctypes.c_int),
        ("bf_path", ctypes.c_int),
        ("bf_variant", ctypes.c_int),
    ]


class FlagParams(ctypes.Structure):
    _fields_ = [("nbeam", ctypes.c_int), ("ntime", ctypes.c_int), ("nchan", ctypes.c_int),
                ("guard", ctypes.c_int), ("filt", ctypes.c_int), ("tbin", ctypes.c_int),
                ("fbin", ctypes.c_int), ("ts_base", ctypes.c_int), ("tsflag", ctypes.c_int),
                ("parity", ctypes.c_int), ("thresh", ctypes.c_float),
                ("var_add", ctypes.c_float), ("ts_thresh", ctypes.c_float),
                ("nperm", ctypes.c_int), ("perm", ctypes.c_int * 8)]


class FlagCleanParams(ctypes.Structure):
    _fields_ = [("mn", ctypes.c_float), ("sig", ctypes.c_float), ("mod_thresh", ctypes.c_float),
                ("naver", ctypes.c_int), ("scale", ctypes.c_int), ("pwr", ctypes.c_int),
                ("modcheck", ctypes.c_int), ("seed", ctypes.c_ulonglong)]


class FlagBlockInfo(ctypes.Structure):
    _fields_ = [("blocks", ctypes.c_int), ("started", ctypes.c_int), ("flagged", ctypes.c_int),
                ("replaced", ctypes.c_int), ("nchan_flagged", ctypes.c_int),
                ("nts_flagged", ctypes.c_int), ("tpwr", ctypes.c_double),
                ("prev_tpwr", ctypes.c_double)]


DTYPE_F32 = 0
DTYPE_U8 = 1


def flag_clean_params(**kw) -> FlagCleanParams:
    cp = FlagCleanParams()
    lib().dsax_default_flag_clean_params(ctypes.byref(cp))
    for k, v in kw.items():
        setattr(cp, k, v)
    return cp


class BlockDesc(ctypes.Structure):
    _fields_ = [("blk", ctypes.c_void_p), ("nchan", ctypes.c_int), ("vis", ctypes.c_void_p),
                ("beams", ctypes.c_void_p), ("chanmask", ctypes.c_void_p),
                ("tsmask", ctypes.c_void_p)]


def flag_params(nbeam: int, ntime: int, nchan: int, **kw) -> FlagParams:
    p = FlagParams()
    lib().dsax_default_flag_params(ctypes.byref(p), nbeam, ntime, nchan)
    perm = kw.pop("perm", None)
    for k, v in kw.items():
        setattr(p, k, v)
    if perm is not None:
        p.nperm = len(perm)
        for i, c in enumerate(perm):
            p.perm[i] = c
    return p


_lib = None


def build(force: bool = False) -> str:
    """Run the package Makefile (nvcc, sm_100a) and return the library path."""
    args = ["make", "-s", "-C", _PKG_DIR, "-j8"]
    if force:
        args.insert(2, "-B")
    subprocess.check_call(args)
    return LIB_PATH


def lib():
    """Load libdsax.so (raises OSError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"libdsax.so not built at {LIB_PATH}; run `make -C {_PKG_DIR}`")
    L = ctypes.CDLL(LIB_PATH)
    P, I, Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    CP = ctypes.POINTER(Config)
    L.dsax_default_config.argtypes = [CP]
    L.dsax_default_config.restype = None
    for fn in ("dsax_block_bytes",):
        getattr(L, fn).argtypes = [CP, I]
        getattr(L, fn).restype = Z
    for fn in ("dsax_vis_bytes", "dsax_beam_bytes"):
        getattr(L, fn).argtypes = [CP]
        getattr(L, fn).restype = Z
    L.dsax_create.argtypes = [ctypes.POINTER(P), CP, I]
    L.dsax_create.restype = I
    L.dsax_destroy.argtypes = [P]
    L.dsax_destroy.restype = None
    L.dsax_strerror.argtypes = [I]
    L.dsax_strerror.restype = ctypes.c_char_p
    L.dsax_last_error.argtypes = [P]
    L.dsax_last_error.restype = ctypes.c_char_p
    L.dsax_stream.argtypes = [P]
    L.dsax_stream.restype = P
    L.dsax_sync.argtypes = [P]
    L.dsax_sync.restype = I
    L.dsax_host_alloc.argtypes = [P, Z, ctypes.POINTER(P)]
    L.dsax_host_alloc.restype = I
    L.dsax_host_free.argtypes = [P, P]
    L.dsax_host_free.restype = I
    L.dsax_correlate.argtypes = [P, P, P, I]
    L.dsax_correlate.restype = I
    L.dsax_correlate_fmt.argtypes = [P, I, P, P, I, I]
    L.dsax_correlate_fmt.restype = I
    _bind_optional(L)
    _lib = L
    return L


def _bind_optional(L):
    """Signatures of the entry points beyond the correlator."""
    P, I = ctypes.c_void_p, ctypes.c_int
    table = {
        "dsax_set_weights": ([P, P, P], I),
        "dsax_beamform": ([P, P, P, P, I], I),
        "dsax_default_flag_params": ([ctypes.POINTER(FlagParams), I, I, I], None),
        "dsax_flag": ([P, ctypes.POINTER(FlagParams), P, P, P, P, P, P, I], I),
        "dsax_reorder": ([P, P, P, I], I),
        "dsax_corner_turn": ([P, P, P, I, I], I),
        "dsax_correlate_many": ([P, P, P, I, I], I),
        "dsax_agc_enable": ([P, I], I),
        "dsax_extract": ([P, P, P, I], I),
        "dsax_place_packets": ([P, P, I, I, I, P, I, ctypes.c_ulonglong, ctypes.c_ulonglong, I, P, P,
                                P], I),
        "dsax_correlate_extract": ([P, P, P, I], I),
        "dsax_extract_ex": ([P, P, P, I, P, I], I),
        "dsax_correlate_extract_ex": ([P, P, P, I, P, I], I),
        "dsax_set_geometric_weights": ([P, P, P, P, ctypes.c_double, ctypes.c_double], I),
        "dsax_set_two_arm_weights": ([P, P, P, P, P, P, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double], I),
        "dsax_agc_state": ([P, P, ctypes.POINTER(I), ctypes.POINTER(I)], I),
        "dsax_lf_nparams": ([], I),
        "dsax_lf_init": ([P, ctypes.c_ulonglong], I),
        "dsax_lf_set_params": ([P, P, I], I),
        "dsax_lf_get_params": ([P, P, I], I),
        "dsax_lf_features": ([P, P, ctypes.POINTER(FlagParams), I, P], I),
        "dsax_lf_train_step": ([P, P, P, P, ctypes.POINTER(FlagParams), I, ctypes.c_float,
                                ctypes.c_float, I, P, P], I),
        "dsax_flag_learned": ([P, P, ctypes.POINTER(FlagParams), I, P, P, I], I),
        "dsax_run_batch": ([P, ctypes.POINTER(BlockDesc), I, I], I),
        "dsax_default_flag_clean_params": ([ctypes.POINTER(FlagCleanParams)], None),
        "dsax_probe_tensor_peak": ([P, I, I, ctypes.POINTER(ctypes.c_double)], I),
        "dsax_ct_pack": ([P, P, I, I, I, I, P], I),
        "dsax_check_wait_limit": ([P, ctypes.c_ulonglong], I),
        "dsax_ct_unpack": ([P, P, I, I, I, I, P, I, I, I, I], I),
        "dsax_flag_state_create": ([P, ctypes.POINTER(FlagParams), ctypes.POINTER(FlagCleanParams),
                                    I, ctypes.POINTER(P)], I),
        "dsax_flag_state_destroy": ([P], None),
        "dsax_flag_clean": ([P, P, P, P, P, I], I),
        "dsax_flag_state_info": ([P, P, ctypes.POINTER(FlagBlockInfo)], I),
        "dsax_flag_state_get_baseline": ([P, P, P, P], I),
        "dsax_flag_state_set_baseline": ([P, P, P, P], I),
        "dsax_flag_state_noise": ([P, P, P], I),
        "dsax_autotune": ([P, I, P, I, P], I),
        "dsax_autotune_beamformer": ([P, I, P, I, P], I),
    }
    for name, (args, res) in table.items():
        if hasattr(L, name):
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res


def default_config(**kw) -> Config:
    c = Config()
    lib().dsax_default_config(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def block_bytes(cfg: Config, fmt: int = FMT_CAPTURED) -> int:
    return int(lib().dsax_block_bytes(ctypes.byref(cfg), fmt))


def vis_bytes(cfg: Config) -> int:
    return int(lib().dsax_vis_bytes(ctypes.byref(cfg)))


def beam_bytes(cfg: Config) -> int:
    return int(lib().dsax_beam_bytes(ctypes.byref(cfg)))


def strerror(status: int) -> str:
    return lib().dsax_strerror(status).decode()


def _ptr(x) -> int:
    """Raw address of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


class Context:
    """One dsax context: one device, one stream, its scratch buffers."""

    def __init__(self, cfg: Config | None = None, device: int = 0):
        self.cfg = cfg if cfg is not None else default_config()
        self._h = ctypes.c_void_p()
        rc = lib().dsax_create(ctypes.byref(self._h), ctypes.byref(self.cfg), device)
        if rc != DSAX_OK:
            raise DsaxError(rc, f"dsax_create: {strerror(rc)}")
        self.device = device

    # -- plumbing ----------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc != DSAX_OK:
            msg = lib().dsax_last_error(self._h).decode()
            raise DsaxError(rc, f"{what}: {strerror(rc)} ({msg})")

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return int(lib().dsax_stream(self._h) or 0)

    def sync(self):
        self._check(lib().dsax_sync(self._h), "dsax_sync")

    def close(self):
        if self._h:
            lib().dsax_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- correlator --------------------------------------------------------
    def correlate(self, blk, vis, mem: int = MEM_DEVICE, fmt: int = FMT_CAPTURED,
                  accumulate: bool = False):
        rc = lib().dsax_correlate_fmt(self._h, fmt, _ptr(blk), _ptr(vis), mem, int(accumulate))
        self._check(rc, "dsax_correlate_fmt")

    def correlate_many(self, blocks, vis, mem: int = MEM_DEVICE):
        """blocks, vis: equal-length lists of buffers (device tensors or host
        arrays); stages of consecutive blocks overlap on side streams."""
        n = len(blocks)
        if n != len(vis) or n == 0:
            raise ValueError("blocks and vis must be non-empty and of equal length")
        pb = (ctypes.c_void_p * n)(*[_ptr(b) for b in blocks])
        pv = (ctypes.c_void_p * n)(*[_ptr(v) for v in vis])
        self._check(lib().dsax_correlate_many(self._h, pb, pv, n, mem), "dsax_correlate_many")

    def reorder(self, captured, reordered, mem: int = MEM_DEVICE):
        """massage() on the GPU: captured -> REORDER-key layout."""
        self._check(lib().dsax_reorder(self._h, _ptr(captured), _ptr(reordered), mem),
                    "dsax_reorder")

    def corner_turn(self, captured, out, out_fmt: int = FMT_CHANMAJOR, mem: int = MEM_DEVICE):
        self._check(lib().dsax_corner_turn(self._h, _ptr(captured), _ptr(out), out_fmt, mem),
                    "dsax_corner_turn")

    # -- beamformer --------------------------------------------------------
    def set_weights(self, wre, wim):
        """FP64 weights [nchan/8][2][nbeam][64] (numpy, host)."""
        import numpy as np
        wre = np.ascontiguousarray(wre, dtype=np.float64)
        wim = np.ascontiguousarray(wim, dtype=np.float64)
        self._check(lib().dsax_set_weights(self._h, _ptr(wre), _ptr(wim)), "dsax_set_weights")

    def set_geometric_weights(self, antpos, cal, flagged=None, fch1_mhz: float = 1530.0,
                              sep_arcmin: float = 1.0):
        """antpos[64] (m), cal[64][nchan/8][2][2] (re, im), flagged[64] or None."""
        import numpy as np
        antpos = np.ascontiguousarray(antpos, dtype=np.float64)
        cal = np.ascontiguousarray(cal, dtype=np.float64)
        fl = None if flagged is None else np.ascontiguousarray(flagged, dtype=np.int32)
        self._check(lib().dsax_set_geometric_weights(self._h, _ptr(antpos), _ptr(cal), _ptr(fl),
                                                     float(fch1_mhz), float(sep_arcmin)),
                    "dsax_set_geometric_weights")

    def set_two_arm_weights(self, antpos_e, antpos_n, arm, cal, flagged=None,
                            sfreq_mhz: float = 1498.75, sep_arcmin: float = 1.0,
                            dec_deg: float = 0.0):
        """Two-arm weights with the declination term (see include/dsax.h)."""
        import numpy as np
        ae = np.ascontiguousarray(antpos_e, dtype=np.float64)
        an = np.ascontiguousarray(antpos_n, dtype=np.float64)
        ar = np.ascontiguousarray(arm, dtype=np.int32)
        cal = np.ascontiguousarray(cal, dtype=np.float64)
        fl = None if flagged is None else np.ascontiguousarray(flagged, dtype=np.int32)
        self._check(lib().dsax_set_two_arm_weights(self._h, _ptr(ae), _ptr(an), _ptr(ar), _ptr(cal),
                                                   _ptr(fl), float(sfreq_mhz), float(sep_arcmin),
                                                   float(dec_deg)),
                    "dsax_set_two_arm_weights")

    def place_packets(self, pkts, npk, stride, payload, ant_lookup, act0, nslots, slots_per_seq,
                      block, counts, next_block=None):
        """Device tensors: pkts (bytes), ant_lookup (int32), block, counts (int64[4])."""
        rc = lib().dsax_place_packets(self._h, _ptr(pkts), npk, stride, payload, _ptr(ant_lookup),
                                      int(ant_lookup.numel()), act0, nslots, slots_per_seq,
                                      _ptr(block), _ptr(next_block), _ptr(counts))
        self._check(rc, "dsax_place_packets")

    def extract(self, vis, out, mem: int = MEM_DEVICE):
        """simple_extract: XX/YY averaged over the two time slots."""
        self._check(lib().dsax_extract(self._h, _ptr(vis), _ptr(out), mem), "dsax_extract")

    def correlate_extract(self, blk, out, mem: int = MEM_DEVICE, order: int = 0, autos=None):
        """order 0: xGPU baselines, 1: "Greg" order; autos: spectra added to."""
        self._check(lib().dsax_correlate_extract_ex(self._h, _ptr(blk), _ptr(out), order,
                                                    _ptr(autos), mem),
                    "dsax_correlate_extract_ex")

    def extract_ex(self, vis, out, order: int = 0, autos=None, mem: int = MEM_DEVICE):
        self._check(lib().dsax_extract_ex(self._h, _ptr(vis), _ptr(out), order, _ptr(autos), mem),
                    "dsax_extract_ex")

    def agc_enable(self, mode: int = 1):
        """1 adaptive, 2 frozen at the first block's median, 0 off."""
        self._check(lib().dsax_agc_enable(self._h, mode), "dsax_agc_enable")

    def agc_state(self):
        """Returns (scale [nbeam] numpy, started, blocks)."""
        import numpy as np
        sc = np.zeros(self.cfg.nbeam, np.float32)
        st, nb = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().dsax_agc_state(self._h, _ptr(sc), ctypes.byref(st), ctypes.byref(nb)),
                    "dsax_agc_state")
        return sc, st.value, nb.value

    def beamform(self, blk, out_u8=None, out_f32=None, mem: int = MEM_DEVICE):
        rc = lib().dsax_beamform(self._h, _ptr(blk), _ptr(out_u8), _ptr(out_f32), mem)
        self._check(rc, "dsax_beamform")

    # -- plain flagger -----------------------------------------------------
    def flag(self, params: FlagParams, x, chanmask, tsmask, oldspec=None, stats=None,
             counts=None, mem: int = MEM_DEVICE):
        rc = lib().dsax_flag(self._h, ctypes.byref(params), _ptr(x), _ptr(oldspec),
                             _ptr(chanmask), _ptr(tsmask), _ptr(stats), _ptr(counts), mem)
        self._check(rc, "dsax_flag")

    def flag_state(self, params: FlagParams, clean: FlagCleanParams | None = None,
                   dtype: int = DTYPE_F32) -> "FlagState":
        return FlagState(self, params, clean if clean is not None else flag_clean_params(), dtype)

    # -- learned flagger ---------------------------------------------------
    def lf_init(self, seed: int = 0):
        self._check(lib().dsax_lf_init(self._h, seed), "dsax_lf_init")

    def lf_set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().dsax_lf_set_params(self._h, _ptr(p), p.size), "dsax_lf_set_params")

    def lf_get_params(self):
        import numpy as np
        p = np.zeros(lib().dsax_lf_nparams(), np.float32)
        self._check(lib().dsax_lf_get_params(self._h, _ptr(p), p.size), "dsax_lf_get_params")
        return p

    def lf_features(self, params: FlagParams, x, F, tds: int = 32):
        self._check(lib().dsax_lf_features(self._h, _ptr(x), ctypes.byref(params), tds, _ptr(F)),
                    "dsax_lf_features")

    def lf_train_step(self, params: FlagParams, x, chanmask, tsmask, tds: int = 32,
                      lr: float = 1e-3, pos_weight: float = 1.0, update: bool = True,
                      want_grads: bool = False):
        import numpy as np
        loss = ctypes.c_float(0.0)
        g = np.zeros(lib().dsax_lf_nparams(), np.float32) if want_grads else None
        rc = lib().dsax_lf_train_step(self._h, _ptr(x), _ptr(chanmask), _ptr(tsmask),
                                      ctypes.byref(params), tds, lr, pos_weight, int(update),
                                      ctypes.byref(loss), _ptr(g))
        self._check(rc, "dsax_lf_train_step")
        return (loss.value, g) if want_grads else loss.value

    def flag_learned(self, params: FlagParams, x, mask, logits=None, tds: int = 32,
                     mem: int = MEM_DEVICE):
        rc = lib().dsax_flag_learned(self._h, _ptr(x), ctypes.byref(params), tds, _ptr(mask),
                                     _ptr(logits), mem)
        self._check(rc, "dsax_flag_learned")

    def ct_pack(self, beams, nt: int, nb: int, nc: int, ndest: int, send):
        """Beam corner turn, sending side: [nt][nb][nc] -> [ndest][nb/ndest][nt][nc]."""
        self._check(lib().dsax_ct_pack(self._h, _ptr(beams), nt, nb, nc, ndest, _ptr(send)),
                    "dsax_ct_pack")

    def ct_unpack(self, recv, nsrc: int, nbl: int, nt: int, nc: int, fil, fil_nt: int,
                  fil_nc: int, t0: int = 0, ch0: int = 0):
        """Beam corner turn, receiving side: [nsrc][nbl][nt][nc] -> filterbank."""
        self._check(lib().dsax_ct_unpack(self._h, _ptr(recv), nsrc, nbl, nt, nc, _ptr(fil), fil_nt,
                                         fil_nc, t0, ch0), "dsax_ct_unpack")

    def probe_tensor_peak(self, kind: int = 0, reps: int = 3) -> float:
        """Measured dense tensor-core ops/s: kind 0 int8, 1 BF16, 2 FP8 E4M3."""
        v = ctypes.c_double(0.0)
        self._check(lib().dsax_probe_tensor_peak(self._h, kind, reps, ctypes.byref(v)),
                    "dsax_probe_tensor_peak")
        return v.value

    # -- autotuner ---------------------------------------------------------
    def autotune(self, reps: int = 10):
        """Returns ({corr_path: ms}, chosen corr_path); the context keeps the choice."""
        import numpy as np
        t = np.zeros(7, np.float32)
        best = ctypes.c_int(0)
        self._check(lib().dsax_autotune(self._h, reps, _ptr(t), 7, ctypes.byref(best)),
                    "dsax_autotune")
        self.cfg.corr_path = best.value
        return {k + 1: float(t[k]) for k in range(7)}, best.value

    def autotune_beamformer(self, reps: int = 10):
        """Returns ({candidate: ms}, chosen candidate): 1 = the one-CTA form,
        2-5 = CTA pairs with bf_variant 1-4; the context keeps the choice
        (dsax_set_weights first)."""
        import numpy as np
        t = np.zeros(5, np.float32)
        best = ctypes.c_int(0)
        self._check(lib().dsax_autotune_beamformer(self._h, reps, _ptr(t), 5, ctypes.byref(best)),
                    "dsax_autotune_beamformer")
        self.cfg.bf_path = 1 if best.value == 1 else 2
        self.cfg.bf_variant = 0 if best.value == 1 else best.value - 1
        return {k + 1: float(t[k]) for k in range(5)}, best.value

    # -- batches -----------------------------------------------------------
    def run_batch(self, descs, use_graph: bool = True):
        """descs: list of dicts with keys blk, nchan, vis, beams, chanmask,
        tsmask (device tensors or None)."""
        arr = (BlockDesc * len(descs))()
        for i, d in enumerate(descs):
            arr[i].blk = _ptr(d["blk"])
            arr[i].nchan = int(d["nchan"])
            arr[i].vis = _ptr(d.get("vis"))
            arr[i].beams = _ptr(d.get("beams"))
            arr[i].chanmask = _ptr(d.get("chanmask"))
            arr[i].tsmask = _ptr(d.get("tsmask"))
        self._check(lib().dsax_run_batch(self._h, arr, len(descs), int(use_graph)),
                    "dsax_run_batch")


class FlagState:
    """The plain flagger's per-block data path (dsax_flag_clean) and its
    state: baseline, previous spectrum and total power, noise block."""

    def __init__(self, ctx: Context, params: FlagParams, clean: FlagCleanParams, dtype: int):
        self.ctx = ctx
        self.params = params
        self.clean_params = clean
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        ctx._check(lib().dsax_flag_state_create(ctx.handle, ctypes.byref(params),
                                                ctypes.byref(clean), dtype, ctypes.byref(self._h)),
                   "dsax_flag_state_create")

    def close(self):
        if self._h:
            lib().dsax_flag_state_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clean(self, data, chanmask=None, tsmask=None, mem: int = MEM_DEVICE):
        """One block, cleaned in place."""
        self.ctx._check(lib().dsax_flag_clean(self.ctx.handle, self._h, _ptr(data), _ptr(chanmask),
                                              _ptr(tsmask), mem), "dsax_flag_clean")

    def info(self) -> FlagBlockInfo:
        inf = FlagBlockInfo()
        self.ctx._check(lib().dsax_flag_state_info(self.ctx.handle, self._h, ctypes.byref(inf)),
                        "dsax_flag_state_info")
        return inf

    def baseline(self):
        import numpy as np
        n = self.params.nbeam * self.params.nchan
        s0, v0 = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.ctx._check(lib().dsax_flag_state_get_baseline(self.ctx.handle, self._h, _ptr(s0),
                                                           _ptr(v0)), "dsax_flag_state_get_baseline")
        shape = (self.params.nbeam, self.params.nchan)
        return s0.reshape(shape), v0.reshape(shape)

    def set_baseline(self, spec0, var0):
        import numpy as np
        s0 = np.ascontiguousarray(spec0, dtype=np.float32)
        v0 = np.ascontiguousarray(var0, dtype=np.float32)
        self.ctx._check(lib().dsax_flag_state_set_baseline(self.ctx.handle, self._h, _ptr(s0),
                                                           _ptr(v0)), "dsax_flag_state_set_baseline")

    def noise(self):
        import numpy as np
        dt = np.uint8 if self.dtype == DTYPE_U8 else np.float32
        out = np.zeros((self.params.ntime, self.params.nchan), dt)
        self.ctx._check(lib().dsax_flag_state_noise(self.ctx.handle, self._h, _ptr(out)),
                        "dsax_flag_state_noise")
        return out

"""The oracle restatement pinned to the reference's own code (CPU).

oracle/make_ref.py lifts the reference's plain-C functions -- the flagger's
host decisions and element kernels, the visibility extractors, both reorder
threads -- out of the reference tree into oracle/_ref/libref.so.  These
tests run them beside the oracle (oracle/*.c, oracle/oracle.py) on the same
seeded inputs: masks, indices and bytes must be identical, floating-point
results bit-identical where the two evaluate the same expression in the same
order.  The reference's compile-time shapes apply (see make_ref.py):
flagger [64 beams][2048 t][1024 ch] with its 128-channel guard band,
reorders [packets][63 antennas][384 ch][2 t][2 pol].
"""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built and no reference tree to build it from")
    return oracle.ref_lib()


@pytest.fixture(scope="module")
def ref_small(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built and no reference tree to build it from")
    return oracle.ref_lib(small=True)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _shape(ref):
    B, T, C = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    ref.ref_flag_shape(ctypes.byref(B), ctypes.byref(T), ctypes.byref(C))
    return B.value, T.value, C.value


def _params(oracle, B, T, C, parity=1):
    # the reference's constants: guard 128, nFiltSize 21, FBIN 8, T/16,
    # permanent channel 10 (inside the guard band, so never applied)
    return oracle.flag_params(B, T, C, guard=128, filt=21, fbin=8, ts_base=T // 16,
                              parity=parity, perm=[10])


def _spectra(seed, B, C):
    """Spectrum-like inputs: smooth bandpass + noise + a few tones and a
    dip, so every test fires somewhere and most channels stay clean."""
    rng = np.random.default_rng(seed)
    c = np.arange(C)
    base = 40 + 8 * np.sin(c / 97.0)[None, :] + rng.normal(0, 0.3, (B, C))
    for b in range(B):
        for ch in rng.integers(130, C - 130, size=3):
            base[b, ch] += rng.uniform(2, 30)
        base[b, rng.integers(130, C - 130)] -= rng.uniform(2, 10)
    return base.astype(np.float32)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_channflag_matches_reference(ref, oracle, seed):
    B, T, C = _shape(ref)
    p = _params(oracle, B, T, C)
    spec = _spectra(seed, B, C)
    for thr in (5.0, 5.5, 3.0):
        rm = np.zeros(B * C, np.int32)
        ref.ref_channflag(_p(spec), thr, _p(rm))
        om = np.zeros(B * C, np.int32)
        oracle.lib().oracle_channflag(_p(spec), thr, ctypes.byref(p), _p(om), None)
        assert rm.sum() > 0
        np.testing.assert_array_equal(om, rm)


@pytest.mark.parametrize("seed", [4, 5])
def test_simple_channflag_matches_reference(ref, oracle, seed):
    """Parity mode: the reference's FBIN loop adds spec[j] FBIN times
    (src/gpu_flagger.cu:594)."""
    B, T, C = _shape(ref)
    p = _params(oracle, B, T, C, parity=1)
    pp = np.abs(_spectra(seed, B, C) - 40.0).astype(np.float32)
    rm = np.zeros(B * C, np.int32)
    ref.ref_simple_channflag(_p(pp), 5.0, _p(rm))
    om = np.zeros(B * C, np.int32)
    oracle.lib().oracle_simple_channflag(_p(pp), 5.0, ctypes.byref(p), _p(om), None)
    assert rm.sum() > 0
    np.testing.assert_array_equal(om, rm)


def test_simple_tsflag_matches_reference(ref, oracle):
    B, T, C = _shape(ref)
    p = _params(oracle, B, T, C)
    rng = np.random.default_rng(7)
    ts = rng.normal(50, 1, (B, T)).astype(np.float32)
    ts[:, 300:304] += 30
    ts[5, 1000] += 200
    rm = np.zeros(B * T, np.int32)
    ref.ref_simple_tsflag(_p(ts), 10.0, _p(rm))
    om, _ = oracle.ts_flags(ts, p)
    assert rm.sum() >= B * 4
    np.testing.assert_array_equal(om.reshape(-1), rm)


def test_medval_matches_reference(ref):
    rng = np.random.default_rng(8)
    for n in (1, 2, 21, 256, 768):
        a = rng.normal(0, 1, n).astype(np.float32)
        a[: n // 3] = a[0]   # ties
        got = ref.ref_medval(_p(a), n)
        assert got == np.sort(a)[(n + 1) // 2 - 1]


def test_calc_bpwr_matches_reference(ref, oracle):
    B, T, C = _shape(ref)
    spec = _spectra(9, B, C)
    rb = np.zeros(B, np.float32)
    ref.ref_calc_bpwr(_p(spec), _p(rb))
    np.testing.assert_array_equal(oracle.calc_bpwr(spec, guard=128, mn=48.0), rb)


def test_median_calc_matches_reference(ref, oracle):
    B, T, C = _shape(ref)
    a = _spectra(10, B, C)
    r = a.copy()
    ref.ref_median_calc(_p(r))
    np.testing.assert_array_equal(oracle.median_calc(a), r)


def test_gather_mask_matches_reference(ref):
    B, T, C = _shape(ref)
    rng = np.random.default_rng(11)
    m = (rng.random(B * C) < 0.05).astype(np.int32)
    idx = np.zeros(B * C, np.int32)
    n = ctypes.c_int(0)
    ref.ref_gather_mask(_p(idx), _p(m), ctypes.byref(n))
    np.testing.assert_array_equal(idx[: n.value], np.nonzero(m)[0])


def test_scaley_matches_reference(ref, oracle):
    """scaley on a uint8 block, including values that wrap modulo 256."""
    B, T, C = _shape(ref)
    rng = np.random.default_rng(12)
    x = rng.integers(0, 256, (B, T, C), dtype=np.uint8)
    spec0 = rng.uniform(20, 120, (B, C)).astype(np.float32)
    var0 = rng.uniform(0.5, 400, (B, C)).astype(np.float32)
    r = x.copy()
    ref.ref_scaley(_p(r), _p(spec0), _p(var0))
    for b0 in range(0, B, 8):
        got = oracle.scaley(x[b0:b0 + 8], spec0[b0:b0 + 8], var0[b0:b0 + 8])
        np.testing.assert_array_equal(got, r[b0:b0 + 8])


def test_flag_and_flagts_match_reference(ref, oracle):
    """Column and row replacement by MN x bpwr on a uint8 block."""
    B, T, C = _shape(ref)
    rng = np.random.default_rng(13)
    x = rng.integers(0, 256, (B, T, C), dtype=np.uint8)
    bpwr = rng.uniform(0.5, 3.0, B).astype(np.float32)
    cm = np.zeros((B, C), np.int32)
    cm[:, 200] = 1
    cm[3, 500:503] = 1
    tm = np.zeros((B, T), np.int32)
    tm[:, 77] = 1
    tm[9, 1000:1010] = 1
    cidx = np.nonzero(cm.reshape(-1))[0].astype(np.int32)
    tidx = np.nonzero(tm.reshape(-1))[0].astype(np.int32)
    r = x.copy()
    ref.ref_flag(_p(r), _p(cidx), len(cidx), _p(bpwr))
    ref.ref_flagts(_p(r), _p(tidx), len(tidx), _p(bpwr))
    lev = oracle.repl_level(48.0 * bpwr, np.uint8)
    o = x.copy()
    for b in range(B):
        o[b][:, np.nonzero(cm[b])[0]] = lev[b]
        o[b][np.nonzero(tm[b])[0], 128:C - 128] = lev[b]
    np.testing.assert_array_equal(o, r)


def test_massage_matches_reference(ref_small, oracle):
    """dsaX_reorder_raw.c massage() (byte reorder) on 64 packets, 1 and 4
    threads; the padded antenna 63 is left as it was (zero here)."""
    npk, nant = ref_small.ref_npackets(), ref_small.ref_nants()
    blk = oracle.gen_block(14, npk, nant, 384, "uniform")
    want = oracle.massage(blk)
    for nt in (1, 4):
        out = np.zeros(npk * 768 * 64 * 2, np.uint8)
        assert ref_small.ref_massage_raw(_p(np.ascontiguousarray(blk)), _p(out), nt) == 0
        np.testing.assert_array_equal(out.reshape(want.shape), want)


def test_fluff_reorder_matches_reference(ref_small, oracle):
    """dsaX_reorder_raw.c.bak massage() (AVX-512 fluff + 32-bit transpose)."""
    if " avx512bw" not in open("/proc/cpuinfo").read():
        pytest.skip("host CPU has no AVX-512BW")
    npk, nant = ref_small.ref_npackets(), ref_small.ref_nants()
    blk = oracle.gen_block(15, npk, nant, 384, "uniform")
    want = oracle.fluff_reorder(blk)
    for nt in (1, 4):
        out = np.zeros(npk * 768 * 64 * 4, np.int8)
        assert ref_small.ref_massage_bak(_p(np.ascontiguousarray(blk)), _p(out), nt) == 0
        np.testing.assert_array_equal(out.reshape(want.shape), want)


def test_simple_extract_matches_reference(ref, oracle):
    rng = np.random.default_rng(16)
    vis = rng.integers(-3000, 3000, (768, 2080, 4, 2)).astype(np.float32)
    out = np.zeros(2080 * 384 * 2 * 2, np.float32)
    ref.ref_simple_extract(_p(vis), _p(out))
    np.testing.assert_array_equal(oracle.simple_extract(vis).reshape(-1), out)


def test_auto_extract_matches_reference(ref, oracle):
    rng = np.random.default_rng(17)
    ex = rng.normal(0, 100, (2080, 384, 2, 2)).astype(np.float32)
    specs = rng.normal(0, 10, (63, 384)).astype(np.float32)
    r = specs.copy()
    ref.ref_auto_extract(_p(ex), _p(r))
    np.testing.assert_array_equal(oracle.auto_extract(ex, specs.copy()), r)


def test_greg_order_matches_reference(ref, oracle):
    idx = np.zeros(2080, np.int32)
    ref.ref_gen_lookup(_p(idx))
    np.testing.assert_array_equal(oracle.greg_order(), idx)
    rng = np.random.default_rng(18)
    ex = rng.normal(0, 1, (2080, 1536)).astype(np.float32)
    out = np.zeros_like(ex)
    ref.ref_reorder_gh(_p(ex), _p(out), _p(idx))
    np.testing.assert_array_equal(ex[oracle.greg_order()], out)


def test_two_arm_weights_match_reference(ref, oracle):
    """populate_weights_matrix (src/dsaX_bfCorr.cu:815-863): two arms of 48
    antennas, 256 beams each, the N-S arm's beam angle offset by the
    declination.  The reference evaluates the phase in float: positions
    within +-10 m keep that phase error below 1e-3 rad, and the weights
    (unit magnitude) must agree with the FP64 restatement to 2e-3."""
    na, ng, nbeams = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int())
    ref.ref_bfcorr_shape(ctypes.byref(na), ctypes.byref(ng), ctypes.byref(nbeams))
    na, ng, nbeams = na.value, ng.value, nbeams.value
    rng = np.random.default_rng(19)
    ae = rng.uniform(-10, 10, na).astype(np.float32)
    an = rng.uniform(-10, 10, na).astype(np.float32)
    cal = rng.normal(0, 1, (na, ng, 2, 2)).astype(np.float32)
    flagged = np.zeros(na, np.int32)
    flagged[[3, 60]] = 1
    # the reference's host side (calc_weights, :886-903): unit gains, flagged zero
    calr = cal.copy().reshape(-1, 2)
    nrm = np.sqrt((calr.astype(np.float32) ** 2).sum(axis=1)).astype(np.float32)
    calr = (calr / np.where(nrm == 0, 1, nrm)[:, None]).astype(np.float32)
    calr.reshape(na, ng * 2, 2)[flagged == 1] = 0
    sfreq, dec = 1498.75, 37.23 - 71.6
    fqs = (1e6 * (sfreq - np.arange(ng) * 250.0 / 1024.0)).astype(np.float32)
    n = 2 * ng * (nbeams // 2) * 4 * (na // 2) * 8 * 2 * 2
    wr = np.zeros(n, np.float32)
    wi = np.zeros(n, np.float32)
    ref.ref_populate_weights(_p(ae), _p(an), _p(np.ascontiguousarray(calr.reshape(-1))), _p(wr),
                             _p(wi), _p(fqs), float(dec))
    shp = (2, ng, nbeams // 2, 4, na // 2, 8, 2, 2)
    wr, wi = wr.reshape(shp), wi.reshape(shp)
    arm = np.repeat([0, 1], na // 2)
    ore, oim = oracle.two_arm_weights(ae.astype(np.float64), an.astype(np.float64), arm, cal,
                                      flagged, ng, nbeams, sfreq, 1.0, dec, pi=3.14159265359)
    for A in (0, 1):
        for pol in (0, 1):
            got = wr[A, :, :, 0, :, 0, 0, pol] + 1j * wi[A, :, :, 0, :, 0, 0, pol]  # [g][b][a]
            want = (ore[:, pol, A * nbeams // 2:(A + 1) * nbeams // 2, A * na // 2:(A + 1) * na // 2]
                    + 1j * oim[:, pol, A * nbeams // 2:(A + 1) * nbeams // 2,
                               A * na // 2:(A + 1) * na // 2])
            assert np.abs(got - want).max() < 2e-3
            # the replicated time/channel copies are identical
            assert np.array_equal(wr[A, :, :, 3, :, 7, 1, pol], wr[A, :, :, 0, :, 0, 0, pol])

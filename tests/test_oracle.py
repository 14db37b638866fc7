"""CPU tests of the oracle against the reference's golden vectors and
brute-force restatements (no GPU)."""
import base64
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


# ---------------------------------------------------------------- decode
def test_decode_matches_reference_decoder(oracle):
    """utils/packet.out decoded by the oracle reproduces what the reference's
    make_spectrum / make_histogram (utils/gen_packet.py:15-67) returned."""
    g = _load("packet_decode.json")
    pkt = np.frombuffer(base64.b64decode(g["packet_b64"]), dtype=np.uint8)
    assert hashlib.sha256(pkt.tobytes()).hexdigest() == g["sha256"]
    re, im = oracle.unpack4(pkt)
    re = re.astype(np.float64).reshape(3, 384, 2, 2)
    im = im.astype(np.float64).reshape(3, 384, 2, 2)
    for key, spec in g["spectra"].items():
        ant, pol = map(int, key.split(","))
        mine = (re[ant, :, :, pol] ** 2 + im[ant, :, :, pol] ** 2).mean(axis=1)
        np.testing.assert_allclose(mine, np.array(spec), rtol=0, atol=1e-12)
    # histogram of all 2*768 values of antenna-major order as make_histogram
    # (it histograms the first 768 entries of the flattened packet only)
    flat_r = re.reshape(-1)[:768]
    flat_i = im.reshape(-1)[:768]
    h = np.zeros(16)
    for v in np.concatenate([flat_r, flat_i]):
        h[int(v) + 8] += 1
    np.testing.assert_allclose(h / h.max(), np.array(g["hist_norm"]), atol=1e-12)
    rms = np.sqrt(0.5 * (np.std(re.reshape(-1)) ** 2 + np.std(im.reshape(-1)) ** 2))
    assert abs(rms - g["rms"]) < 1e-12


def test_promote_matches_nibble_rule(oracle):
    """promoter (src/dsaX_xgpu.cu:67-77): low nibble -> out[2i], high -> out[2i+1]."""
    allb = np.arange(256, dtype=np.uint8)
    out = oracle.promote(allb).reshape(256, 2)
    for b in range(256):
        lo, hi = b & 15, b >> 4
        assert out[b, 0] == (lo - 16 if lo >= 8 else lo)
        assert out[b, 1] == (hi - 16 if hi >= 8 else hi)


# ---------------------------------------------------------------- reorder
def _tone_block(desc):
    """One packet [1][63][384][2][2] with the tone of utils/test.out."""
    blk = np.zeros((1, desc["nant_in"], 384, 2, 2), dtype=np.uint8)
    for a in range(desc["nant_in"]):
        if a % 3 != desc["ants_mod3"]:
            continue
        for c in desc["chans"]:
            for t in desc["times"]:
                blk[0, a, c, t, 0] = oracle_pack(desc["pol0_re"], desc["imag"])
                blk[0, a, c, t, 1] = oracle_pack(desc["pol1_re"], desc["imag"])
    return blk


def oracle_pack(re, im):
    return (re & 15) | ((im & 15) << 4)


def test_reorder_reproduces_reference_test_out(oracle):
    """The fluff + transpose of the tone packet equals utils/test.out byte
    for byte (src/dsaX_reorder_raw.c.bak:304-339 wrote it)."""
    g = _load("reorder_tone.json")
    out = oracle.fluff_reorder(_tone_block(g["tone"]))
    assert out.shape == (1, 768, 64, 2, 2)
    assert hashlib.sha256(out.tobytes()).hexdigest() == g["sha256"]
    want = np.zeros((768, 64, 2, 2), np.int8)
    for k, a, p, c, v in g["nonzero"]:
        want[k, a, p, c] = v
    np.testing.assert_array_equal(out[0], want)


def test_massage_then_promote_equals_fluff(oracle):
    blk = oracle.gen_block(3, 8, 63, 16, "uniform")
    ms = oracle.massage(blk)
    assert ms.shape == (8, 32, 64, 2)
    assert not ms[:, :, 63].any()  # padded antenna zero-filled
    np.testing.assert_array_equal(oracle.promote(ms).reshape(8, 32, 64, 2, 2),
                                  oracle.fluff_reorder(blk))


def test_ramp_block_decode(oracle):
    """utils/gen_testblock.py:48-69 restated: real = 32*((j%9)-5+(i+p-3)) as
    int8 (wrapping), keep the top nibble; imag 0.  Decoding returns
    ((2s + 8) mod 16) - 8 with s = (j%9)-5+(i+p-3)."""
    npk, nant, nch = 4, 96, 384
    blk = np.zeros((npk, nant, nch, 2, 2), np.uint8)
    exp = np.zeros((npk, nant, nch), np.int16)
    for p in range(npk):
        for a in range(nant):
            i = a % 3
            for j in range(nch):
                s = (j % 9) - 5 + (i + p - 3)
                v8 = ((32 * s + 128) % 256) - 128
                blk[p, a, j, :, :] = (v8 & 0xFF) >> 4
                exp[p, a, j] = ((2 * s + 8) % 16) - 8
    re, im = oracle.unpack4(blk)
    np.testing.assert_array_equal(re[..., 0, 0], exp)
    assert not im.any()


# ---------------------------------------------------------------- correlator
def _brute_vis(blk):
    re, im = [v.astype(np.int64) for v in __import__("oracle").unpack4(blk)]
    npkt, nant, nch = blk.shape[:3]
    x = np.zeros((npkt, 64, nch, 2, 2), complex)
    x[:, :nant] = re + 1j * im
    out = np.zeros((2 * nch, 2080, 4, 2), np.float32)
    for c in range(nch):
        for t in range(2):
            X = x[:, :, c, t, :].reshape(npkt, 128)
            V = X.T @ X.conj()
            for i in range(64):
                for j in range(i + 1):
                    bl = i * (i + 1) // 2 + j
                    blockv = V[2 * i:2 * i + 2, 2 * j:2 * j + 2].reshape(4)
                    out[2 * c + t, bl, :, 0] = blockv.real
                    out[2 * c + t, bl, :, 1] = blockv.imag
    return out


@pytest.mark.parametrize("npkt,nant,nch", [(16, 63, 3), (37, 64, 2), (1, 5, 1)])
def test_correlate_matches_bruteforce(oracle, npkt, nant, nch):
    blk = oracle.gen_block(npkt * 7 + nant, npkt, nant, nch, "uniform")
    np.testing.assert_array_equal(oracle.correlate(blk), _brute_vis(blk))


def test_correlate_conjugation_convention(oracle):
    """V_ij = sum x_i conj(x_j) for i >= j (the reference's own restatement,
    src/dsaX_bfCorr.cu:442-447,509-552): with x_1 = 1 and x_0 = i,
    V_10 = 1 * conj(i) = -i."""
    blk = np.zeros((1, 2, 1, 2, 2), np.uint8)
    blk[0, 0, 0, 0, 0] = oracle_pack(0, 1)   # station 0 pol 0: +i
    blk[0, 1, 0, 0, 0] = oracle_pack(1, 0)   # station 1 pol 0: 1
    vis = oracle.correlate(blk)
    bl10 = 1 * 2 // 2 + 0
    assert tuple(vis[0, bl10, 0]) == (0.0, -1.0)
    assert tuple(vis[0, 0, 0]) == (1.0, 0.0)   # auto of station 0
    assert tuple(vis[0, 2, 0]) == (1.0, 0.0)   # auto of station 1


def test_correlate_channel_subset(oracle):
    blk = oracle.gen_block(5, 12, 63, 10, "gauss")
    full = oracle.correlate(blk)
    np.testing.assert_array_equal(oracle.correlate(blk, ch0=3, nch=4), full[6:14])


def test_xengine_int8_equals_correlate(oracle):
    blk = oracle.gen_block(9, 20, 63, 6, "gauss")
    fl = oracle.fluff_reorder(blk)
    np.testing.assert_array_equal(oracle.xengine_int8(fl.reshape(20, 12, 64, 2, 2)),
                                  oracle.correlate(blk))


def test_simple_extract(oracle):
    """src/dsaX_writevis.c:55-74: XX/YY averaged over the 2 time slots."""
    blk = oracle.gen_block(2, 8, 63, 4, "gauss")
    vis = oracle.correlate(blk)
    ex = oracle.simple_extract(vis)
    for bl in (0, 5, 2079):
        for pol in range(2):
            for f in range(4):
                pp = 3 * pol
                want = 0.5 * (vis[2 * f, bl, pp] + vis[2 * f + 1, bl, pp])
                np.testing.assert_allclose(ex[bl, f, pol], want)


# ---------------------------------------------------------------- beamformer
def test_beamform_oracle_bruteforce(oracle):
    npkt, nant, nch, nbeam, ppo = 8, 63, 16, 8, 4
    blk = oracle.gen_block(11, npkt, nant, nch, "gauss")
    wre, wim = oracle.random_phase_weights(4, nch // 8, nbeam)
    pw = oracle.beamform_power(blk, wre, wim, pkt_per_out=ppo)
    re, im = oracle.unpack4(blk)
    x = np.zeros((npkt, 64, nch, 2, 2), complex)
    x[:, :nant] = re + 1j * im
    w = wre + 1j * wim  # [g][pol][b][a]
    want = np.zeros((npkt // ppo, nbeam, nch // 8))
    for g in range(nch // 8):
        for pol in range(2):
            xs = x[:, :, 8 * g:8 * g + 8, :, pol]            # [p][a][c][t]
            beam = np.einsum("ba,pact->pbct", w[g, pol], xs)  # no conjugate
            pwr = (np.abs(beam) ** 2).sum(axis=(2, 3))       # [p][b]
            want[:, :, g] += pwr.reshape(npkt // ppo, ppo, nbeam).sum(axis=1)
    np.testing.assert_allclose(pw, want, rtol=1e-12, atol=1e-9)


def test_geometric_weights_formula(oracle):
    """calc_weights (src/dsaX_beamformer.cu:421-449) in FP64."""
    rng = np.random.default_rng(0)
    pos = rng.uniform(-500, 500, 64)
    cal = rng.normal(size=(64, 2, 2, 2))
    flagged = np.zeros(64, np.int32)
    flagged[5] = 1
    wre, wim = oracle.geometric_weights(pos, cal, flagged, 2, 256)
    g, pol, b, a = 1, 0, 37, 9
    c = cal[a, g, pol, 0] + 1j * cal[a, g, pol, 1]
    c = c / abs(c) ** 2
    nu = (1530.0 - (8 * g + 4) * 250.0 / 8192.0) * 1e6
    theta = (127 - b) * np.pi / 10800.0
    afac = -2 * np.pi * nu * theta / 299792458.0
    w = np.exp(1j * afac * pos[a]) * c
    assert abs(wre[g, pol, b, a] - w.real) < 1e-12 and abs(wim[g, pol, b, a] - w.imag) < 1e-12
    assert not wre[:, :, :, 5].any() and not wim[:, :, :, 5].any()


# ---------------------------------------------------------------- flagger
def test_plain_flagger_finds_injected_tone(oracle):
    rng = np.random.default_rng(1)
    B, T, C = 4, 1024, 48
    x = rng.exponential(2.0, size=(B, T, C)).astype(np.float32)
    x[2, :, 20] += 3.0          # persistent narrowband tone
    x[1, 500:503, :] += 40.0    # broadband burst
    p = oracle.flag_params(B, T, C, tbin=32)
    cm, tm, _, _, st = oracle.plain_flag(x, p)
    assert cm[2, 20] == 1
    assert tm[1, 500:503].all()
    assert cm.sum() < 0.2 * B * C
    np.testing.assert_allclose(st["spec"], x.mean(axis=1), rtol=1e-5)
    np.testing.assert_allclose(st["var"], x.var(axis=1), rtol=1e-4)
    # the series is formed after the flagged columns are set to MN = 48, as
    # flag() runs before make_ts (src/gpu_flagger.cu:1379-1386)
    xr = x.copy()
    for b in range(B):
        xr[b][:, cm[b] == 1] = 48.0
    np.testing.assert_allclose(st["ts"], xr.mean(axis=2), rtol=1e-5)


def test_plain_flagger_parity_quirks(oracle):
    """Parity mode: max spectrum = mean (src/gpu_flagger.cu:1334) and the
    FBIN boxcar of simple_channflag reads spec[j] only (:594)."""
    rng = np.random.default_rng(2)
    x = rng.exponential(2.0, size=(2, 256, 48)).astype(np.float32)
    _, _, _, _, st = oracle.plain_flag(x, oracle.flag_params(2, 256, 48, tbin=32, parity=1))
    np.testing.assert_array_equal(st["max"], st["spec"])
    _, _, _, _, st2 = oracle.plain_flag(x, oracle.flag_params(2, 256, 48, tbin=32, parity=0))
    np.testing.assert_allclose(st2["max"], x.max(axis=1))

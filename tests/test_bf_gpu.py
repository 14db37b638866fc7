"""GPU tests of the tcgen05 BF16 beamformer through the C-ABI against the
FP64 oracle.  Tolerances: FP32 power within 5e-3 relative of FP64 -- the
BF16 weight rounding bounds the power error by 2 * 2^-9 = 3.9e-3 when one
antenna dominates a beam (geometric x calibration weights), and averages to
well under 1e-3 for unit-magnitude weights; uint8 Stokes-I within 1 LSB of
the FP64 oracle quantised the same way."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 5e-3
MEAN_TOL = 1e-3


def _beamform(dsax, blk, wre, wim, nbeam, ppo, scale, ctx=None, set_w=True, bf_path=0, fp8=0,
              bf_variant=0):
    import torch
    npkt, nant, nchan = blk.shape[:3]
    cfg = dsax.default_config(npkt=npkt, nant_in=nant, nchan=nchan, nbeam=nbeam,
                              bf_pkt_per_out=ppo, bf_scale=scale, bf_path=bf_path, bf_fp8=fp8,
                              bf_variant=bf_variant)
    own = ctx is None
    ctx = ctx or dsax.Context(cfg)
    try:
        if set_w:
            ctx.set_weights(wre, wim)
        d_in = torch.from_numpy(blk.reshape(-1)).cuda()
        nout = (npkt // ppo) * nbeam * (nchan // 8)
        u8 = torch.zeros(nout, dtype=torch.uint8, device="cuda")
        f32 = torch.zeros(nout, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.beamform(d_in, u8, f32)
        ctx.sync()
        shp = (npkt // ppo, nbeam, nchan // 8)
        return u8.cpu().numpy().reshape(shp), f32.cpu().numpy().reshape(shp)
    finally:
        if own:
            ctx.close()


def _check(oracle, blk, wre, wim, u8, f32, ppo, scale, g0=0, ng=None):
    ng = f32.shape[2] - g0 if ng is None else ng
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=ppo, g0=g0, ng=ng)
    got = f32[:, :, g0:g0 + ng].astype(np.float64)
    rel = np.abs(got - ref) / np.maximum(ref, 1e-30)
    assert rel.max() < REL_TOL, f"max rel err {rel.max():.3e}"
    assert rel.mean() < MEAN_TOL, f"mean rel err {rel.mean():.3e}"
    ref_u8 = oracle.quantize_u8(ref, scale)
    diff = np.abs(u8[:, :, g0:g0 + ng].astype(int) - ref_u8.astype(int))
    assert diff.max() <= 1, f"uint8 off by {diff.max()}"
    return rel, diff


def test_beamformer_config3_full_block(dsax, oracle):
    """Full-size block: 64 ants (63 populated) x 2 pols x 384 ch x 4096 t,
    256 beams, unit-magnitude random-phase weights, 32 t x 8 ch sums; every
    one of the 128 x 256 x 48 outputs against the FP64 oracle."""
    blk = oracle.gen_block(303, 2048, 63, 384, "gauss")
    wre, wim = oracle.random_phase_weights(9, 48, 256)
    scale = 128.0 / (512 * 64 * 2 * 6.25)   # E[P] = 512 samples x 64 ants x E|x|^2
    u8, f32 = _beamform(dsax, blk, wre, wim, 256, 16, scale)
    assert f32.shape == (128, 256, 48)
    rel, diff = _check(oracle, blk, wre, wim, u8, f32, 16, scale)
    assert np.median(u8) > 60 and np.median(u8) < 200   # fixed scaling lands mid-range


@pytest.mark.parametrize("bf_path", [1, 2])
@pytest.mark.parametrize("nbeam,ppo,npkt,nant,nchan", [(64, 16, 32, 63, 8), (128, 4, 64, 64, 16),
                                                       (256, 8, 48, 63, 8), (192, 32, 64, 40, 24),
                                                       (256, 32, 96, 40, 24), (512, 16, 32, 63, 16)])
def test_beamformer_shapes(dsax, oracle, nbeam, ppo, npkt, nant, nchan, bf_path):
    blk = oracle.gen_block(nbeam + ppo + npkt, npkt, nant, nchan, "gauss")
    wre, wim = oracle.random_phase_weights(nbeam, nchan // 8, nbeam)
    scale = 128.0 / (2 * ppo * 16 * nant * 2 * 6.25 * 0.93)
    u8, f32 = _beamform(dsax, blk, wre, wim, nbeam, ppo, scale, bf_path=bf_path)
    _check(oracle, blk, wre, wim, u8, f32, ppo, scale)


@pytest.mark.parametrize("fp8", [0, 1])
def test_beamformer_paths_agree_full_block(dsax, oracle, fp8):
    """The CTA-pair kernel (cta_group::2), with each of its stage-parameter
    variants, against the one-CTA kernel on a full block, BF16 and FP8: the
    same products, the epilogue's partial sums added in another order, so
    FP32 power within 1e-5 relative and uint8 within 1 LSB."""
    blk = oracle.gen_block(304, 2048, 63, 384, "gauss")
    wre, wim = oracle.random_phase_weights(10, 48, 256)
    scale = 128.0 / (512 * 64 * 2 * 6.25)
    u8a, fa = _beamform(dsax, blk, wre, wim, 256, 16, scale, bf_path=1, fp8=fp8)
    for v in (1, 2, 3, 4):
        u8b, fb = _beamform(dsax, blk, wre, wim, 256, 16, scale, bf_path=2, fp8=fp8, bf_variant=v)
        rel = np.abs(fb.astype(np.float64) - fa) / np.maximum(fa, 1e-30)
        assert rel.max() < 1e-5, (v, rel.max())
        assert np.abs(u8b.astype(int) - u8a.astype(int)).max() <= 1, v


def test_beamformer_geometric_weights(dsax, oracle):
    """calc_weights geometry with calibration and a flagged antenna."""
    rng = np.random.default_rng(3)
    pos = rng.uniform(-600, 600, 64)
    cal = rng.normal(size=(64, 2, 2, 2))
    flagged = np.zeros(64, np.int32)
    flagged[[3, 40]] = 1
    wre, wim = oracle.geometric_weights(pos, cal, flagged, 2, 256)
    blk = oracle.gen_block(77, 64, 63, 16, "gauss")
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=16)
    scale = 128.0 / float(np.median(ref))
    u8, f32 = _beamform(dsax, blk, wre, wim, 256, 16, scale)
    _check(oracle, blk, wre, wim, u8, f32, 16, scale)
    # the library's own FP64 weight generation gives the same beams
    cfg = dsax.default_config(npkt=64, nant_in=63, nchan=16, nbeam=256, bf_pkt_per_out=16,
                              bf_scale=scale)
    with dsax.Context(cfg) as ctx:
        ctx.set_geometric_weights(pos, cal, flagged)
        u8b, f32b = _beamform(dsax, blk, wre, wim, 256, 16, scale, ctx=ctx, set_w=False)
    np.testing.assert_array_equal(f32b, f32)
    np.testing.assert_array_equal(u8b, u8)


def test_beamformer_two_arm_declination_weights(dsax, oracle):
    """The cuBLAS beamformer's two-arm weights (E-W arm beams from
    eastings, N-S arm beams from northings with the declination offset) on
    the tcgen05 beamformer: 256 beams, 32 antennas per arm, against the FP64
    oracle with the same weights; the library's FP64 generation must match
    the oracle's weights image exactly."""
    rng = np.random.default_rng(31)
    ae = rng.uniform(-400, 400, 64)
    an = rng.uniform(-400, 400, 64)
    arm = np.repeat([0, 1], 32)
    arm[63] = -1                                   # the padded antenna
    cal = rng.normal(size=(64, 2, 2, 2))
    flagged = np.zeros(64, np.int32)
    flagged[[5, 44]] = 1
    sfreq, dec = 1498.75, 37.23 - 52.0
    wre, wim = oracle.two_arm_weights(ae, an, arm, cal, flagged, 2, 256, sfreq, 1.0, dec)
    blk = oracle.gen_block(78, 64, 63, 16, "gauss")
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=16)
    scale = 128.0 / float(np.median(ref))
    u8, f32 = _beamform(dsax, blk, wre, wim, 256, 16, scale)
    _check(oracle, blk, wre, wim, u8, f32, 16, scale)
    cfg = dsax.default_config(npkt=64, nant_in=63, nchan=16, nbeam=256, bf_pkt_per_out=16,
                              bf_scale=scale)
    with dsax.Context(cfg) as ctx:
        ctx.set_two_arm_weights(ae, an, arm, cal, flagged, sfreq, 1.0, dec)
        u8b, f32b = _beamform(dsax, blk, wre, wim, 256, 16, scale, ctx=ctx, set_w=False)
    np.testing.assert_array_equal(f32b, f32)
    np.testing.assert_array_equal(u8b, u8)


def test_beamformer_single_antenna_tone(dsax, oracle):
    """Only antenna 7 carries a constant 3+2i and weights pick it with
    magnitude 1: every beam's power is |3+2i|^2 x samples."""
    blk = np.zeros((16, 63, 8, 2, 2), np.uint8)
    blk[:, 7] = (3 & 15) | ((2 & 15) << 4)
    wre = np.zeros((1, 2, 64, 64)); wim = np.zeros_like(wre)
    ph = np.linspace(0, 2 * np.pi, 64, endpoint=False)
    wre[:, :, :, 7] = np.cos(ph)[None, None, :]
    wim[:, :, :, 7] = np.sin(ph)[None, None, :]
    u8, f32 = _beamform(dsax, blk, wre, wim, 64, 16, 1.0)
    want = 13.0 * 16 * 16 * 2
    np.testing.assert_allclose(f32, want, rtol=REL_TOL)
    assert (u8 == 255).all()   # saturates instead of wrapping


def test_agc_bandpass_sequence(dsax, oracle):
    """Eleven blocks through the AGC: the per-beam scales after every block
    against the oracle's restatement (median phase, then the 8-block mean
    with the 10 % clamp -- block 9 at twice the amplitude drives beams into
    the clamp), and the uint8 beams of each block quantised with the
    previous scale (zeros for the first block) within 1 LSB."""
    import torch
    npkt, nant, nchan, nbeam, ppo = 64, 63, 16, 256, 16
    wre, wim = oracle.random_phase_weights(77, nchan // 8, nbeam)
    cfg = dsax.default_config(npkt=npkt, nant_in=nant, nchan=nchan, nbeam=nbeam,
                              bf_pkt_per_out=ppo)
    ref = oracle.AgcOracle(nbeam, nchan // 8, npkt // 16)
    clamped = 0
    with dsax.Context(cfg) as ctx:
        ctx.set_weights(wre, wim)
        ctx.agc_enable(1)
        for k in range(11):
            blk = oracle.gen_block(900 + k, npkt, nant, nchan, "gauss", sigma=5.0 if k == 9 else 2.5)
            d_in = torch.from_numpy(blk.reshape(-1)).cuda()
            u8 = torch.zeros((npkt // ppo) * nbeam * (nchan // 8), dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            prev = ref.scale.copy()
            ctx.beamform(d_in, u8)
            scale, started, nblk = ctx.agc_state()
            pw = oracle.beamform_power(blk, wre, wim, pkt_per_out=ppo)
            want_u8 = oracle.quantize_u8_agc(pw, prev)
            got_u8 = u8.cpu().numpy().reshape(want_u8.shape)
            assert np.abs(got_u8.astype(int) - want_u8.astype(int)).max() <= 1
            if k == 0:
                assert got_u8.max() == 0
            want = ref.update(pw.sum(axis=(0, 2)))
            assert nblk == k + 1 and started == ref.started
            np.testing.assert_allclose(scale, want, rtol=2e-3)
            if k >= 8:
                clamped += int(np.sum(np.abs(ref.hist.mean(axis=0) - ref.medbp) / ref.medbp > 0.1))
    assert clamped > 0


@pytest.mark.parametrize("bf_path", [1, 2])
@pytest.mark.parametrize("weights", ["unit", "calibrated"])
def test_beamformer_fp8(dsax, oracle, weights, bf_path):
    """FP8 E4M3 operands (kind::f8f6f4) with the per-antenna power-of-two
    scale, one CTA per beam tile (bf_path 1) and CTA pairs (2; calibrated:
    gains spread over e^6 between antennas): against the FP64
    oracle run with the same E4M3-rounded
    weights the FP32 power agrees to 1e-4 (the data are exact in E4M3 and
    the products exact in FP32); against the unrounded FP64 weights the
    error is the weight rounding (3 mantissa bits), reported and bounded."""
    import torch
    npkt, nant, nchan, nbeam, ppo = 64, 63, 16, 256, 16
    if weights == "unit":
        wre, wim = oracle.random_phase_weights(51, nchan // 8, nbeam)
    else:
        rng = np.random.default_rng(8)
        cal = rng.normal(size=(64, nchan // 8, 2, 2)) * np.exp(rng.uniform(-3, 3, 64))[:, None, None, None]
        wre, wim = oracle.geometric_weights(rng.uniform(-600, 600, 64), cal, np.zeros(64, np.int32),
                                            nchan // 8, nbeam)
    qre, qim, d, _ = oracle.fp8_weights(wre, wim)
    # unit weights share one exponent (no data shift); calibrated gains
    # spread over e^6 exercise the per-antenna shift
    assert np.any(d != 0) == (weights == "calibrated")
    # uniform data: every 4-bit value, -8 included, in every nibble position
    blk = oracle.gen_block(61, npkt, nant, nchan, "uniform" if weights == "unit" else "gauss")
    ref_q = oracle.beamform_power(blk, qre, qim, pkt_per_out=ppo)
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=ppo)
    scale = 128.0 / float(np.median(ref))
    cfg = dsax.default_config(npkt=npkt, nant_in=nant, nchan=nchan, nbeam=nbeam,
                              bf_pkt_per_out=ppo, bf_scale=scale, bf_fp8=1, bf_path=bf_path)
    with dsax.Context(cfg) as ctx:
        ctx.set_weights(wre, wim)
        d_in = torch.from_numpy(blk.reshape(-1)).cuda()
        n = ref.size
        u8 = torch.zeros(n, dtype=torch.uint8, device="cuda")
        f32 = torch.zeros(n, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.beamform(d_in, u8, f32)
        ctx.sync()
        got = f32.cpu().numpy().reshape(ref.shape).astype(np.float64)
    rel_q = np.abs(got - ref_q) / np.maximum(ref_q, 1e-30)
    assert rel_q.max() < 1e-4, rel_q.max()
    rel = np.abs(got - ref) / np.maximum(ref, 1e-30)
    print(f"FP8 vs FP64 weights: mean rel {rel.mean():.2e}, max rel {rel.max():.2e}")
    assert rel.mean() < 2e-2


def test_autotune_beamformer_picks_fastest_and_stays_correct(dsax, oracle):
    """dsax_autotune_beamformer times the one-CTA form and the CTA-pair form
    with its four stage-parameter variants on the context's geometry, keeps
    the fastest, and the beams stay within the oracle tolerances
    afterwards."""
    blk = oracle.gen_block(707, 256, 63, 64, "gauss")
    wre, wim = oracle.random_phase_weights(12, 8, 256)
    scale = 128.0 / (2 * 16 * 16 * 63 * 2 * 6.25 * 0.93)
    cfg = dsax.default_config(npkt=256, nant_in=63, nchan=64, bf_scale=scale)
    with dsax.Context(cfg) as ctx:
        ctx.set_weights(wre, wim)
        times, best = ctx.autotune_beamformer(reps=3)
        assert best in (1, 2, 3, 4, 5) and all(t > 0 for t in times.values())
        assert times[best] == min(times.values())
        u8, f32 = _beamform(dsax, blk, wre, wim, 256, 16, scale, ctx=ctx, set_w=False)
    _check(oracle, blk, wre, wim, u8, f32, 16, scale)

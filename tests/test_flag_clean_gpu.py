"""GPU tests of the plain flagger's data path (dsax_flag_clean) through the
C-ABI against the oracle's restatement of src/gpu_flagger.cu's block loop
(oracle.CleanOracle), whose pieces tests/test_ref_pin.py pins to the
reference's own functions.

Per block the cleaned data must be identical (uint8: byte for byte; FP32:
the same values, since both sides evaluate scaley with the same float /
double steps and replace with the same level), and the masks identical
except where the oracle's decision margin is below 1e-4 MAD (a last-bit
difference in an FP64-accumulated statistic could flip those)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MARGIN = 1e-4


def _u8_blocks(seed, nblk, B, T, C):
    """uint8 filterbank blocks: noise around 60 with persistent tones, a
    drifting tone and broadband bursts (the reference's input type)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nblk):
        x = rng.normal(60, 8, (B, T, C))
        for b in range(B):
            for ch in rng.integers(C // 8, C - C // 8, size=2):
                x[b, :, ch] += rng.uniform(20, 60)
            t0 = rng.integers(0, T - 8)
            x[b, t0:t0 + rng.integers(1, 8), :] += rng.uniform(30, 80)
            drift = (C // 4 + (np.arange(T) * (C // 2) // T) + k) % C
            x[b, np.arange(T), drift] += 25
        out.append(np.clip(np.rint(x), 0, 255).astype(np.uint8))
    return out


def _run(dsax, oracle, blocks, params, dtype, mem, **cp):
    odt = np.uint8 if dtype == dsax.DTYPE_U8 else np.float32
    ocl = oracle.CleanOracle(params, dtype=odt, **cp)
    cpp = dsax.flag_clean_params(**{k: v for k, v in cp.items()})
    B, T, C = params.nbeam, params.ntime, params.nchan
    results = []
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        st = ctx.flag_state(params, cpp, dtype)
        try:
            for x in blocks:
                cm = np.zeros((B, C), np.uint8)
                tm = np.zeros((B, T), np.uint8)
                if mem == dsax.MEM_HOST:
                    got = np.ascontiguousarray(x).copy()
                    st.clean(got, cm, tm, mem=dsax.MEM_HOST)
                else:
                    import torch
                    d = torch.from_numpy(np.ascontiguousarray(x).copy()).cuda()
                    dcm = torch.zeros(B * C, dtype=torch.uint8, device="cuda")
                    dtm = torch.zeros(B * T, dtype=torch.uint8, device="cuda")
                    torch.cuda.synchronize()
                    st.clean(d, dcm, dtm, mem=dsax.MEM_DEVICE)
                    ctx.sync()
                    got, cm, tm = d.cpu().numpy(), dcm.cpu().numpy().reshape(B, C), \
                        dtm.cpu().numpy().reshape(B, T)
                info = st.info()
                want, ocm, otm, oinfo, (cmg, tmg) = ocl.step(x)
                results.append((got, cm, tm, info, want, ocm, otm, oinfo, cmg, tmg))
            noise = st.noise()
            base = st.baseline()
        finally:
            st.close()
    return results, noise, base, ocl


def _check_block(r, exact_data=True):
    got, cm, tm, info, want, ocm, otm, oinfo, cmg, tmg = r
    assert bool(info.flagged) == oinfo["flagged"]
    assert bool(info.replaced) == oinfo["replaced"]
    sure_c, sure_t = cmg > MARGIN, tmg > MARGIN
    np.testing.assert_array_equal(cm[sure_c], ocm[sure_c])
    np.testing.assert_array_equal(tm[sure_t], otm[sure_t])
    if sure_c.all() and sure_t.all() and exact_data:
        np.testing.assert_array_equal(got, want)
    else:   # a near-threshold decision differs: the rest of the data agrees
        same = got == want
        assert same.mean() > 0.999
    if oinfo["flagged"]:
        assert info.nchan_flagged == int(cm.sum()) and info.nts_flagged == int(tm.sum())
        np.testing.assert_allclose(info.tpwr, oinfo["tpwr"], rtol=1e-12)


def test_clean_uint8_reference_channels(dsax, oracle):
    """uint8 at the reference's channel count (1024, guard 128), 16 beams x
    2048 samples: two measured blocks build the baseline (fix_zspec +
    median_calc), then four cleaned blocks; the third is given a 5 % power
    step and is replaced by the noise block (modulation check)."""
    B, T, C = 16, 2048, 1024
    p = dsax.flag_params(B, T, C, guard=128, ts_base=128, tsflag=1, parity=1, perm=[10])
    blocks = _u8_blocks(21, 6, B, T, C)
    blocks[4] = np.clip(blocks[4].astype(np.int32) * 21 // 20, 0, 255).astype(np.uint8)
    res, noise, base, ocl = _run(dsax, oracle, blocks, p, dsax.DTYPE_U8, dsax.MEM_DEVICE,
                                 naver=2, mod_thresh=0.02)
    np.testing.assert_allclose(base[0], ocl.spec0, rtol=1e-6)
    np.testing.assert_allclose(base[1], ocl.var0, rtol=1e-5)
    assert np.array_equal(base[0], np.broadcast_to(base[0][:1], base[0].shape))
    # the noise block: same generator; libm and numpy may differ in the last
    # bit of log/cos, which moves a rare sample across a rounding boundary
    nz = oracle.noise_block(1, T, C, dtype=np.uint8)
    assert (np.abs(noise.astype(int) - nz.astype(int)) <= 1).all()
    assert (noise == nz).mean() > 0.9999
    for k, r in enumerate(res):
        if k < 2:   # measured only
            assert not r[3].flagged and np.array_equal(r[0], blocks[k])
            assert r[1].sum() == 0 and r[2].sum() == 0
            continue
        if r[7]["replaced"]:
            assert k in (4, 5)
            assert np.array_equal(r[0], np.broadcast_to(noise, r[0].shape))
            continue
        _check_block(r)
        assert r[1].sum() > 0 and r[2].sum() > 0
    assert res[4][3].replaced == 1 and res[5][3].replaced == 1   # 5 % up, then 5 % back down


def test_clean_fp32_config4_shape(dsax, oracle):
    """FP32 filterbank of the flagger benchmark shape (256 x 4096 x 48):
    baseline from two blocks, then two cleaned blocks with per-beam
    replacement levels from the spectrum (calc_bpwr, pwr = 1)."""
    B, T, C = 256, 4096, 48
    p = dsax.flag_params(B, T, C)
    blocks = [oracle.gen_filterbank(30 + k)[0] for k in range(4)]
    res, _, base, ocl = _run(dsax, oracle, blocks, p, dsax.DTYPE_F32, dsax.MEM_DEVICE,
                             naver=2, pwr=1, mod_thresh=0.5)
    np.testing.assert_allclose(base[0], ocl.spec0, rtol=1e-6)
    for r in res[2:]:
        assert r[3].flagged and not r[3].replaced
        _check_block(r)
        assert r[1].sum() > 0


def test_clean_host_memory_matches_device(dsax, oracle):
    """The host-memory form of dsax_flag_clean gives the same blocks."""
    B, T, C = 8, 1024, 256
    p = dsax.flag_params(B, T, C, guard=32, ts_base=64)
    blocks = _u8_blocks(41, 3, B, T, C)
    rh, *_ = _run(dsax, oracle, blocks, p, dsax.DTYPE_U8, dsax.MEM_HOST, naver=1,
                  mod_thresh=1.0)
    rd, *_ = _run(dsax, oracle, blocks, p, dsax.DTYPE_U8, dsax.MEM_DEVICE, naver=1,
                  mod_thresh=1.0)
    for a, b in zip(rh, rd):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[2], b[2])
    for r in rh[1:]:
        _check_block(r)


def test_clean_set_baseline_starts_flagging(dsax, oracle):
    """A saved baseline (the reference's specvar0.dat) turns flagging on
    from the first block."""
    B, T, C = 8, 1024, 128
    p = dsax.flag_params(B, T, C, guard=16, ts_base=64)
    x = _u8_blocks(51, 1, B, T, C)[0]
    s0 = np.full((B, C), 60.0, np.float32)
    v0 = np.full((B, C), 64.0, np.float32)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        with ctx.flag_state(p, dsax.flag_clean_params(), dsax.DTYPE_U8) as st:
            st.set_baseline(s0, v0)
            got = x.copy()
            cm = np.zeros((B, C), np.uint8)
            tm = np.zeros((B, T), np.uint8)
            st.clean(got, cm, tm, mem=dsax.MEM_HOST)
            inf = st.info()
    ocl = oracle.CleanOracle(p, dtype=np.uint8)
    ocl.spec0, ocl.var0, ocl.started = s0, v0, True
    want, ocm, otm, oinfo, (cmg, tmg) = ocl.step(x)
    assert inf.flagged and not inf.replaced and inf.prev_tpwr == 0.0
    _check_block((got, cm, tm, inf, want, ocm, otm, oinfo, cmg, tmg))


def test_stateless_flag_reference_channels(dsax, oracle):
    """dsax_flag (masks only, FP32) at 1024 channels: eight channel slabs
    per beam, the series built from the flagged-column-replaced data."""
    B, T, C = 8, 2048, 1024
    blocks = _u8_blocks(61, 1, B, T, C)
    x = blocks[0].astype(np.float32)
    pd = dsax.flag_params(B, T, C, guard=128, ts_base=128)
    po = oracle.flag_params(B, T, C, guard=128, ts_base=128)
    cm = np.zeros((B, C), np.uint8)
    tm = np.zeros((B, T), np.uint8)
    st = np.zeros(4 * B * C + B * T, np.float32)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        ctx.flag(pd, x, cm, tm, stats=st, mem=dsax.MEM_HOST)
    ocm, otm, cmg, tmg, ost = oracle.plain_flag(x, po)
    bc = B * C
    np.testing.assert_allclose(st[:bc].reshape(B, C), ost["spec"], rtol=1e-6)
    np.testing.assert_allclose(st[bc:2 * bc].reshape(B, C), ost["var"], rtol=1e-5)
    np.testing.assert_allclose(st[4 * bc:].reshape(B, T), ost["ts"], rtol=1e-6)
    sure_c, sure_t = cmg > MARGIN, tmg > MARGIN
    np.testing.assert_array_equal(cm[sure_c], ocm[sure_c])
    np.testing.assert_array_equal(tm[sure_t], otm[sure_t])
    assert cm.sum() > 0 and tm.sum() > 0

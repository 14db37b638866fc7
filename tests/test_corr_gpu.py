"""GPU parity tests of the tcgen05 correlator through the C-ABI, against the
CPU oracle.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(dsax, blk, fmt=0, nant_in=None, ctx=None, accumulate=False, vis=None, corr_path=0):
    import torch
    npkt = blk.shape[0]
    nchan = blk.shape[2] if fmt == 0 else (blk.shape[0] if fmt == 3 else blk.shape[1] // 2)
    npkt = blk.shape[1] if fmt == 3 else npkt
    nant = blk.shape[1] if fmt == 0 else 64
    cfg = dsax.default_config(npkt=npkt, nant_in=nant if nant_in is None else nant_in, nchan=nchan,
                              corr_path=corr_path)
    own = ctx is None
    ctx = ctx or dsax.Context(cfg)
    try:
        d_in = torch.from_numpy(np.ascontiguousarray(blk).view(np.uint8).reshape(-1)).cuda()
        if vis is None:
            vis = torch.zeros(2 * nchan * 2080 * 8, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.correlate(d_in, vis, dsax.MEM_DEVICE, fmt=fmt, accumulate=accumulate)
        ctx.sync()
        return vis.cpu().numpy().reshape(2 * nchan, 2080, 4, 2)
    finally:
        if own:
            ctx.close()


@pytest.mark.parametrize("corr_path", [1, 2, 3, 4, 5, 6, 7])
def test_config1_small_uniform_bit_exact(dsax, oracle, corr_path):
    """64 dual-pol antennas, 48 channels, 2048 packets (xGPU NTIME), samples
    uniform on [-8, 7]: whole output bit-exact (fused and corner-turn paths)."""
    blk = oracle.gen_block(101, 2048, 64, 48, "uniform")
    np.testing.assert_array_equal(_run(dsax, blk, corr_path=corr_path), oracle.correlate(blk))


def test_reorder_matches_massage(dsax, oracle):
    """GPU corner turn == massage() of src/dsaX_reorder_raw.c:153-169 (with
    the padded antenna zeroed), byte for byte, including a channel count
    that is not a multiple of the 32-channel tile."""
    import torch
    for npkt, nant, nch in ((64, 63, 384), (5, 63, 40), (3, 64, 7)):
        blk = oracle.gen_block(npkt * nch, npkt, nant, nch, "uniform")
        cfg = dsax.default_config(npkt=npkt, nant_in=nant, nchan=nch)
        with dsax.Context(cfg) as ctx:
            d_in = torch.from_numpy(blk.reshape(-1)).cuda()
            out = torch.full((npkt * 2 * nch * 64 * 2,), 0xAB, dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            ctx.reorder(d_in, out)
            ctx.sync()
            got = out.cpu().numpy().reshape(npkt, 2 * nch, 64, 2)
        np.testing.assert_array_equal(got, oracle.massage(blk))


_FULL = {}


def _full_block(oracle):
    """The config-2 block and its oracle visibilities (computed once)."""
    if not _FULL:
        blk = oracle.gen_block(202, 2048, 63, 384, "gauss")
        _FULL["blk"], _FULL["vis"] = blk, oracle.correlate(blk)
    return _FULL["blk"], _FULL["vis"]


@pytest.mark.parametrize("corr_path", [1, 2, 3, 4, 5, 6, 7])
def test_config2_full_block(dsax, oracle, corr_path):
    """Full block [2048][63->64][384][2][2], Gaussian sigma 2.5 clipped to
    [-8, 7]: all 768 frequencies x 2080 baselines x 4 products bit-exact
    against the oracle, plus size-independent properties."""
    blk, want = _full_block(oracle)
    vis = _run(dsax, blk, corr_path=corr_path)
    np.testing.assert_array_equal(vis, want)
    # autocorrelation power of every (freq, station, pol) equals sum |x|^2
    lre, lim = oracle.unpack4(np.arange(256, dtype=np.uint8))
    lut = (lre.astype(np.int16) ** 2 + lim.astype(np.int16) ** 2).astype(np.uint8)
    pw = lut[blk].sum(axis=0, dtype=np.int64)                 # [a][c][t][pol]
    auto = np.array([i * (i + 1) // 2 + i for i in range(64)])
    v = vis.reshape(384, 2, 2080, 4, 2)
    for pol in range(2):
        got = v[:, :, auto[:63], 3 * pol, 0]                  # [c][t][a]
        np.testing.assert_array_equal(got, np.transpose(pw[..., pol], (1, 2, 0)))
        assert not v[:, :, auto, 3 * pol, 1].any()            # autos are real
    # cross-hand autos are conjugates of each other
    np.testing.assert_array_equal(v[:, :, auto, 1, 0], v[:, :, auto, 2, 0])
    np.testing.assert_array_equal(v[:, :, auto, 1, 1], -v[:, :, auto, 2, 1])
    # padded station 63 is all zero
    row63 = np.arange(63 * 64 // 2, 2080)
    assert not v[:, :, row63].any()


def test_formats_agree(dsax, oracle):
    """REORDER-key (massage), xGPU int8 and channel-major inputs give the
    same products."""
    blk = oracle.gen_block(303, 256, 63, 32, "gauss")
    want = oracle.correlate(blk)
    np.testing.assert_array_equal(_run(dsax, blk), want)
    np.testing.assert_array_equal(_run(dsax, oracle.massage(blk), fmt=1), want)
    np.testing.assert_array_equal(_run(dsax, oracle.fluff_reorder(blk), fmt=2), want)
    cm = np.zeros((32, 256, 64, 4), np.uint8)
    cm[:, :, :63] = np.transpose(blk.reshape(256, 63, 32, 4), (2, 0, 1, 3))
    np.testing.assert_array_equal(_run(dsax, cm, fmt=3), want)


def test_corner_turn_chanmajor(dsax, oracle):
    """Channel-major corner turn: [nchan][npkt][64][4 B], padded antenna zero."""
    import torch
    for npkt, nant, nch in ((64, 63, 384), (5, 63, 40), (7, 64, 3)):
        blk = oracle.gen_block(npkt * nch + 1, npkt, nant, nch, "uniform")
        cfg = dsax.default_config(npkt=npkt, nant_in=nant, nchan=nch)
        with dsax.Context(cfg) as ctx:
            d_in = torch.from_numpy(blk.reshape(-1)).cuda()
            out = torch.full((nch * npkt * 64 * 4,), 0xCD, dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            ctx.corner_turn(d_in, out, dsax.FMT_CHANMAJOR)
            ctx.sync()
            got = out.cpu().numpy().reshape(nch, npkt, 64, 4)
        want = np.zeros((nch, npkt, 64, 4), np.uint8)
        want[:, :, :nant] = np.transpose(blk.reshape(npkt, nant, nch, 4), (2, 0, 1, 3))
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("corr_path", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("npkt,nant,nchan", [(4, 63, 8), (100, 63, 5), (64, 1, 1), (1, 64, 3),
                                             (130, 64, 2), (64, 63, 33)])
def test_ragged_shapes(dsax, oracle, npkt, nant, nchan, corr_path):
    blk = oracle.gen_block(npkt + 13 * nant + nchan, npkt, nant, nchan, "uniform")
    np.testing.assert_array_equal(_run(dsax, blk, corr_path=corr_path), oracle.correlate(blk))


@pytest.mark.parametrize("corr_path", [6, 7])
@pytest.mark.parametrize("npkt,nant,nchan", [(4, 63, 8), (100, 63, 4), (64, 1, 4), (1, 64, 4),
                                             (130, 64, 8), (64, 63, 36), (200, 40, 12)])
def test_captured_cluster_ragged_shapes(dsax, oracle, npkt, nant, nchan, corr_path):
    """The fused captured-block feed (clusters of four channel CTAs) on
    shapes that leave TMA boxes partly or wholly past the last packet, and
    odd, even and tiny antenna counts."""
    blk = oracle.gen_block(3 * npkt + 7 * nant + nchan, npkt, nant, nchan, "uniform")
    np.testing.assert_array_equal(_run(dsax, blk, corr_path=corr_path), oracle.correlate(blk))


@pytest.mark.parametrize("corr_path", [3, 4])
def test_more_channels_than_sms_bit_exact(dsax, oracle, corr_path):
    """300 channels: more CTAs than SMs, a partial last wave."""
    npkt, nant, nchan = 64, 63, 300
    blk = oracle.gen_block(31, npkt, nant, nchan, "gauss")
    np.testing.assert_array_equal(_run(dsax, blk, corr_path=corr_path), oracle.correlate(blk))


def test_extreme_values(dsax, oracle):
    """Every sample -8-8i (largest magnitude; -(-8) = 8 in the rotated
    operand) and a block of all +7+7i."""
    for byte in (0x88, 0x77, 0x78, 0x87):
        blk = np.full((2048, 63, 4, 2, 2), byte, np.uint8)
        np.testing.assert_array_equal(_run(dsax, blk), oracle.correlate(blk))


def test_ramp_block(dsax, oracle):
    """Deterministic pattern of utils/gen_testblock.py (4 packets)."""
    npk, nant, nch = 4, 63, 384
    blk = np.zeros((npk, nant, nch, 2, 2), np.uint8)
    for p in range(npk):
        for a in range(nant):
            s = (np.arange(nch) % 9) - 5 + (a % 3 + p - 3)
            blk[p, a, :, :, :] = ((((32 * s + 128) % 256) - 128) & 0xFF)[:, None, None] >> 4
    np.testing.assert_array_equal(_run(dsax, blk), oracle.correlate(blk))


@pytest.mark.parametrize("corr_path,nchan", [(0, 16), (3, 16), (0, 160), (5, 160), (6, 160), (7, 16)])
def test_accumulate_integrates_blocks(dsax, oracle, corr_path, nchan):
    """accumulate=1 adds into vis like xGPU's device integration buffer (160
    channels: more CTAs than SMs)."""
    import torch
    b1 = oracle.gen_block(1, 128, 63, nchan, "gauss")
    b2 = oracle.gen_block(2, 128, 63, nchan, "gauss")
    cfg = dsax.default_config(npkt=128, nant_in=63, nchan=nchan, corr_path=corr_path)
    with dsax.Context(cfg) as ctx:
        vis = torch.zeros(2 * nchan * 2080 * 8, dtype=torch.float32, device="cuda")
        _run(dsax, b1, ctx=ctx, vis=vis, accumulate=True)
        got = _run(dsax, b2, ctx=ctx, vis=vis, accumulate=True)
    np.testing.assert_array_equal(got, oracle.correlate(b1) + oracle.correlate(b2))


def test_host_memory_call(dsax, oracle):
    blk = oracle.gen_block(5, 512, 63, 24, "gauss")
    cfg = dsax.default_config(npkt=512, nant_in=63, nchan=24)
    vis = np.zeros((48, 2080, 4, 2), np.float32)
    with dsax.Context(cfg) as ctx:
        ctx.correlate(blk, vis, dsax.MEM_HOST)
        np.testing.assert_array_equal(vis, oracle.correlate(blk))
        vis2 = np.full_like(vis, 7.0)
        ctx.correlate(blk, vis2, dsax.MEM_HOST)   # overwrites
        np.testing.assert_array_equal(vis2, vis)


def test_misaligned_device_pointer_rejected(dsax):
    import torch
    cfg = dsax.default_config(npkt=64, nant_in=63, nchan=1)
    with dsax.Context(cfg) as ctx:
        buf = torch.zeros(64 * 63 * 4 + 64, dtype=torch.uint8, device="cuda")
        vis = torch.zeros(2 * 2080 * 8, dtype=torch.float32, device="cuda")
        with pytest.raises(dsax.DsaxError) as ei:
            ctx.correlate(buf.data_ptr() + 4, vis)
        assert ei.value.status == dsax.DSAX_ERR_ARG


def test_autotune_picks_fastest_and_stays_exact(dsax, oracle):
    import torch
    blk = oracle.gen_block(606, 256, 63, 64, "gauss")
    cfg = dsax.default_config(npkt=256, nant_in=63, nchan=64)
    with dsax.Context(cfg) as ctx:
        times, best = ctx.autotune(reps=3)
        assert best in (1, 2, 3, 4, 5, 6, 7) and all(t > 0 for t in times.values())
        assert times[best] == min(times.values())
        d_in = torch.from_numpy(blk.reshape(-1)).cuda()
        vis = torch.zeros(128 * 2080 * 8, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.correlate(d_in, vis)
        ctx.sync()
        np.testing.assert_array_equal(vis.cpu().numpy().reshape(128, 2080, 4, 2),
                                      oracle.correlate(blk))


@pytest.mark.parametrize("corr_path", [3, 4, 5, 6])
def test_correlate_many_device_pipelined(dsax, oracle, corr_path):
    """Five blocks through dsax_correlate_many (corner turns overlapped with
    correlations on a side stream): each output bit-exact."""
    import torch
    cfg = dsax.default_config(npkt=256, nant_in=63, nchan=48, corr_path=corr_path)
    blks = [oracle.gen_block(700 + k, 256, 63, 48, "gauss") for k in range(5)]
    with dsax.Context(cfg) as ctx:
        d_in = [torch.from_numpy(b.reshape(-1)).cuda() for b in blks]
        vis = [torch.full((96 * 2080 * 8,), -1.0, dtype=torch.float32, device="cuda")
               for _ in blks]
        torch.cuda.synchronize()
        ctx.correlate_many(d_in, vis)
        ctx.sync()
        for b, v in zip(blks, vis):
            np.testing.assert_array_equal(v.cpu().numpy().reshape(96, 2080, 4, 2),
                                          oracle.correlate(b))


def test_correlate_many_full_blocks_match_single_calls(dsax, oracle):
    """Three full-size blocks [2048][63][384][2][2] through the pipelined
    correlator (corner turn of block i+1 overlapped with the correlation of
    block i) equal, bit for bit, one dsax_correlate call per block; one
    channel per block also against the oracle."""
    import torch
    cfg = dsax.default_config()
    blks = [oracle.gen_block(900 + k, 2048, 63, 384, "gauss") for k in range(3)]
    n = 768 * 2080 * 8
    with dsax.Context(cfg) as ctx:
        d_in = [torch.from_numpy(b.reshape(-1)).cuda() for b in blks]
        many = [torch.full((n,), -1.0, dtype=torch.float32, device="cuda") for _ in blks]
        one = torch.zeros(n, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.correlate_many(d_in, many)
        ctx.sync()
        for k, (b, d, v) in enumerate(zip(blks, d_in, many)):
            ctx.correlate(d, one, dsax.MEM_DEVICE)
            ctx.sync()
            assert torch.equal(v, one), k
            c = 97 * k + 5
            got = v.cpu().numpy().reshape(768, 2080, 4, 2)[2 * c:2 * c + 2]
            np.testing.assert_array_equal(got, oracle.correlate(b, ch0=c, nch=1))


def test_correlate_many_host_pipelined(dsax, oracle):
    """Host buffers in and out (copies overlapped with the device stages)."""
    cfg = dsax.default_config(npkt=128, nant_in=63, nchan=32)
    blks = [oracle.gen_block(800 + k, 128, 63, 32, "uniform") for k in range(4)]
    vis = [np.zeros(64 * 2080 * 8, np.float32) for _ in blks]
    with dsax.Context(cfg) as ctx:
        ctx.correlate_many([np.ascontiguousarray(b.reshape(-1)) for b in blks], vis,
                           mem=dsax.MEM_HOST)
    for b, v in zip(blks, vis):
        np.testing.assert_array_equal(v.reshape(64, 2080, 4, 2), oracle.correlate(b))


def test_extract_and_correlate_extract(dsax, oracle):
    """simple_extract on the GPU (from device visibilities, and fused after
    the correlator with host buffers) against the oracle: bit-exact."""
    import torch
    cfg = dsax.default_config(npkt=128, nant_in=63, nchan=40)
    blk = oracle.gen_block(1300, 128, 63, 40, "gauss")
    want = oracle.simple_extract(oracle.correlate(blk))
    with dsax.Context(cfg) as ctx:
        out = np.zeros(want.size, np.float32)
        ctx.correlate_extract(np.ascontiguousarray(blk.reshape(-1)), out, mem=dsax.MEM_HOST)
        np.testing.assert_array_equal(out.reshape(want.shape), want)
        vis = torch.from_numpy(oracle.correlate(blk).reshape(-1)).cuda()
        dout = torch.zeros(want.size, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.extract(vis, dout)
        ctx.sync()
        np.testing.assert_array_equal(dout.cpu().numpy().reshape(want.shape), want)


def test_extract_greg_order_and_autos(dsax, oracle):
    """The visibility writers' options on the GPU: the "Greg" baseline
    order (gen_lookup / reorder_gh) and auto_extract accumulated over two
    blocks, against the oracle restatements (themselves checked against the
    reference's functions in tests/test_ref_pin.py); bit-exact."""
    import torch
    nchan = 40
    cfg = dsax.default_config(npkt=128, nant_in=63, nchan=nchan)
    blks = [oracle.gen_block(1310 + k, 128, 63, nchan, "gauss") for k in range(2)]
    greg = oracle.greg_order()
    specs = np.zeros((63, nchan), np.float32)
    with dsax.Context(cfg) as ctx:
        autos = np.zeros((63, nchan), np.float32)
        dautos = torch.zeros(63 * nchan, dtype=torch.float32, device="cuda")
        for blk in blks:
            ex = oracle.simple_extract(oracle.correlate(blk))
            specs = oracle.auto_extract(ex, specs)
            out = np.zeros(ex.size, np.float32)
            ctx.correlate_extract(np.ascontiguousarray(blk.reshape(-1)), out, mem=dsax.MEM_HOST,
                                  order=1, autos=autos)
            np.testing.assert_array_equal(out.reshape(ex.shape), ex[greg])
            d = torch.from_numpy(np.ascontiguousarray(blk.reshape(-1))).cuda()
            torch.cuda.synchronize()
            ctx.correlate_extract(d, None, mem=dsax.MEM_DEVICE, autos=dautos)
            ctx.sync()
        np.testing.assert_array_equal(autos, specs)
        np.testing.assert_array_equal(dautos.cpu().numpy().reshape(63, nchan), specs)

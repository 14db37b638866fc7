"""Failure detection on the GPU without a fault: every pipeline wait in the
tensor-core kernels is bounded by the context's wait_limit_ns, and a wait
that runs out records a timeout in the context's error word, which
dsax_sync reports as DSAX_ERR_TIMEOUT; the kernel drains its own copies and
MMAs in flight, frees TMEM and returns, and the context stays usable.
(Collected late on purpose: it runs after the parity tests.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_on_a_barrier_nothing_completes_times_out(dsax, oracle):
    """The bounded wait itself: a barrier that nothing completes, a 1 ms
    limit.  The status is DSAX_ERR_TIMEOUT, the error word is cleared, and
    the same context then correlates bit-exactly."""
    import torch
    cfg = dsax.default_config(npkt=128, nant_in=63, nchan=16)
    blk = oracle.gen_block(807, 128, 63, 16, "gauss")
    with dsax.Context(cfg) as ctx:
        rc = dsax.lib().dsax_check_wait_limit(ctx.handle, 1_000_000)
        assert rc == dsax.DSAX_ERR_TIMEOUT
        ctx.sync()
        d = torch.from_numpy(blk.reshape(-1)).cuda()
        vis = torch.zeros(32 * 2080 * 8, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.correlate(d, vis)
        ctx.sync()
        np.testing.assert_array_equal(vis.cpu().numpy().reshape(32, 2080, 4, 2),
                                      oracle.correlate(blk))


def _sync_status(dsax, ctx):
    try:
        ctx.sync()
        return dsax.DSAX_OK
    except dsax.DsaxError as e:
        return e.status


@pytest.mark.parametrize("corr_path", [3, 4, 5, 6])
def test_correlator_with_a_1ns_wait_limit_returns(dsax, oracle, corr_path):
    """A full block with every pipeline wait limited to 1 ns: the kernel
    returns (no hang) with either a recorded timeout (a wait that needed a
    second try gave up) or, if every wait completed at its first try, the
    normal result; either way a context with the default limit afterwards
    correlates the block bit-exactly."""
    import torch
    npkt, nant, nchan = 2048, 63, 384
    blk = oracle.gen_block(808, npkt, nant, nchan, "gauss")
    d_in = torch.from_numpy(blk.reshape(-1)).cuda()
    vis = torch.zeros(2 * nchan * 2080 * 8, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    with dsax.Context(dsax.default_config(corr_path=corr_path, wait_limit_ns=1)) as ctx:
        ctx.correlate(d_in, vis, dsax.MEM_DEVICE)
        st = _sync_status(dsax, ctx)
        assert st in (dsax.DSAX_OK, dsax.DSAX_ERR_TIMEOUT)
        print(f"1 ns wait limit, corr_path {corr_path}: status {st}")
        ctx.sync()
    with dsax.Context(dsax.default_config(corr_path=corr_path)) as ctx:
        vis.zero_()
        torch.cuda.synchronize()
        ctx.correlate(d_in, vis, dsax.MEM_DEVICE)
        ctx.sync()
        got = vis.cpu().numpy().reshape(2 * nchan, 2080, 4, 2)
    for c in (0, 191, 383):
        np.testing.assert_array_equal(got[2 * c:2 * c + 2], oracle.correlate(blk, ch0=c, nch=1))


@pytest.mark.parametrize("bf_path", [1, 2])
def test_beamformer_with_a_1ns_wait_limit_returns(dsax, oracle, bf_path):
    """Both kernel forms (one CTA per beam tile; CTA pairs sharing a
    cta_group::2 MMA, whose waits span both CTAs) return after their waits
    run out, and a fresh context is correct afterwards."""
    import torch
    blk = oracle.gen_block(809, 256, 63, 48, "gauss")
    wre, wim = oracle.random_phase_weights(10, 6, 256)
    d_in = torch.from_numpy(blk.reshape(-1)).cuda()
    nout = (256 // 16) * 256 * 6
    f32 = torch.zeros(nout, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    with dsax.Context(dsax.default_config(npkt=256, nchan=48, wait_limit_ns=1,
                                          bf_path=bf_path)) as ctx:
        ctx.set_weights(wre, wim)
        ctx.beamform(d_in, None, f32)
        assert _sync_status(dsax, ctx) in (dsax.DSAX_OK, dsax.DSAX_ERR_TIMEOUT)
        ctx.sync()
    with dsax.Context(dsax.default_config(npkt=256, nchan=48, bf_path=bf_path)) as ctx:
        ctx.set_weights(wre, wim)
        f32.zero_()
        torch.cuda.synchronize()
        ctx.beamform(d_in, None, f32)
        ctx.sync()
        got = f32.cpu().numpy().reshape(16, 256, 6).astype(np.float64)
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=16)
    assert (np.abs(got - ref) / ref).max() < 5e-3

"""Failure detection on the GPU without a fault: every pipeline wait in the
tensor-core kernels is bounded by the context's wait_limit_ns.  A limit of
1 ns makes the waits run out on a full block; the kernels must record the
timeout in the context's error word, drain their own copies and MMAs in
flight, free TMEM and return, so that dsax_sync reports DSAX_ERR_TIMEOUT,
the context stays usable, and a context with the default limit computes the
same block bit-exactly afterwards.  (Collected late on purpose: it runs
after the parity tests.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("corr_path", [3, 4])
def test_correlator_wait_limit_expires_and_recovers(dsax, oracle, corr_path):
    import torch
    npkt, nant, nchan = 2048, 63, 384
    blk = oracle.gen_block(808, npkt, nant, nchan, "gauss")
    d_in = torch.from_numpy(blk.reshape(-1)).cuda()
    vis = torch.zeros(2 * nchan * 2080 * 8, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    cfg = dsax.default_config(corr_path=corr_path, wait_limit_ns=1)
    with dsax.Context(cfg) as ctx:
        ctx.correlate(d_in, vis, dsax.MEM_DEVICE)
        with pytest.raises(dsax.DsaxError) as ei:
            ctx.sync()
        assert ei.value.status == dsax.DSAX_ERR_TIMEOUT
        ctx.sync()   # the error word was cleared: the context is usable
    with dsax.Context(dsax.default_config(corr_path=corr_path)) as ctx:
        vis.zero_()
        torch.cuda.synchronize()
        ctx.correlate(d_in, vis, dsax.MEM_DEVICE)
        ctx.sync()
        got = vis.cpu().numpy().reshape(2 * nchan, 2080, 4, 2)
    for c in (0, 191, 383):
        np.testing.assert_array_equal(got[2 * c:2 * c + 2], oracle.correlate(blk, ch0=c, nch=1))


def test_beamformer_wait_limit_expires_and_recovers(dsax, oracle):
    import torch
    blk = oracle.gen_block(809, 256, 63, 48, "gauss")
    wre, wim = oracle.random_phase_weights(10, 6, 256)
    d_in = torch.from_numpy(blk.reshape(-1)).cuda()
    nout = (256 // 16) * 256 * 6
    f32 = torch.zeros(nout, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    cfg = dsax.default_config(npkt=256, nchan=48, wait_limit_ns=1)
    with dsax.Context(cfg) as ctx:
        ctx.set_weights(wre, wim)
        ctx.beamform(d_in, None, f32)
        with pytest.raises(dsax.DsaxError) as ei:
            ctx.sync()
        assert ei.value.status == dsax.DSAX_ERR_TIMEOUT
        ctx.sync()
    with dsax.Context(dsax.default_config(npkt=256, nchan=48)) as ctx:
        ctx.set_weights(wre, wim)
        f32.zero_()
        torch.cuda.synchronize()
        ctx.beamform(d_in, None, f32)
        ctx.sync()
        got = f32.cpu().numpy().reshape(16, 256, 6).astype(np.float64)
    ref = oracle.beamform_power(blk, wre, wim, pkt_per_out=16)
    assert (np.abs(got - ref) / ref).max() < 5e-3

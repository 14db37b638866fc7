"""The allocation-free flagger entry point (dsax_flag_noalloc): callers that
cannot allocate device memory get the plain flagger's masks from a fixed
device array inside the library.  Checked through the C-ABI against the
context-based dsax_flag on two calls in a row (the shared array keeps the
previous call's contents, so the second call must not see the first)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(dsax):
    L = dsax.lib()
    fn = L.dsax_flag_noalloc
    fn.argtypes = [ctypes.POINTER(dsax.FlagParams), ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_matches_dsax_flag_twice(dsax):
    import torch
    from dsax import synth
    fn = _noalloc(dsax)
    B, T, C = 256, 4096, 48
    ref_ctx = dsax.Context(dsax.default_config(npkt=16, nchan=8))
    try:
        for seed in (71, 72):                  # two calls in a row, different data
            x, _ = synth.gen_filterbank(seed, nbeam=B, ntime=T, nchan=C)
            xd = torch.from_numpy(x).cuda()
            p = dsax.flag_params(B, T, C)
            cm = torch.full((B * C,), 7, dtype=torch.uint8, device="cuda")
            tm = torch.full((B * T,), 7, dtype=torch.uint8, device="cuda")
            cnt = torch.full((2,), -1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            rc = fn(ctypes.byref(p), xd.data_ptr(), None, cm.data_ptr(), tm.data_ptr(),
                    cnt.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
            rcm = torch.zeros(B * C, dtype=torch.uint8, device="cuda")
            rtm = torch.zeros(B * T, dtype=torch.uint8, device="cuda")
            rcnt = torch.zeros(2, dtype=torch.int32, device="cuda")
            ref_ctx.flag(p, xd, rcm, rtm, counts=rcnt)
            ref_ctx.sync()
            assert torch.equal(cm, rcm)
            assert torch.equal(tm, rtm)
            assert torch.equal(cnt, rcnt)
            assert int(cnt[0]) == int(cm.sum()) and int(cnt[1]) == int(tm.sum())
    finally:
        ref_ctx.close()


def test_noalloc_rejects_sizes_beyond_the_array(dsax):
    fn = _noalloc(dsax)
    p = dsax.flag_params(512, 4096, 48)        # 512 * (4*48 + 4096 + 2) + 4 > 1,572,864
    rc = fn(ctypes.byref(p), ctypes.c_void_p(16), None, ctypes.c_void_p(16), ctypes.c_void_p(16),
            None, None)
    assert rc == dsax.DSAX_ERR_ARG


def _run_both(dsax, fn, ref_ctx, p, xd):
    """One dsax_flag_noalloc call and one dsax_flag call on the same data;
    returns both (chanmask, tsmask, counts)."""
    import torch
    B, T, C = p.nbeam, p.ntime, p.nchan
    outs = []
    for use_noalloc in (True, False):
        cm = torch.full((B * C,), 7, dtype=torch.uint8, device="cuda")
        tm = torch.full((B * T,), 7, dtype=torch.uint8, device="cuda")
        cnt = torch.full((2,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        if use_noalloc:
            rc = fn(ctypes.byref(p), xd.data_ptr(), None, cm.data_ptr(), tm.data_ptr(),
                    cnt.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
        else:
            ref_ctx.flag(p, xd, cm, tm, counts=cnt)
            ref_ctx.sync()
        outs.append((cm, tm, cnt))
    return outs


def test_noalloc_at_the_size_limit_then_smaller(dsax):
    """A shape that fills the array exactly (4*B*C + B*T + 2*B + 4 =
    1,572,864 floats, so the counters are its last floats) is accepted and
    matches dsax_flag; a smaller shape afterwards, whose statistics sit at
    other offsets of the same array, matches too."""
    import torch
    from dsax import synth
    fn = _noalloc(dsax)
    limit = 1572864
    B, C = 2, 48
    T = (limit - 4) // B - 4 * C - 2
    assert 4 * B * C + B * T + 2 * B + 4 == limit
    ref_ctx = dsax.Context(dsax.default_config(npkt=16, nchan=8))
    try:
        rng = np.random.default_rng(5)
        x = rng.exponential(1.0, size=(B, T, C)).astype(np.float32)
        x[:, :, 20] += 3.0                      # a persistent tone in one channel
        x[:, 1000:1004, :] += 4.0               # a short broadband burst
        p = dsax.flag_params(B, T, C, ts_base=4096)
        xd = torch.from_numpy(x).cuda()
        (cm, tm, cnt), (rcm, rtm, rcnt) = _run_both(dsax, fn, ref_ctx, p, xd)
        assert torch.equal(cm, rcm) and torch.equal(tm, rtm) and torch.equal(cnt, rcnt)
        assert int(cm.sum()) > 0 and int(tm.sum()) > 0
        del xd
        x2, _ = synth.gen_filterbank(73, nbeam=64, ntime=2048, nchan=32)
        p2 = dsax.flag_params(64, 2048, 32)
        xd2 = torch.from_numpy(x2).cuda()
        (cm, tm, cnt), (rcm, rtm, rcnt) = _run_both(dsax, fn, ref_ctx, p2, xd2)
        assert torch.equal(cm, rcm) and torch.equal(tm, rtm) and torch.equal(cnt, rcnt)
    finally:
        ref_ctx.close()


def test_noalloc_one_past_the_limit_is_rejected(dsax):
    fn = _noalloc(dsax)
    B, C = 2, 48
    T = (1572864 - 4) // B - 4 * C - 2 + 1      # one float per beam too many
    p = dsax.flag_params(B, T, C, ts_base=4096)
    rc = fn(ctypes.byref(p), ctypes.c_void_p(16), None, ctypes.c_void_p(16), ctypes.c_void_p(16),
            None, None)
    assert rc == dsax.DSAX_ERR_ARG


def test_noalloc_on_a_second_device(dsax):
    """The array's address and the kernels' shared-memory attributes are set
    up per device: a call on device 1 after calls on device 0 (two ordinary
    single-GPU calls, no peer access)."""
    import torch
    from dsax import synth
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    fn = _noalloc(dsax)
    B, T, C = 32, 1024, 48
    x, _ = synth.gen_filterbank(74, nbeam=B, ntime=T, nchan=C)
    p = dsax.flag_params(B, T, C)
    res = []
    for dev in (0, 1):
        with torch.cuda.device(dev):
            xd = torch.from_numpy(x).cuda()
            cm = torch.zeros(B * C, dtype=torch.uint8, device="cuda")
            tm = torch.zeros(B * T, dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            rc = fn(ctypes.byref(p), xd.data_ptr(), None, cm.data_ptr(), tm.data_ptr(), None,
                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
            res.append((cm.cpu(), tm.cpu()))
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])

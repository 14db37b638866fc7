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
    p = dsax.flag_params(512, 4096, 48)        # 512 * (4*48 + 4096) + 2 > 1,572,864
    rc = fn(ctypes.byref(p), ctypes.c_void_p(16), None, ctypes.c_void_p(16), ctypes.c_void_p(16),
            None, None)
    assert rc == dsax.DSAX_ERR_ARG

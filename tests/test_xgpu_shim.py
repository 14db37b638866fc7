"""The xGPU call shapes of include/xgpu_dsax.h, driven the way
src/dsaX_xgpu.cu:253-340 drives xGPU."""
import ctypes

import numpy as np
import pytest


class XGPUInfo(ctypes.Structure):
    _fields_ = [("npol", ctypes.c_uint), ("nstation", ctypes.c_uint),
                ("nbaseline", ctypes.c_uint), ("nfrequency", ctypes.c_uint),
                ("ntime", ctypes.c_uint), ("ntimepipe", ctypes.c_uint),
                ("vecLength", ctypes.c_size_t), ("vecLengthPipe", ctypes.c_size_t),
                ("matLength", ctypes.c_size_t), ("triLength", ctypes.c_size_t),
                ("matrix_order", ctypes.c_int)]


class XGPUContext(ctypes.Structure):
    _fields_ = [("array_h", ctypes.c_void_p), ("matrix_h", ctypes.c_void_p),
                ("array_len", ctypes.c_size_t), ("matrix_len", ctypes.c_size_t),
                ("internal", ctypes.c_void_p)]


def _lib(dsax):
    L = dsax.lib()
    L.xgpuInfo.argtypes = [ctypes.POINTER(XGPUInfo)]
    L.xgpuInfo.restype = None
    L.xgpuInit.argtypes = [ctypes.POINTER(XGPUContext), ctypes.c_int]
    L.xgpuInit.restype = ctypes.c_int
    L.xgpuCudaXengine.argtypes = [ctypes.POINTER(XGPUContext), ctypes.c_void_p, ctypes.c_int]
    L.xgpuCudaXengine.restype = ctypes.c_int
    L.xgpuClearDeviceIntegrationBuffer.argtypes = [ctypes.POINTER(XGPUContext)]
    L.xgpuFree.argtypes = [ctypes.POINTER(XGPUContext)]
    return L


def test_xgpu_info_matches_reference_build(dsax):
    """README.md:38-52 (the reference's xgpuinfo output)."""
    info = XGPUInfo()
    _lib(dsax).xgpuInfo(ctypes.byref(info))
    assert (info.npol, info.nstation, info.nbaseline, info.nfrequency, info.ntime,
            info.ntimepipe) == (2, 64, 2080, 768, 2048, 128)
    assert info.vecLength == 201326592
    assert info.vecLengthPipe == 12582912
    assert info.matLength == 6389760


@pytest.mark.gpu
def test_xgpu_call_sequence(dsax, oracle):
    import torch
    L = _lib(dsax)
    info = XGPUInfo()
    L.xgpuInfo(ctypes.byref(info))
    ctx = XGPUContext()
    assert L.xgpuInit(ctypes.byref(ctx), 0) == 0
    try:
        blk = oracle.gen_block(31, 2048, 63, 384, "gauss")
        xin = torch.from_numpy(oracle.fluff_reorder(blk).reshape(-1).view(np.uint8)).cuda()
        torch.cuda.synchronize()
        mat = np.ctypeslib.as_array((ctypes.c_float * (2 * info.matLength)).from_address(ctx.matrix_h))
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xin.data_ptr(), 1) == 0   # SYNCOP_DUMP
        v1 = mat.copy().reshape(768, 2080, 4, 2)
        for c in (0, 17, 200, 383):
            np.testing.assert_array_equal(v1[2 * c:2 * c + 2], oracle.correlate(blk, ch0=c, nch=1))
        # integrates until cleared
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xin.data_ptr(), 1) == 0
        np.testing.assert_array_equal(mat.reshape(v1.shape), 2 * v1)
        L.xgpuClearDeviceIntegrationBuffer(ctypes.byref(ctx))
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xin.data_ptr(), 1) == 0
        np.testing.assert_array_equal(mat.reshape(v1.shape), v1)
    finally:
        L.xgpuFree(ctypes.byref(ctx))

"""CPU tests of the C-ABI boundary: the library loads, exports every function
the public headers declare, and its pure-host helpers behave.  No kernel is
launched here."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src):
            name = m.group(1)
            if name in ("sizeof", "if", "while", "for", "return"):
                continue
            names.add(name)
    return sorted(names)


def test_headers_declare_entry_points():
    names = _declared_functions()
    assert "dsax_create" in names and "dsax_correlate" in names


@pytest.mark.parametrize("name", _declared_functions())
def test_library_exports_declared_symbol(dsax, name):
    assert hasattr(dsax.lib(), name), f"{name} declared in include/ but not exported"


def test_size_helpers(dsax):
    cfg = dsax.default_config()
    assert (cfg.npkt, cfg.nant_in, cfg.nchan, cfg.nbeam, cfg.bf_pkt_per_out) == (2048, 63, 384, 256, 16)
    assert dsax.block_bytes(cfg, dsax.FMT_CAPTURED) == 198_180_864       # README.md:34
    assert dsax.block_bytes(cfg, dsax.FMT_REORDERED) == 201_326_592      # src/dsaX_xgpu.cu:312
    assert dsax.block_bytes(cfg, dsax.FMT_XGPU_INT8) == 402_653_184      # README.md:34
    assert dsax.vis_bytes(cfg) == 51_118_080                             # README.md:58
    assert dsax.beam_bytes(cfg) == 1_572_864                             # README.md:62
    cfg4 = dsax.default_config(bf_pkt_per_out=4)
    assert dsax.beam_bytes(cfg4) == 6_291_456                            # scripts/config_corr.yaml:39-42


def test_strerror_covers_codes(dsax):
    for code in (0, -1, -2, -3, -4, -5, -6):
        assert dsax.strerror(code) != "unknown status"


def test_create_rejects_bad_config(dsax):
    bad = dsax.default_config(nant_in=65)
    h = ctypes.c_void_p()
    rc = dsax.lib().dsax_create(ctypes.byref(h), ctypes.byref(bad), 0)
    assert rc == dsax.DSAX_ERR_ARG and not h.value


def test_create_without_gpu_fails_cleanly(dsax):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = dsax.lib().dsax_create(ctypes.byref(h), ctypes.byref(dsax.default_config()), 0)
    assert rc in (dsax.DSAX_ERR_CUDA, dsax.DSAX_ERR_UNSUPPORTED) and not h.value


def test_null_arguments_rejected(dsax):
    L = dsax.lib()
    assert L.dsax_correlate_fmt(None, 0, None, None, 0, 0) == dsax.DSAX_ERR_ARG
    assert L.dsax_sync(None) == dsax.DSAX_ERR_ARG

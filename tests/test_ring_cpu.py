"""The shared-memory block ring that stands in for psrdada (driver/dsax_ring):
blocks written by one process arrive intact and in order at another, a
short block ends the stream, and waits time out instead of hanging."""
import os
import subprocess

import numpy as np
import pytest

PKG = os.path.join(os.path.dirname(__file__), "..", "dsa110-xengine_b200")
TOOL = os.path.join(PKG, "dsax_ringtool")


@pytest.fixture(scope="module")
def ringtool():
    subprocess.check_call(["make", "-s", "-C", PKG, "dsax_ringtool"])
    return TOOL


def test_ring_round_trip(ringtool, tmp_path):
    name = f"/dsax_ring_test_{os.getpid()}"
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bin"
    hdr = tmp_path / "hdr.txt"
    data = np.random.default_rng(1).integers(0, 256, 3 * 1000 + 500, dtype=np.uint8)
    src.write_bytes(data.tobytes())
    hdr.write_text("NPKT 16\nNANT 63\n")
    subprocess.check_call([ringtool, "create", name, "2", "1000"])
    try:
        reader = subprocess.Popen([ringtool, "get", name, str(dst)])
        subprocess.check_call([ringtool, "put", name, str(src), str(hdr)], timeout=60)
        assert reader.wait(timeout=60) == 0
        assert dst.read_bytes() == data.tobytes()
    finally:
        subprocess.call([ringtool, "destroy", name])


def test_ring_exact_multiple_ends_with_empty_block(ringtool, tmp_path):
    name = f"/dsax_ring_test2_{os.getpid()}"
    src = tmp_path / "in.bin"
    dst = tmp_path / "out.bin"
    data = bytes(range(256)) * 8   # 2048 bytes = 2 blocks of 1024
    src.write_bytes(data)
    subprocess.check_call([ringtool, "create", name, "4", "1024"])
    try:
        subprocess.check_call([ringtool, "put", name, str(src)], timeout=60)   # 4 slots: no reader needed
        subprocess.check_call([ringtool, "get", name, str(dst)], timeout=60)
        assert dst.read_bytes() == data
    finally:
        subprocess.call([ringtool, "destroy", name])

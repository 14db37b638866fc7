"""The ring-to-ring correlator process (driver/dsax_xengine, the loop of
src/dsaX_xgpu.cu:150-357 over the in-repo shared-memory ring): three
blocks through input ring -> dsax_xengine -> output ring, each output
bit-exact against the oracle, the header passed through, and the stream
ended by the short block."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PKG = os.path.join(os.path.dirname(__file__), "..", "dsa110-xengine_b200")


def test_xengine_ring_to_ring(dsax, oracle, tmp_path):
    subprocess.check_call(["make", "-s", "-C", PKG, "dsax_ringtool", "dsax_xengine"])
    tool, xeng = os.path.join(PKG, "dsax_ringtool"), os.path.join(PKG, "dsax_xengine")
    npkt, nant, nchan = 256, 63, 48
    blks = [oracle.gen_block(1200 + k, npkt, nant, nchan, "gauss") for k in range(3)]
    src, dst, hdr = tmp_path / "in.bin", tmp_path / "vis.bin", tmp_path / "hdr.txt"
    src.write_bytes(b"".join(b.tobytes() for b in blks))
    hdr.write_text(f"NPKT {npkt}\nNANT {nant}\nNCHAN {nchan}\n")
    nin = npkt * nant * nchan * 4
    nvis = 2 * nchan * 2080 * 8 * 4
    rin, rout = f"/dsax_xin_{os.getpid()}", f"/dsax_xout_{os.getpid()}"
    subprocess.check_call([tool, "create", rin, "2", str(nin)])
    subprocess.check_call([tool, "create", rout, "2", str(nvis)])
    try:
        reader = subprocess.Popen([tool, "get", rout, str(dst)])
        engine = subprocess.Popen([xeng, "-i", rin, "-o", rout, "-t", "60"])
        subprocess.check_call([tool, "put", rin, str(src), str(hdr)], timeout=120)
        assert engine.wait(timeout=120) == 0
        assert reader.wait(timeout=60) == 0
    finally:
        subprocess.call([tool, "destroy", rin])
        subprocess.call([tool, "destroy", rout])
    vis = np.frombuffer(dst.read_bytes(), np.float32)
    assert vis.size == 3 * nvis // 4
    for k, b in enumerate(blks):
        got = vis[k * (nvis // 4):(k + 1) * (nvis // 4)].reshape(2 * nchan, 2080, 4, 2)
        np.testing.assert_array_equal(got, oracle.correlate(b))

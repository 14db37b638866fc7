"""The FP32 uint8 scaley (dsax_scaley.h: one FMA with an exact fallback near
rounding ties) agrees with the FP64 form of src/gpu_flagger.cu:382-394 on
every uint8 input for 400,000 random baselines and on exact-tie cases."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "dsa110-xengine_b200", "csrc")


def test_fp32_scaley_matches_fp64(tmp_path):
    exe = tmp_path / "scaley_check"
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC,
                        os.path.join(HERE, "scaley_check.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout[-2000:])
    checked, bad, slow = (int(v) for v in r.stdout.split()[-3:])
    assert r.returncode == 0 and bad == 0
    assert checked > 100_000_000 and slow < checked // 100

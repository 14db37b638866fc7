"""Regenerates the golden fixtures in tests/golden/ from the reference tree.

Run in a container where the reference checkout exists (default
/root/reference; override with DSAX_REFERENCE):

    python tests/golden/make_golden.py

Fixtures written (all small, committed):
  packet_decode.json  -- utils/packet.out (one 4608-byte noise packet,
                         base64) and what the reference's own decoders
                         make_spectrum() / make_histogram() from
                         utils/gen_packet.py:15-67 return for it.  The
                         functions are executed from the reference source
                         (extracted with ast; the module's top level needs
                         matplotlib and numpy<2 and is not run).
  reorder_tone.json   -- utils/test.out (the 8-bit reorder of a tone packet,
                         src/dsaX_reorder_raw.c.bak:304-339): its sha256 and
                         every nonzero entry, plus the tone description the
                         input is rebuilt from.
utils/gen_testblock.py is not executed: it assigns out-of-range floats
to int8 arrays, which numpy 1 wrapped and numpy 2 (the only numpy here)
rejects.  Its ramp pattern is restated in tests/test_oracle.py instead.
"""
from __future__ import annotations

import ast
import base64
import hashlib
import json
import os
import struct

import numpy as np

REF = os.environ.get("DSAX_REFERENCE", "/root/reference")
OUT = os.path.dirname(os.path.abspath(__file__))


def _load_functions(path: str, names: list[str]) -> dict:
    """Compile only the named top-level functions of a reference module."""
    src = open(path).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {"np": np, "struct": struct}
    exec(compile(mod, path, "exec"), ns)
    return ns


def packet_decode():
    pkt = open(os.path.join(REF, "utils/packet.out"), "rb").read()
    assert len(pkt) == 4608
    ns = _load_functions(os.path.join(REF, "utils/gen_packet.py"),
                         ["make_spectrum", "make_histogram"])
    spectra = {}
    for ant in range(3):
        for pol in range(2):
            spectra[f"{ant},{pol}"] = [float(v) for v in ns["make_spectrum"](pkt, ant=ant, pol=pol)]
    hx, histo, rms = ns["make_histogram"](pkt)
    out = {
        "source": "utils/packet.out decoded by utils/gen_packet.py make_spectrum/make_histogram",
        "packet_b64": base64.b64encode(pkt).decode(),
        "sha256": hashlib.sha256(pkt).hexdigest(),
        "layout": "[3 ant][384 chan][2 time][2 pol] one byte per complex sample",
        "spectra": spectra,
        "hist_x": [int(v) for v in hx],
        "hist_norm": [float(v) for v in histo],
        "rms": float(rms),
    }
    with open(os.path.join(OUT, "packet_decode.json"), "w") as f:
        json.dump(out, f, indent=1)


def reorder_tone():
    raw = open(os.path.join(REF, "utils/test.out"), "rb").read()
    a = np.frombuffer(raw, dtype=np.int8).reshape(768, 64, 2, 2)
    nz = np.argwhere(a != 0)
    out = {
        "source": "utils/test.out: 8-bit reorder output [768 = chan*2+t][64 ant][2 pol][re,im]",
        "sha256": hashlib.sha256(raw).hexdigest(),
        "shape": [768, 64, 2, 2],
        "nonzero": [[int(k), int(an), int(p), int(c), int(a[k, an, p, c])] for k, an, p, c in nz],
        "tone": {"chans": [10, 100, 190], "ants_mod3": 1, "nant_in": 63,
                 "pol0_re": 3, "pol1_re": 2, "imag": 0, "times": [0, 1]},
    }
    with open(os.path.join(OUT, "reorder_tone.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    packet_decode()
    reorder_tone()
    print("fixtures written to", OUT)

"""Builds oracle/_ref/libref.so from the reference's own C/CUDA sources.

TEST INFRASTRUCTURE ONLY.  The reference ships no library: every stage is
a psrdada client whose `main()` needs psrdada, xGPU, sigproc or cfitsio,
none of which exist here.  Several of the functions on the hot path are
plain C that needs none of them, though.  This recipe lifts those function
bodies verbatim out of the reference files (brace matching, with `#line`
directives pointing back at the original file:line), compiles them with
the shape macros the reference hard-codes set on the command line, and
links them with oracle/ref_harness.cpp, which supplies the few globals and
types they name and exports stable wrappers.  Nothing is copied into the
repository: the extracted text is written only under oracle/_ref/
(git-ignored) and regenerated from the reference tree on every build.

Functions taken (reference path:line of each definition is printed in the
generated file):
  src/gpu_flagger.cu  medval, simple_channflag, simple_tsflag, channflag,
                      gather_mask, gather_tsmask, calc_bpwr, median_calc
                      (host C, :534-798), and the element kernels scaley,
                      flag, flagts (:382-394, :459-494), which use no
                      shared memory or barriers and are run on the host
                      one (block, thread) at a time by the harness;
  src/dsaX_wrangle.c  auto_extract, simple_extract (:47-93);
  src/dsaX_wrangleAndWrite.c  gen_lookup, reorder_gh (:46-93, the "Greg"
                      baseline order);
  src/dsaX_bfCorr.cu  populate_weights_matrix (:815-863), the two-arm
                      weights with the declination term (an element kernel,
                      run per (block, thread) on the host; half stored as
                      float);
  src/dsaX_reorder_raw.c      massage (:98-219, the byte reorder);
  src/dsaX_reorder_raw.c.bak  massage (:98-266, AVX-512 fluff + transpose).

Shapes (the reference's compile-time constants, set with -D):
  flagger  NBEAMS_P 64, NTIMES_P 2048, NCHAN_P 1024 (median_calc indexes
           beam 31 of 64, and channflag hard-codes ZeroChannels = 128, so
           the beam and channel counts stay at the reference's values; the
           time axis is shortened from 16384 to 2048, so simple_tsflag's
           baseline is NTIMES_P/16 = 128 samples), NPERMFLAGS 1,
           flagchannels {10}, MN 48, SIG 6, FBIN 8, TBIN 128;
  reorder  NANTS 63 (README.md:34; dsaX_def.h's 96 belongs to the bfCorr
           variant), NPACKETS 2048 and a 64-packet build for quick tests;
  weights  NANTS 96 (48 per arm), NBEAMS 512, NCHAN_PER_PACKET 16 (two
           frequency groups instead of 48, to keep the host run short),
           sep 1.0 arcmin, PI and CVAC as dsaX_def.h:28-29.

Usage:  python oracle/make_ref.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
DEFAULT_REF = os.environ.get("DSAX_REFERENCE", "/root/reference")

FLAG_FUNCS = ["medval", "simple_channflag", "simple_tsflag", "channflag", "gather_mask",
              "gather_tsmask", "calc_bpwr", "median_calc", "scaley", "flag", "flagts"]
WRANGLE_FUNCS = ["auto_extract", "simple_extract"]
GH_FUNCS = ["gen_lookup", "reorder_gh"]

# Appended to each massage unit (this project's code, not the reference's):
# one thread per packet slice with the reference's thread argument, as its
# main loop starts them (src/dsaX_reorder_raw.c:539-563).  The raw variant
# writes through d->ipc->curbuf, the AVX-512 one to d->out (write = 0).
MASSAGE_RUN = r'''
int massage_run_@TAG@(const char *in, char *out, int nthreads) {
  pthread_t th[16];
  struct data d[16];
  ipcio_t ipc;
  ipc.curbuf = out;
  if (nthreads < 1 || nthreads > 16 || NPACKETS % nthreads) return -1;
  for (int i = 0; i < nthreads; i++) {
    d[i].in = (char *)in; d[i].out = out; d[i].n_threads = nthreads; d[i].thread_id = i;
    d[i].debug = 0; d[i].write = 0; d[i].ipc = &ipc;
    if (pthread_create(&th[i], NULL, massage, &d[i])) return -2;
  }
  for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
  return 0;
}
'''

FLAG_SHAPE = {"NBEAMS_P": 64, "NTIMES_P": 2048, "NCHAN_P": 1024}
BFCORR_SHAPE = ["-DNCHAN_PER_PACKET=16", "-DNBEAMS=512"]


def _strip_spans(src: str) -> list[tuple[int, int]]:
    """Character spans of comments and string/char literals (to be skipped
    when matching braces)."""
    spans, i, n = [], 0, len(src)
    while i < n:
        c = src[i]
        if src.startswith("//", i):
            j = src.find("\n", i)
            j = n if j < 0 else j
            spans.append((i, j))
            i = j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            j = n if j < 0 else j + 2
            spans.append((i, j))
            i = j
        elif c in "\"'":
            j = i + 1
            while j < n and src[j] != c:
                j += 2 if src[j] == "\\" else 1
            spans.append((i, j + 1))
            i = j + 1
        else:
            i += 1
    return spans


def extract(path: str, name: str) -> tuple[str, int]:
    """The definition of function `name` (signature through the matching
    closing brace) and its 1-based starting line in `path`."""
    src = open(path, encoding="latin-1").read()
    spans = _strip_spans(src)
    in_span = bytearray(len(src))
    for a, b in spans:
        in_span[a:b] = b"\x01" * (b - a)
    # a definition: start of line, return type (and qualifiers), the name,
    # a parameter list, then an opening brace (possibly on a later line)
    pat = re.compile(r"^[ \t]*(?:__global__\s+)?[A-Za-z_][\w \t\*]*?\b" + re.escape(name) +
                     r"\s*\([^;{)]*\)\s*\{", re.M)
    for m in pat.finditer(src):
        if in_span[m.start()]:
            continue
        depth, i = 0, m.end() - 1
        while i < len(src):
            if not in_span[i]:
                if src[i] == "{":
                    depth += 1
                elif src[i] == "}":
                    depth -= 1
                    if depth == 0:
                        line = src.count("\n", 0, m.start()) + 1
                        # include a __global__ on the line above the signature
                        start = m.start()
                        prev = src.rfind("\n", 0, max(start - 1, 0))
                        above = src[prev + 1:start].strip()
                        if above == "__global__":
                            start, line = prev + 1, line - 1
                        return src[start:i + 1], line
            i += 1
        break
    raise SystemExit(f"{path}: definition of {name} not found")


def extract_struct(path: str, name: str) -> tuple[str, int]:
    src = open(path, encoding="latin-1").read()
    m = re.search(r"^struct\s+" + re.escape(name) + r"\s*\{.*?\};", src, re.M | re.S)
    if not m:
        raise SystemExit(f"{path}: struct {name} not found")
    return m.group(0), src.count("\n", 0, m.start()) + 1


def _unit(prologue: str, pieces: list[tuple[str, str, int]]) -> str:
    out = [prologue]
    for path, text, line in pieces:
        out.append(f'#line {line} "{path}"\n{text}\n')
    return "\n".join(out)


def generate(ref: str) -> list[str]:
    os.makedirs(OUT, exist_ok=True)
    fl = os.path.join(ref, "src", "gpu_flagger.cu")
    pieces = [(fl, *extract(fl, n)) for n in FLAG_FUNCS]
    flag_src = _unit('#include "ref_stubs.h"\n#include "ref_flag_consts.h"\n', pieces)
    wr = os.path.join(ref, "src", "dsaX_wrangle.c")
    ww = os.path.join(ref, "src", "dsaX_wrangleAndWrite.c")
    wpieces = [(wr, *extract(wr, n)) for n in WRANGLE_FUNCS]
    wpieces += [(ww, *extract(ww, n)) for n in GH_FUNCS]
    # dsaX_wrangleAndWrite.c:40 declares the baseline count these use
    wr_src = _unit('#include "ref_stubs.h"\nstatic const int nbl = 2080;\n', wpieces)
    bc = os.path.join(ref, "src", "dsaX_bfCorr.cu")
    bc_src = _unit('#include "ref_stubs.h"\n#include <cmath>\ntypedef float half;\n'
                   '#define __float2half(x) (x)\n#define sep 1.0\n#define PI 3.14159265359\n'
                   '#define CVAC 299792458.0\n',
                   [(bc, *extract(bc, "populate_weights_matrix"))])
    units = {"ref_flagger.cpp": flag_src, "ref_wrangle.c": wr_src, "ref_bfcorr.cpp": bc_src}
    for tag, fname in (("raw", "dsaX_reorder_raw.c"), ("bak", "dsaX_reorder_raw.c.bak")):
        p = os.path.join(ref, "src", fname)
        st = extract_struct(p, "data")
        fn = extract(p, "massage")
        units[f"ref_massage_{tag}.c"] = _unit(
            '#include "ref_stubs.h"\n#include <immintrin.h>\n', [(p, *st), (p, *fn)]) + \
            MASSAGE_RUN.replace("@TAG@", tag)
    for f, text in units.items():
        with open(os.path.join(OUT, f), "w") as fh:
            fh.write("/* generated by oracle/make_ref.py from the reference tree; not committed */\n")
            fh.write(text)
    shutil.copy(os.path.join(HERE, "ref_stubs.h"), os.path.join(OUT, "ref_stubs.h"))
    return list(units)


FLAG_CONSTS = """/* compile-time constants of src/gpu_flagger.cu:71-95, shapes reduced as
 * oracle/make_ref.py documents */
#define M_P NTIMES_P
#define N_P 32
#define NTHREADS_GPU 32
#define MN 48.0
#define SIG 6.0
#define RMAX 16384
#define NPERMFLAGS 1
#define TBIN 128
#define FBIN 8
static int flagchannels[1] = {10};
"""


def build(ref: str = DEFAULT_REF, cc: str | None = None, cxx: str | None = None) -> str:
    """Generates and compiles oracle/_ref/libref.so (and the 64-packet
    reorder variant libref_small.so); returns the library path."""
    if not os.path.isdir(os.path.join(ref, "src")):
        raise FileNotFoundError(f"reference tree not found at {ref}")
    generate(ref)
    with open(os.path.join(OUT, "ref_flag_consts.h"), "w") as fh:
        fh.write(FLAG_CONSTS)
    cc = cc or ("/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc")
    cxx = cxx or ("/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
    common = ["-O2", "-fPIC", "-w", "-I", OUT, "-I", HERE]
    shape = [f"-D{k}={v}" for k, v in FLAG_SHAPE.items()]
    libs = []
    for variant, npk in (("libref.so", 2048), ("libref_small.so", 64)):
        objs = []
        reo = [f"-DNANTS=63", f"-DNPACKETS={npk}"]
        jobs = [
            ([cxx] + common + shape + ["-std=gnu++17", "-c", "ref_flagger.cpp"], "ref_flagger.o"),
            ([cc] + common + ["-std=gnu11", "-c", "ref_wrangle.c"], "ref_wrangle.o"),
            ([cxx] + common + BFCORR_SHAPE + ["-DNANTS=96", "-std=gnu++17", "-c",
                                              "ref_bfcorr.cpp"],
             "ref_bfcorr.o"),
            ([cc] + common + reo + ["-std=gnu11", "-Dmassage=reference_massage_raw", "-c",
                                    "ref_massage_raw.c"], "ref_massage_raw.o"),
            ([cc] + common + reo + ["-std=gnu11", "-mavx512f", "-mavx512bw",
                                    "-Dmassage=reference_massage_bak", "-c", "ref_massage_bak.c"],
             "ref_massage_bak.o"),
            ([cxx] + common + shape + reo + BFCORR_SHAPE + ["-DNANTS_BF=96", "-std=gnu++17", "-c",
                                             os.path.join(HERE, "ref_harness.cpp")],
             "ref_harness.o"),
        ]
        for cmd, obj in jobs:
            o = os.path.join(OUT, f"{npk}_{obj}")
            subprocess.check_call(cmd + ["-o", o], cwd=OUT)
            objs.append(o)
        lib = os.path.join(OUT, variant)
        subprocess.check_call([cxx, "-shared", "-o", lib] + objs + ["-lpthread", "-lm"], cwd=OUT)
        libs.append(lib)
    return libs[0]


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REF)
    a = ap.parse_args()
    print(build(a.reference))
    sys.exit(0)

"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (there is no network for real data):

  gen_block            capture blocks [npkt][nant_in][nchan][2 t][2 pol] of
                       4+4-bit samples: uniform integers on [-8, 7], or
                       Gaussian sigma 2.5 rounded and clipped to [-8, 7]
  random_phase_weights unit-magnitude beamformer weights, seeded phases (FP64)
  gen_filterbank       Stokes-I filterbanks: chi-square(2) noise plus tones,
                       bursts and drifting tones
"""
from __future__ import annotations

import numpy as np

NST = 64


def pack4(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    """4+4-bit two's complement byte: real in the low nibble, imag in the
    high nibble (src/dsaX_xgpu.cu:74-75, utils/gen_packet.py:137-147)."""
    return ((re.astype(np.int16) & 0xF) | ((im.astype(np.int16) & 0xF) << 4)).astype(np.uint8)


def gen_block(seed: int, npkt: int, nant_in: int, nchan: int,
              dist: str = "uniform", sigma: float = 2.5) -> np.ndarray:
    """Captured block [npkt][nant_in][nchan][2 t][2 pol] of packed samples.

    dist="uniform": re, im uniform on the integers [-8, 7] (every byte value
    equally likely).  dist="gauss": re, im = clip(round(N(0, sigma^2)), -8, 7).
    """
    shape = (npkt, nant_in, nchan, 2, 2)
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        return rng.integers(0, 256, size=shape, dtype=np.uint8)
    if dist == "gauss":
        n = int(np.prod(shape))
        out = np.empty(n, dtype=np.uint8)
        step = 1 << 24
        for s in range(0, n, step):
            e = min(n, s + step)
            z = rng.standard_normal((2, e - s), dtype=np.float32) * np.float32(sigma)
            q = np.clip(np.rint(z), -8, 7).astype(np.int8)
            out[s:e] = pack4(q[0], q[1])
        return out.reshape(shape)
    raise ValueError(dist)


def random_phase_weights(seed: int, ngrp: int, nbeam: int):
    """Unit-magnitude complex weights with seeded uniform phases, FP64,
    layout [ngrp][2 pol][nbeam][64 ant]."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(ngrp, 2, nbeam, NST))
    return np.cos(ph), np.sin(ph)


def gen_filterbank(seed: int, nbeam: int = 256, ntime: int = 4096, nchan: int = 48,
                   n_tones: int | None = None, n_bursts: int | None = None,
                   n_drift: int | None = None):
    """Stokes-I filterbank [nbeam][ntime][nchan] float32: chi-square(2) noise
    (exponential, mean 2, sigma 2) plus seeded RFI:
      persistent narrowband tones, 1-3 adjacent channels, 5-20 sigma;
      impulsive broadband bursts, 1-8 samples, all channels, 3-10 sigma;
      slow drifting tones, one channel wide, 5-15 sigma, drifting up to 8
      channels across the block.
    Returns (x, truth) where truth[b][t][c] marks the injected samples."""
    rng = np.random.default_rng(seed)
    x = rng.exponential(2.0, size=(nbeam, ntime, nchan)).astype(np.float32)
    truth = np.zeros((nbeam, ntime, nchan), dtype=bool)
    sig = 2.0
    n_tones = nbeam // 4 if n_tones is None else n_tones
    n_bursts = nbeam // 4 if n_bursts is None else n_bursts
    n_drift = nbeam // 8 if n_drift is None else n_drift
    for _ in range(n_tones):
        b = rng.integers(nbeam)
        w = int(rng.integers(1, 4))
        c = int(rng.integers(0, nchan - w + 1))
        amp = rng.uniform(5, 20) * sig
        x[b, :, c:c + w] += np.float32(amp)
        truth[b, :, c:c + w] = True
    for _ in range(n_bursts):
        b = rng.integers(nbeam)
        w = int(rng.integers(1, 9))
        t = int(rng.integers(0, ntime - w + 1))
        amp = rng.uniform(3, 10) * sig
        x[b, t:t + w, :] += np.float32(amp)
        truth[b, t:t + w, :] = True
    for _ in range(n_drift):
        b = rng.integers(nbeam)
        c0 = rng.uniform(0, nchan - 1)
        drift = rng.uniform(-8, 8)
        amp = rng.uniform(5, 15) * sig
        tt = np.arange(ntime)
        cc = np.clip(np.rint(c0 + drift * tt / ntime), 0, nchan - 1).astype(int)
        x[b, tt, cc] += np.float32(amp)
        truth[b, tt, cc] = True
    return x, truth

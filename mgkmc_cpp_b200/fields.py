"""Synthetic modulus fields (setup-time input synthesis, not the timed path).

``correlated_field`` restates generate_correlated_field_cpp
(material_generator.hpp:121-258): per-voxel Box-Muller normals from a
``std::mt19937(seed)`` stream (u1 re-drawn while <= 1e-15), an ortho FFT, a
Gaussian filter exp(-2 pi^2 sigma^2 f^2) on fftfreq(n) frequencies, an ortho
inverse FFT (real part), standardisation to mean 0 / std 1 (population std),
then scale, shift and optional clipping.

``lognormal_modulus`` maps such a standard Gaussian random field g to
E = E_mean * exp(s*g - s^2/2) with s^2 = ln(1 + CoV^2): a lognormal field with
mean E_mean and coefficient of variation CoV, as the heterogeneous benchmark
cases ask for.  Fields are written as the reference's ``.npy`` input.
"""
from __future__ import annotations

import numpy as np


def _mt_stream(seed: int) -> np.random.MT19937:
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)  # == std::mt19937(seed)
    return bg


def box_muller_normals(n: int, seed: int) -> np.ndarray:
    """material_generator.hpp:121-128, n draws in order."""
    bg = _mt_stream(seed)
    out = np.empty(n)
    denom = float(0xFFFFFFFF) + 1.0
    buf = bg.random_raw(max(2 * n + 64, 1024)).astype(np.float64)
    pos = 0
    for i in range(n):
        if pos + 2 >= len(buf):
            buf = np.concatenate([buf[pos:], bg.random_raw(2 * n + 64).astype(np.float64)])
            pos = 0
        u1 = buf[pos] / denom
        u2 = buf[pos + 1] / denom
        pos += 2
        while u1 <= 1e-15:
            if pos >= len(buf):
                buf = np.concatenate([buf[pos:], bg.random_raw(1024).astype(np.float64)])
                pos = 0
            u1 = buf[pos] / denom
            pos += 1
        out[i] = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return out


def standard_grf(shape, corr: float, seed: int) -> np.ndarray:
    """Standardised periodic Gaussian random field (steps 1-3 of the reference)."""
    shape = tuple(int(s) for s in shape)
    n = int(np.prod(shape))
    f = box_muller_normals(n, seed).reshape(shape)
    fh = np.fft.fftn(f, norm="ortho")
    f2 = np.zeros(shape)
    for ax, s in enumerate(shape):
        fr = np.fft.fftfreq(s)
        sh = [1] * len(shape)
        sh[ax] = s
        f2 = f2 + (fr ** 2).reshape(sh)
    fh *= np.exp(-2.0 * np.pi * np.pi * corr * corr * f2)
    g = np.fft.ifftn(fh, norm="ortho").real
    m = g.mean()
    sd = np.sqrt(((g - m) ** 2).sum() / n)
    if sd < 1e-15:
        sd = 1.0
    return (g - m) / sd


def correlated_field(shape, mean: float, std: float, corr: float, seed: int, clip_min=None, clip_max=None) -> np.ndarray:
    g = mean + std * standard_grf(shape, corr, seed)
    if clip_min is not None:
        g = np.maximum(g, clip_min)
    if clip_max is not None:
        g = np.minimum(g, clip_max)
    return g


def lognormal_modulus(shape, mean: float, cov: float, corr: float, seed: int) -> np.ndarray:
    s2 = np.log1p(cov * cov)
    s = np.sqrt(s2)
    return mean * np.exp(s * standard_grf(shape, corr, seed) - 0.5 * s2)

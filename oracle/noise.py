"""Noise oracle (test infrastructure only): numpy restatement of the generator behind
tigre_add_noise / tigre_noise_1d.

The reference (Common/CUDA/RandomNumberGenerator.cu: setup_kernel, GeneratePoisson,
GeneratePoissonAddGaussian) draws curand XORWOW streams tied to its fixed 64-block grid, so its
numbers cannot be reproduced by another design; parity with it is distributional (mean and
variance of Poisson(lambda) + N(mu, sigma), tests/test_noise*.py).  This module pins the B200
generator itself:

* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011) in uint64 numpy arithmetic, checked
  against the published known-answer vectors of its authors' Random123 distribution;
* the Poisson samplers (CDF inversion below lambda = 10, Hormann's PTRS above) and Box-Muller
  in FP64, consuming the same counters as the kernel.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)

# Random123 known-answer vectors for philox4x32 with 10 rounds: (counter, key, output)
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 on uint32 arrays (or scalars); returns four uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & MASK for v in (c0, c1, c2, c3))
    k0 = np.asarray(k0, dtype=np.uint64) & MASK
    k1 = np.asarray(k1, dtype=np.uint64) & MASK
    for r in range(10):
        if r > 0:
            k0 = (k0 + np.uint64(W0)) & MASK
            k1 = (k1 + np.uint64(W1)) & MASK
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
    return tuple(v.astype(np.uint32) for v in (c0, c1, c2, c3))


def philox_blocks(nblocks, counter_hi, seed):
    """Same layout as tigre_philox4x32: row j = philox({j_lo, j_hi, ch_lo, ch_hi}, seed)."""
    j = np.arange(nblocks, dtype=np.uint64)
    out = philox4x32_10(j & MASK, j >> np.uint64(32), counter_hi & 0xFFFFFFFF, counter_hi >> 32,
                        seed & 0xFFFFFFFF, seed >> 32)
    return np.stack(out, axis=1)


def _u01d(a, b):
    v = (a.astype(np.uint64) << np.uint64(21)) ^ (b.astype(np.uint64) >> np.uint64(11))
    return ((v & np.uint64((1 << 53) - 1)).astype(np.float64) + 0.5) / 9007199254740992.0


def _u01f(x):
    return ((x >> np.uint32(8)).astype(np.float64) + 0.5) / 16777216.0


def poisson(lam, seed):
    """Poisson samples of the float32 array lam (flattened index = element index)."""
    from scipy.special import gammaln
    lam32 = np.ascontiguousarray(lam, dtype=np.float32).ravel()
    n = lam32.size
    out = np.zeros(n, dtype=np.float64)
    idx = np.arange(n, dtype=np.uint64)
    ilo, ihi = idx & MASK, idx >> np.uint64(32)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    lam64 = lam32.astype(np.float64)
    out[np.isnan(lam64)] = np.nan
    small = (lam64 > 0) & (lam64 < 10)
    if small.any():
        r = philox4x32_10(ilo[small], ihi[small], 0, 0, k0, k1)
        u = _u01d(r[0], r[1])
        L = lam64[small]
        p = np.exp(-L)
        s = p.copy()
        k = np.zeros_like(L)
        for _ in range(200):
            go = u > s
            if not go.any():
                break
            k = np.where(go, k + 1, k)
            p = np.where(go, p * L / np.maximum(k, 1), p)
            s = np.where(go, s + p, s)
        out[small] = k
    big = lam64 >= 10
    if big.any():
        L = lam64[big]
        bl, bh = ilo[big], ihi[big]
        slam, loglam = np.sqrt(L), np.log(L)
        b = 0.931 + 2.53 * slam
        a = -0.059 + 0.02483 * b
        invalpha = 1.1239 + 1.1328 / (b - 3.4)
        vr = 0.9277 - 3.6224 / (b - 2.0)
        res = np.full(L.shape, np.nan)
        todo = np.ones(L.shape, dtype=bool)
        for att in range(64):
            if not todo.any():
                break
            r = philox4x32_10(bl, bh, att, 0, k0, k1)
            U = _u01d(r[0], r[1]) - 0.5
            V = _u01d(r[2], r[3])
            us = 0.5 - np.abs(U)
            with np.errstate(divide="ignore", invalid="ignore"):
                k = np.floor((2.0 * a / us + b) * U + L + 0.43)
                quick = (us >= 0.07) & (V <= vr)
                reject = (k < 0) | ((us < 0.013) & (V > us))
                slow = (np.log(V) + np.log(invalpha) - np.log(a / (us * us) + b)
                        <= -L + k * loglam - gammaln(k + 1.0))
            acc = todo & (quick | (~reject & slow))
            res = np.where(acc, k, res)
            todo &= ~acc
        out[big] = res
    return out.astype(np.float32).reshape(np.shape(lam))


def gaussian(n, mu, sigma, seed):
    """The Box-Muller normals the kernel adds (purpose-1 counters), in FP64."""
    idx = np.arange(n, dtype=np.uint64)
    r = philox4x32_10(idx & MASK, idx >> np.uint64(32), 0, 1, seed & 0xFFFFFFFF, seed >> 32)
    u1, u2 = _u01f(r[0]), _u01f(r[1])
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2) * sigma + mu

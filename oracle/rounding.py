"""Rounding oracle (test infrastructure only): numpy restatement of the FP32 -> 16-bit rounding
of tigre_sart_update, bit for bit, given the same FP32 values.

* nearest: IEEE round-to-nearest-even (numpy astype for FP16; bit arithmetic for BF16, which
  numpy lacks);
* stochastic, BF16: add 16 random bits to the FP32 pattern, keep the upper half;
* stochastic, FP16: round-up neighbour when (r + 1/2) / 2^16 < (v - lo) / (hi - lo).

Random bits: Philox4x32-10 (oracle.noise.philox4x32_10) with key = seed and counter =
{g, z, step_lo, step_hi}, g = voxel index within the z plane // 8; voxel 8g + e of the plane
takes the low (e even) or high (e odd) 16 bits of word e // 2.
"""
from __future__ import annotations

import numpy as np

from .noise import philox4x32_10


def random16(nz, nyx, seed, step):
    """(nz, nyx) uint32 array of the 16-bit random values each voxel draws."""
    ng = (nyx + 7) // 8
    g = np.tile(np.arange(ng, dtype=np.uint64), nz)
    z = np.repeat(np.arange(nz, dtype=np.uint64), ng)
    r = np.stack(philox4x32_10(g, z, step & 0xFFFFFFFF, step >> 32, seed & 0xFFFFFFFF, seed >> 32), axis=1)
    r = r.reshape(nz, ng, 4)
    halves = np.stack([r & 0xFFFF, r >> 16], axis=-1).reshape(nz, ng * 8)
    return halves[:, :nyx].astype(np.uint32)


def bf16_bits_nearest(v32):
    b = np.ascontiguousarray(v32, dtype=np.float32).view(np.uint32).astype(np.uint64)
    special = (b & 0x7F800000) == 0x7F800000
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    nan = special & ((b & 0x7FFFFF) != 0)
    r = np.where(special, b >> 16, r)
    r = np.where(nan, (b >> 16) | 0x40, r)   # quiet NaN
    return r.astype(np.uint16)


def bf16_bits_stochastic(v32, r16):
    b = np.ascontiguousarray(v32, dtype=np.float32).view(np.uint32).astype(np.uint64)
    special = (b & 0x7F800000) == 0x7F800000
    out = (b + r16.astype(np.uint64)) >> 16
    # a finite value rounded past the largest finite BF16 saturates to it, keeping its sign
    out = np.where((out & 0x7F80) == 0x7F80, ((b >> 16) & 0x8000) | 0x7F7F, out)
    return np.where(special, bf16_bits_nearest(v32).astype(np.uint64), out).astype(np.uint16)


def bf16_to_f32(bits):
    return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32)


def f16_stochastic(v32, r16):
    v = np.ascontiguousarray(v32, dtype=np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        h = v.astype(np.float16)
        hf = h.astype(np.float32)
        lo = np.where(hf > v, np.nextafter(h, np.float16(-np.inf)), h)
        hi = np.where(hf < v, np.nextafter(h, np.float16(np.inf)), h)
        lf, hf2 = lo.astype(np.float32), hi.astype(np.float32)
        p = (v - lf) / (hf2 - lf)
        u = (r16.astype(np.float32) + np.float32(0.5)) * np.float32(1.0 / 65536.0)
        out = np.where(u < p, hi, lo)
        out = np.where(~(hf2 > lf), lo, out)
        out = np.where(np.isinf(lf) & (hf2 > lf), hi, out)
    return out


def sart_update(x, bp, v, lmbda, noneg, dtype, rounding="nearest", seed=0, step=0):
    """x <- round(max(x + (lmbda / v) * bp, 0)) with x given as float32 values of the storage type;
    returns the new values as float32 (FP16 / BF16 values exactly representable)."""
    x = np.asarray(x, dtype=np.float32)
    nz = x.shape[0]
    nyx = int(np.prod(x.shape[1:]))
    t = (np.float32(lmbda) / np.asarray(v, dtype=np.float32)).reshape(1, nyx)
    r = x.reshape(nz, nyx) + t * np.asarray(bp, dtype=np.float32).reshape(nz, nyx)
    if noneg:
        r = np.where(r < 0, np.float32(0), r)
    r = r.astype(np.float32)
    if dtype == "float32":
        out = r
    elif dtype == "bfloat16":
        bits = bf16_bits_nearest(r) if rounding == "nearest" else bf16_bits_stochastic(r, random16(nz, nyx, seed,
                                                                                                    step))
        out = bf16_to_f32(bits)
    elif dtype == "float16":
        with np.errstate(over="ignore"):
            out = (r.astype(np.float16) if rounding == "nearest"
                   else f16_stochastic(r, random16(nz, nyx, seed, step))).astype(np.float32)
    else:
        raise ValueError(dtype)
    return out.reshape(x.shape)

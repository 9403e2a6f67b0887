"""Seeded initial conditions for the benchmark workloads.

The reference seeds C rand() (samples/standalone/model/host_memory.cc:617) and
its acHostMeshRandomize uses unseeded rand() (src/core/astaroth.cc:243-258);
neither is reproducible across platforms. The workloads here therefore use a
counter-based generator: SplitMix64 of (seed, field, global interior index),
mapped to a double in [-1, 1). The same key gives the same value anywhere, so
meshes of any size can be regenerated plane by plane and compared exactly.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import NGHOST, NUM_VTXBUF_HANDLES

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLD = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + _GOLD
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, field: int, idx: np.ndarray) -> np.ndarray:
    """U(-1, 1) keyed by (seed, field, idx); idx is a uint64 array of linear
    interior indices i + j*nx + k*nx*ny."""
    key = np.uint64((seed & 0xFFFFFFFF) << 32 | (field & 0xFF) << 24)
    with np.errstate(over="ignore"):
        h = _splitmix64(idx.astype(np.uint64) * np.uint64(0x100000001B3) ^ key)
    # 53 random bits -> [0, 1) -> [-1, 1)
    u = (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def noise_interior(seed: int, field: int, nx: int, ny: int, nz: int, amplitude: float,
                   k0: int = 0, k1: int | None = None) -> np.ndarray:
    """amplitude * U(-1,1) on interior planes [k0, k1) as float64, shape (k1-k0, ny, nx)."""
    k1 = nz if k1 is None else k1
    base = np.uint64(k0) * np.uint64(nx * ny)
    idx = base + np.arange((k1 - k0) * ny * nx, dtype=np.uint64)
    return (amplitude * uniform_pm1(seed, field, idx)).reshape(k1 - k0, ny, nx)


def noise_interior_torch(seed: int, field: int, nx: int, ny: int, nz: int, amplitude: float,
                         device="cuda"):
    """Same values as noise_interior (bit for bit), generated with torch on
    `device`; int64 arithmetic wraps like uint64, logical shifts are masked."""
    import torch

    def lsr(x, s):
        return (x >> s) & ((1 << (64 - s)) - 1)

    def as_i64(u: int) -> int:
        return u - (1 << 64) if u >= (1 << 63) else u

    m1, m2, gold = as_i64(0xBF58476D1CE4E5B9), as_i64(0x94D049BB133111EB), as_i64(0x9E3779B97F4A7C15)
    mul = as_i64(0x100000001B3)
    key = as_i64(((seed & 0xFFFFFFFF) << 32) | ((field & 0xFF) << 24))
    out = torch.empty((nz, ny, nx), dtype=torch.float64, device=device)
    plane = nx * ny
    chunk = max(1, (1 << 26) // plane)
    for k0 in range(0, nz, chunk):
        k1 = min(nz, k0 + chunk)
        idx = torch.arange(k0 * plane, k1 * plane, dtype=torch.int64, device=device)
        z = (idx * mul) ^ key
        z = z + gold
        z = (z ^ lsr(z, 30)) * m1
        z = (z ^ lsr(z, 27)) * m2
        z = z ^ lsr(z, 31)
        u = lsr(z, 11).to(torch.float64) * (1.0 / 9007199254740992.0)
        out[k0:k1] = (amplitude * (2.0 * u - 1.0)).reshape(k1 - k0, ny, nx)
    return out


def workload_fields_torch(nx: int, ny: int, nz: int, dtype, seed: int = 1,
                          amplitude: float = 1e-3, velocity_mode: float = 0.0, device="cuda"):
    """Torch twin of workload_fields: returns eight (nz+6, ny+6, nx+6) tensors of
    `dtype` (a torch dtype) with periodic ghosts, equal to the numpy version."""
    return [workload_field_torch(w, nx, ny, nz, dtype, seed, amplitude, velocity_mode, device)
            for w in range(NUM_VTXBUF_HANDLES)]


def workload_field_torch(w: int, nx: int, ny: int, nz: int, dtype, seed: int = 1,
                         amplitude: float = 1e-3, velocity_mode: float = 0.0, device="cuda"):
    """Field w of workload_fields_torch alone (for meshes too large to hold
    all eight initial fields beside the solver's state)."""
    import torch

    f = noise_interior_torch(seed, w, nx, ny, nz, amplitude, device)
    if velocity_mode and w in (1, 2, 3):
        axis, n = {1: ("y", ny), 2: ("z", nz), 3: ("x", nx)}[w]
        s = velocity_mode * torch.sin(
            2.0 * (2.0 * math.pi / n) * torch.arange(n, dtype=torch.float64, device=device))
        if axis == "x":
            f += s[None, None, :]
        elif axis == "y":
            f += s[None, :, None]
        else:
            f += s[:, None, None]
    g = f.to(dtype)
    del f
    g = torch.cat([g[-NGHOST:], g, g[:NGHOST]], dim=0)
    g = torch.cat([g[:, -NGHOST:], g, g[:, :NGHOST]], dim=1)
    g = torch.cat([g[:, :, -NGHOST:], g, g[:, :, :NGHOST]], dim=2)
    return g.contiguous()


def wrap_ghosts(interior: np.ndarray) -> np.ndarray:
    """Pad an interior (nz, ny, nx) array with NGHOST periodic ghost cells per side;
    equal to applying the reference's periodic boundary conditions."""
    return np.pad(interior, NGHOST, mode="wrap")


def workload_fields(nx: int, ny: int, nz: int, dtype, seed: int = 1, amplitude: float = 1e-3,
                    velocity_mode: float = 0.0, ds: float | None = None) -> list[np.ndarray]:
    """The eight initial fields of the benchmark workloads, ghosts filled.

    - all fields: amplitude * U(-1, 1) noise from (seed, field, index);
    - velocity_mode != 0 adds the k=2 mode u = A (sin 2y, sin 2z, sin 2x)
      with x = (i - NGHOST) * ds, ds = 2*pi/n by default (the 512^3 workload).
    Values are formed in float64 and rounded once to `dtype`."""
    out = []
    for w in range(NUM_VTXBUF_HANDLES):
        f = noise_interior(seed, w, nx, ny, nz, amplitude)
        if velocity_mode and w in (1, 2, 3):
            # ux depends on y, uy on z, uz on x
            axis, n = {1: ("y", ny), 2: ("z", nz), 3: ("x", nx)}[w]
            step = 2.0 * math.pi / n if ds is None else ds
            s = velocity_mode * np.sin(2.0 * step * np.arange(n))
            if axis == "x":
                f = f + s[None, None, :]
            elif axis == "y":
                f = f + s[None, :, None]
            else:
                f = f + s[:, None, None]
        out.append(wrap_ghosts(f.astype(dtype)))
    return out

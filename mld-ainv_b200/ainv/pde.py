"""Synthetic operators and right-hand sides for the benchmark workloads.

7-point 3-D operator on an idim^3 unit-cube grid with Dirichlet boundaries,
unknowns numbered x fastest (row = ix + idim*(iy + idim*iz)), columns in
ascending order.  'poisson': diagonal 6, off-diagonals -1 (unscaled).
'convdiff': -Lap(u) + b.grad(u) with h = 1/(idim+1), central differences for
diffusion and first-order upwind for convection.

Random vectors come from a counter-based splitmix64 stream
u_i = top53(splitmix64((seed << 40) + i)) / 2^53, so host and device inputs
are reproducible element by element.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def gen_pde3d(idim: int, kind: str = "poisson", beta=(0.0, 0.0, 0.0)):
    """Returns (irp int32[n+1], ja int32[nnz], val float64[nnz])."""
    m = int(idim)
    n = m ** 3
    if kind == "poisson":
        lo = [-1.0, -1.0, -1.0]
        up = [-1.0, -1.0, -1.0]
        diag = 6.0
    elif kind == "convdiff":
        h = 1.0 / (m + 1)
        ih2 = 1.0 / (h * h)
        diag = 6.0 * ih2
        lo, up = [0.0] * 3, [0.0] * 3
        for a in range(3):
            b = float(beta[a])
            lo[a] = -ih2 - (b if b > 0 else 0.0) / h
            up[a] = -ih2 + (b if b < 0 else 0.0) / h
            diag += abs(b) / h
    else:
        raise ValueError(f"unknown kind {kind!r}")
    r = np.arange(n, dtype=np.int64)
    ix, iy, iz = r % m, (r // m) % m, r // (m * m)
    offs = np.array([-m * m, -m, -1, 0, 1, m, m * m], dtype=np.int64)
    valid = np.stack([iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < m - 1, iy < m - 1,
                      iz < m - 1], axis=1)
    vals = np.array([lo[2], lo[1], lo[0], diag, up[0], up[1], up[2]])
    cols = (r[:, None] + offs[None, :])[valid]
    v = np.broadcast_to(vals, (n, 7))[valid]
    irp = np.zeros(n + 1, np.int64)
    np.cumsum(valid.sum(axis=1), out=irp[1:])
    return irp.astype(np.int32), cols.astype(np.int32), np.ascontiguousarray(v, np.float64)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def _u01(seed: int, idx: np.ndarray) -> np.ndarray:
    base = np.uint64((int(seed) << 40) & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        x = _splitmix64(base + idx.astype(np.uint64))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def rand_uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    return lo + (hi - lo) * _u01(seed, np.arange(n, dtype=np.uint64))


def rand_normal(seed: int, n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.uint64)
    u1 = _u01(seed, 2 * i)
    u2 = _u01(seed, 2 * i + 1)
    return np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(6.283185307179586476925286766559 * u2)

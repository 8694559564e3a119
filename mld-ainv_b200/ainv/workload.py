"""Synthetic serving workload: resident operators and a request stream.

Operators: 3-D Poisson (6/-1) or convection-diffusion (upwind, convection
magnitude U(0, 20) in a random direction) on n^3 grids, n log-uniform in
[24, 128].  Requests: Poisson arrivals at a given mean rate, each against a
uniformly drawn operator, with an N(0, 1) right-hand side seeded by the
request id.  All draws come from the counter-based splitmix64 streams of
`pde`, so every platform builds the same workload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import pde


@dataclass(frozen=True)
class OperatorSpec:
    idim: int
    kind: str                  # "poisson" | "convdiff"
    beta: tuple                # convection vector (zeros for Poisson)

    @property
    def n(self) -> int:
        return self.idim ** 3


def serving_operators(count: int = 16, seed: int = 5, nmin: int = 24, nmax: int = 128):
    u = pde.rand_uniform(seed, 3 * count, 0.0, 1.0).reshape(count, 3)
    g = pde.rand_normal(seed + 1, 3 * count).reshape(count, 3)
    out = []
    for k in range(count):
        idim = int(round(math.exp(math.log(nmin) + u[k, 0] * (math.log(nmax) - math.log(nmin)))))
        idim = min(max(idim, nmin), nmax)
        if u[k, 1] < 0.5:
            out.append(OperatorSpec(idim, "poisson", (0.0, 0.0, 0.0)))
        else:
            mag = 20.0 * u[k, 2]
            d = g[k] / max(np.linalg.norm(g[k]), 1e-300)
            out.append(OperatorSpec(idim, "convdiff", tuple(float(mag * c) for c in d)))
    return out


def poisson_arrivals(rate: float, count: int, seed: int = 11) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson process of the given rate."""
    u = pde.rand_uniform(seed, count, 0.0, 1.0)
    return np.cumsum(-np.log1p(-u) / rate)


def request_ops(count: int, nops: int, seed: int = 13) -> np.ndarray:
    u = pde.rand_uniform(seed, count, 0.0, 1.0)
    return np.minimum((u * nops).astype(np.int64), nops - 1)


def request_rhs(request_id: int, n: int) -> np.ndarray:
    """N(0, 1) right-hand side seeded by the request id."""
    return pde.rand_normal(request_id, n)

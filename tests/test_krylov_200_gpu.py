"""Iteration parity at full size: the 200^3 convection-diffusion case
(n = 8,000,000, upwind convection, beta = 10(1,1,1)/sqrt(3), b = A x* with
x* ~ U(-1,1) seed 0, BiCGSTAB to 1e-9, x0 = 0) preconditioned by AINV (drop
0.1, cap 20), INVK (fill 1, 1) and INVT (0.05, 20).

With FP64 factors the device loop sums its dots in the canonical order and
rounds every FP64 operation separately, like the oracle's loop in its
"device" dot order, so the device must reproduce the oracle's iteration
count, residual history and solution bit for bit (tests/pdegen/ppde3d.f90:
276-281 is the reference driver of this solve)."""
import numpy as np
import pytest

import ainv
import oracle as O
from test_krylov_gpu import _same_iterates, _true_relres
from util import build_factors, build_inverse_factors, device_factors, oracle_factors

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.slow]
CONVDIFF = (10 / np.sqrt(3),) * 3


@pytest.fixture(scope="module")
def convdiff200():
    irp, ja, val = ainv.pde.gen_pde3d(200, "convdiff", CONVDIFF)
    n = len(irp) - 1
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    return irp, ja, val, b


@pytest.mark.parametrize("solver", ["AINV", "INVK", "INVT"])
def test_bicgstab_200_same_iterates(convdiff200, solver):
    irp, ja, val, b = convdiff200
    f = (build_factors(irp, ja, val) if solver == "AINV"
         else build_inverse_factors(solver, irp, ja, val))
    df = device_factors(f)
    res, xs = _same_iterates("BICGSTAB", irp, ja, val, oracle_factors(f), df, b, 1e-9, 1000)
    assert res.err <= 1e-9
    assert _true_relres(irp, ja, val, xs, b) <= 1e-9

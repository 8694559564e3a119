"""GPU apply and Krylov loop with INVK / INVT factors (the same device
layout and kernels as AINV: W^T ~ L^-1 lower, Z ~ U^-1 upper, d the
inverted ILU pivots), against the CPU oracle on the same factors.

Tolerances as for AINV: FP64 apply 1e-12, FP32 5e-6, BF16 3e-2 (norm-wise
relative); FP64 solves compute the oracle's iterates bit for bit (same
count, residual history and solution), and mixed-precision solves reach
the FP64 relative residual 1e-9.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import ainv
import oracle as O
from test_krylov_gpu import _same_iterates, _t, _true_relres
from util import build_inverse_factors, device_factors, oracle_factors, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = {"FP64": 1e-12, "FP32": 5e-6, "BF16": 3e-2}
CONVDIFF = (10 / np.sqrt(3),) * 3


def _gpu_apply(df, x, alpha, beta, y0, trans):
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(DEV)
    yd = torch.from_numpy(np.ascontiguousarray(y0)).to(DEV)
    df.apply(xd, yd, alpha, beta, trans)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
@pytest.mark.parametrize("idim,kind,beta", [
    (40, "poisson", (0, 0, 0)),
    (45, "convdiff", CONVDIFF),
    (21, "convdiff", (90.0, -40.0, 25.0)),
])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_fp64_parity(solver, idim, kind, beta, trans):
    irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
    f = build_inverse_factors(solver, irp, ja, val)
    of = oracle_factors(f)
    n = len(f["d"])
    x, y0 = ainv.pde.rand_uniform(21, n), ainv.pde.rand_uniform(22, n)
    df = device_factors(f)
    for alpha, beta_ in [(1.0, 0.0), (1.5, 0.5), (-2.0, 1.0)]:
        y = _gpu_apply(df, x, alpha, beta_, y0, trans)
        ref = O.ainv_apply(of, x, alpha, beta_, y0, trans)
        assert relerr(y, ref) <= 1e-12, (alpha, beta_)
        if trans == "N":  # same operations in the same order: the same bits
            np.testing.assert_array_equal(y, ref)


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
@pytest.mark.parametrize("prec", ["FP32", "BF16"])
def test_apply_mixed_precision(solver, prec):
    irp, ja, val = ainv.pde.gen_pde3d(30, "convdiff", CONVDIFF)
    f = build_inverse_factors(solver, irp, ja, val)
    n = len(f["d"])
    x, y0 = ainv.pde.rand_uniform(3, n), ainv.pde.rand_uniform(4, n)
    df = device_factors(f, prec)
    for trans in ("N", "T"):
        y = _gpu_apply(df, x, 1.25, -0.5, y0, trans)
        ref = O.ainv_apply(oracle_factors(f), x, 1.25, -0.5, y0, trans)
        assert relerr(y, ref) <= TOL[prec], trans


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
def test_apply_full_size_convdiff_200(solver):
    """200^3 convection-diffusion INVK(1) / INVT(0.05, 20) factors: GPU vs
    oracle apply, and linearity of the device apply."""
    irp, ja, val = ainv.pde.gen_pde3d(200, "convdiff", CONVDIFF)
    f = build_inverse_factors(solver, irp, ja, val)
    n = len(f["d"])
    x = ainv.pde.rand_uniform(0, n)
    df = device_factors(f)
    y = _gpu_apply(df, x, 1.0, 0.0, np.zeros(n), "N")
    assert relerr(y, O.ainv_apply(oracle_factors(f), x)) <= 1e-12
    x2 = ainv.pde.rand_uniform(1, n)
    y2 = _gpu_apply(df, x2, 1.0, 0.0, np.zeros(n), "N")
    y12 = _gpu_apply(df, 2.0 * x - 3.0 * x2, 1.0, 0.0, np.zeros(n), "N")
    assert relerr(y12, 2.0 * y - 3.0 * y2) <= 1e-12


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
def test_bicgstab_convdiff(solver):
    """Convection-diffusion, b = A x*, x* ~ U(-1,1) seed 0, BiCGSTAB to 1e-9
    preconditioned by INVK / INVT: the oracle's iterates."""
    irp, ja, val = ainv.pde.gen_pde3d(40, "convdiff", CONVDIFF)
    n = len(irp) - 1
    f = build_inverse_factors(solver, irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    _, xs = _same_iterates("BICGSTAB", irp, ja, val, oracle_factors(f), device_factors(f), b,
                           1e-9, 2000)
    assert _true_relres(irp, ja, val, xs, b) <= 1e-9


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
def test_mixed_factors_reach_fp64_tolerance(solver):
    irp, ja, val = ainv.pde.gen_pde3d(40, "convdiff", CONVDIFF)
    n = len(irp) - 1
    f = build_inverse_factors(solver, irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    A = ainv.DeviceOperator(irp, ja, val)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(_t(b), x, device_factors(f, "FP32"), "BICGSTAB", 1e-9, 2000)
    assert res.converged, res
    assert _true_relres(irp, ja, val, x.cpu().numpy(), b) <= 1e-9


def test_invk_cg_on_poisson():
    """Poisson is symmetric, so ILU(k) gives L = U^T and INVK gives W = Z:
    the preconditioner is symmetric and CG applies."""
    irp, ja, val = ainv.pde.gen_pde3d(40, "poisson")
    n = len(irp) - 1
    f = build_inverse_factors("INVK", irp, ja, val)
    Wt = sp.csr_matrix((f["wt_val"], f["wt_ja"], f["wt_irp"]), shape=(n, n))
    Z = sp.csr_matrix((f["z_val"], f["z_ja"], f["z_irp"]), shape=(n, n))
    assert abs(Wt.T - Z).max() <= 1e-15 * abs(Z).max()
    b = O.spmv(O.CSR(n, irp, ja, val), np.ones(n))
    _same_iterates("CG", irp, ja, val, oracle_factors(f), device_factors(f), b, 1e-9, 1000)

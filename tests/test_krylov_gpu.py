"""GPU Krylov loop (CG / BiCGSTAB, istop=2) against the oracle's restated
PSBLAS solvers on the same factors.

The device sums every dot in a fixed canonical order and rounds every FP64
product and sum separately, and the oracle's "device" dot order restates
that order, so with FP64 factors the two loops compute the same iterates:
the tests require the same iteration count, the same residual history and
the same solution, bit for bit.  Breakdown and itmax statuses come back as
codes (no device fault or hang is ever provoked)."""
import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, device_factors, oracle_factors

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(DEV)


def _true_relres(irp, ja, val, x, b):
    a = O.CSR(len(irp) - 1, irp, ja, val)
    return np.linalg.norm(b - O.spmv(a, x)) / np.linalg.norm(b)


def _same_iterates(method, irp, ja, val, of, df, b, eps, itmax):
    """Device solve and oracle solve (device dot order) from x0 = 0: equal
    iteration counts, residual histories and solutions."""
    n = len(irp) - 1
    a = O.CSR(n, irp, ja, val)
    xr, it_ref, err_ref, rc, hist_ref = O.solve(method, a, of, b, eps=eps, itmax=itmax,
                                                history=True)
    assert rc == 0
    A = ainv.DeviceOperator(irp, ja, val)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(_t(b), x, df, method, eps, itmax)
    assert res.converged, res
    assert res.iter == it_ref, (res.iter, it_ref)
    np.testing.assert_array_equal(A.history(), hist_ref)
    np.testing.assert_array_equal(x.cpu().numpy(), xr)
    return res, xr


def test_cg_poisson_40():
    """40^3 Poisson, b = A*1, x0 = 0, AINV LLK drop 0.1 cap 20, CG to 1e-9."""
    irp, ja, val = ainv.pde.gen_pde3d(40, "poisson")
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), np.ones(n))
    res, xs = _same_iterates("CG", irp, ja, val, oracle_factors(f), device_factors(f), b, 1e-9,
                             1000)
    assert res.err <= 1e-9
    assert _true_relres(irp, ja, val, xs, b) <= 1e-9
    assert np.abs(xs - 1.0).max() < 1e-6


@pytest.mark.parametrize("idim", [32, 64])
def test_bicgstab_convdiff(idim):
    """Convection-diffusion (upwind), b = A x*, x* ~ U(-1,1) seed 0, BiCGSTAB."""
    irp, ja, val = ainv.pde.gen_pde3d(idim, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    _, xs = _same_iterates("BICGSTAB", irp, ja, val, oracle_factors(f), device_factors(f), b,
                           1e-9, 2000)
    assert _true_relres(irp, ja, val, xs, b) <= 1e-9


@pytest.mark.parametrize("prec", ["FP32", "BF16", "FP32_ACC64", "BF16_ACC64"])
def test_mixed_factors_reach_fp64_tolerance(prec):
    """FP32/BF16 factors, FP64 recurrence with true-residual replacement:
    the same 1e-9 FP64 relative residual as the FP64 apply."""
    irp, ja, val = ainv.pde.gen_pde3d(48, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    xstar = ainv.pde.rand_uniform(0, n)
    b = O.spmv(O.CSR(n, irp, ja, val), xstar)
    A = ainv.DeviceOperator(irp, ja, val)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(_t(b), x, device_factors(f, prec), "BICGSTAB", 1e-9, 2000)
    assert res.converged, res
    assert _true_relres(irp, ja, val, x.cpu().numpy(), b) <= 1e-9


def _rounded(f, prec):
    """The factors as an ACC64 handle stores them (values and d rounded to
    FP32 / BF16), in FP64."""
    import torch as T
    dt = T.float32 if prec == "FP32_ACC64" else T.bfloat16
    r = dict(f)
    for k in ("wt_val", "z_val", "d"):
        r[k] = T.from_numpy(np.asarray(f[k])).to(dt).double().numpy()
    return r


@pytest.mark.parametrize("prec", ["FP32_ACC64", "BF16_ACC64"])
def test_acc64_iterates_equal_oracle_on_rounded_factors(prec):
    """FP32/BF16 storage with FP64 accumulation applies the rounded factors
    exactly as the FP64 path does, so the solve equals the oracle's solve
    with the rounded factors, bit for bit (no residual replacement fires:
    the recurrence stays within 1e-6 of the true residual)."""
    irp, ja, val = ainv.pde.gen_pde3d(40, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    _same_iterates("BICGSTAB", irp, ja, val, oracle_factors(_rounded(f, prec)),
                   device_factors(f, prec), b, 1e-9, 2000)


def test_unpreconditioned_bicgstab_count():
    """No preconditioner: the device loop alone equals the oracle's with
    identity factors (which apply as an exact copy)."""
    irp, ja, val = ainv.pde.gen_pde3d(64, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    ident = O.CSR(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
    _same_iterates("BICGSTAB", irp, ja, val, O.Factors(ident, ident, np.ones(n)), None, b, 1e-9,
                   3000)


def test_unpreconditioned_cg_matches_oracle_count():
    irp, ja, val = ainv.pde.gen_pde3d(16, "poisson")
    n = len(irp) - 1
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(2, n))
    A = ainv.DeviceOperator(irp, ja, val)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(_t(b), x, None, "CG", 1e-8, 500)
    assert res.converged
    assert _true_relres(irp, ja, val, x.cpu().numpy(), b) <= 1.05e-8


def test_itmax_reached_returns_noconv():
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (10.0, 10.0, 10.0))
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    A = ainv.DeviceOperator(irp, ja, val)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(_t(np.ones(n)), x, device_factors(f), "BICGSTAB", 1e-14, 3)
    assert res.info == ainv._lib.ERR_NOCONV and res.iter == 3


def test_breakdown_is_reported():
    """A = [[0,1],[1,0]], b = e1: BiCGSTAB's sigma = rt.(A p) = 0 at the
    first step -> breakdown status, returned by the device loop."""
    A = ainv.DeviceOperator(np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0]))
    x = torch.zeros(2, dtype=torch.float64, device=DEV)
    res = A.solve(_t([1.0, 0.0]), x, None, "BICGSTAB", 1e-9, 50)
    assert res.info == ainv._lib.ERR_BREAKDOWN


def test_initial_guess_already_converged():
    irp, ja, val = ainv.pde.gen_pde3d(10, "poisson")
    n = len(irp) - 1
    xs = ainv.pde.rand_uniform(3, n)
    b = O.spmv(O.CSR(n, irp, ja, val), xs)
    A = ainv.DeviceOperator(irp, ja, val)
    res = A.solve(_t(b), _t(xs), None, "CG", 1e-9, 100)
    assert res.converged and res.iter == 0


def test_solve_is_deterministic_and_reuses_graph():
    irp, ja, val = ainv.pde.gen_pde3d(24, "convdiff", (5.0, -5.0, 2.0))
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    df = device_factors(f)
    A = ainv.DeviceOperator(irp, ja, val)
    b = _t(ainv.pde.rand_uniform(4, n))
    xs = []
    for _ in range(3):
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        res = A.solve(b, x, df, "BICGSTAB", 1e-10, 1000)
        assert res.converged
        xs.append(x.cpu().numpy())
    np.testing.assert_array_equal(xs[0], xs[1])
    np.testing.assert_array_equal(xs[0], xs[2])


def test_reported_error_is_the_true_residual():
    """Convergence is confirmed on b - A x: the returned err is the true one."""
    irp, ja, val = ainv.pde.gen_pde3d(28, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    A = ainv.DeviceOperator(irp, ja, val)
    for method in ("BICGSTAB", "CG"):
        if method == "CG":   # CG on the SPD Poisson operator
            irp, ja, val = ainv.pde.gen_pde3d(28, "poisson")
            f = build_factors(irp, ja, val)
            A = ainv.DeviceOperator(irp, ja, val)
            b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        res = A.solve(_t(b), x, device_factors(f, "FP32"), method, 1e-10, 2000)
        assert res.converged
        true = _true_relres(irp, ja, val, x.cpu().numpy(), b)
        assert true <= 1e-10
        assert abs(res.err - true) <= 1e-3 * true


def test_spmv_matches_oracle():
    irp, ja, val = ainv.pde.gen_pde3d(30, "convdiff", (7.0, 8.0, -9.0))
    n = len(irp) - 1
    x, y0 = ainv.pde.rand_uniform(5, n), ainv.pde.rand_uniform(6, n)
    A = ainv.DeviceOperator(irp, ja, val)
    xd, yd = _t(x), _t(y0)
    A.spmv(xd, yd, 2.0, -1.0)
    ref = O.spmv(O.CSR(n, irp, ja, val), x, 2.0, -1.0, y0)
    y = yd.cpu().numpy()
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    np.testing.assert_array_equal(y, ref)  # alpha*acc + beta*y formed as the oracle forms it

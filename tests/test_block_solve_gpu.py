"""Multi-right-hand-side CG (ainv_gpu_block_solve) on the GPU.

Each column follows the single-vector CG recurrence with the same per-row
arithmetic, so every column is held to the single-vector bar: it reaches
the FP64 relative residual 1e-9 on b - A x, and its iteration count lies
within 5% of the oracle CG's rounding-level spread (FP64 factors) or of the
single-vector GPU solve with the same FP32 factors.
"""
import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, device_factors, oracle_factors, oracle_spread, within_spread

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _rhs(n, m, seed0=0):
    return np.stack([ainv.pde.rand_normal(seed0 + k, n) for k in range(m)], axis=1)


def _relres(a, x, b):
    return np.linalg.norm(b - O.spmv(a, x)) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_block_cg_poisson_matches_single(prec):
    irp, ja, val = ainv.pde.gen_pde3d(24, "poisson")
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    a = O.CSR(n, irp, ja, val)
    m = 32
    Bh = _rhs(n, m)
    A = ainv.DeviceOperator(irp, ja, val)
    df = device_factors(f, prec)
    B = torch.from_numpy(Bh).to(DEV)
    X = torch.zeros_like(B)
    res = A.block_solve(B, X, df, 1e-9, 1000)
    assert res.converged, res
    Xh = X.cpu().numpy()
    for l in range(m):
        assert _relres(a, Xh[:, l], Bh[:, l]) <= 1.05e-9
        assert res.errs[l] <= 1e-9
    for l in (0, 7, 31):
        b = Bh[:, l].copy()
        x1 = torch.zeros(n, dtype=torch.float64, device=DEV)
        single = A.solve(torch.from_numpy(b).to(DEV), x1, df, "CG", 1e-9, 1000)
        if prec == "FP64":
            lo, hi = oracle_spread("CG", a, oracle_factors(f), b, 1e-9, 1000, k=3)
            assert within_spread(res.iters[l], lo, hi), (l, res.iters[l], lo, hi)
        assert abs(res.iters[l] - single.iter) <= max(1, int(np.ceil(0.05 * single.iter))), \
            (l, res.iters[l], single.iter)
        np.testing.assert_allclose(Xh[:, l], x1.cpu().numpy(), rtol=0, atol=1e-7)


@pytest.mark.parametrize("m", [1, 5, 17])
def test_block_cg_fewer_columns_and_ld(m):
    """m < 32 columns with a leading dimension larger than m."""
    irp, ja, val = ainv.pde.gen_pde3d(13, "poisson")
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    A = ainv.DeviceOperator(irp, ja, val)
    df = device_factors(f, "FP32")
    Bh = _rhs(n, m, 100)
    B = torch.from_numpy(Bh).to(DEV)
    X = torch.zeros_like(B)
    res = A.block_solve(B, X, df, 1e-9, 1000)
    assert res.converged and len(res.iters) == m
    a = O.CSR(n, irp, ja, val)
    for l in range(m):
        assert _relres(a, X.cpu().numpy()[:, l], Bh[:, l]) <= 1.05e-9
    # wider leading dimension through the C-ABI directly
    import ctypes as C
    ld = m + 3
    Bw = torch.zeros((n, ld), dtype=torch.float64, device=DEV)
    Bw[:, :m] = B
    Xw = torch.full((n, ld), 5.0, dtype=torch.float64, device=DEV)
    Xw[:, :m] = 0.0
    it = (C.c_int * m)()
    info = ainv.lib().ainv_gpu_block_solve(df.handle, A.handle, m,
                                           C.c_void_p(Bw.data_ptr()), ld,
                                           C.c_void_p(Xw.data_ptr()), ld, 1e-9, 1000, it,
                                           None, None, None)
    assert info == 0 and list(it) == res.iters
    assert torch.equal(Xw[:, :m], X) and bool((Xw[:, m:] == 5.0).all())


def test_block_cg_zero_column_and_itmax():
    irp, ja, val = ainv.pde.gen_pde3d(12, "poisson")
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    A = ainv.DeviceOperator(irp, ja, val)
    Bh = _rhs(n, 4)
    Bh[:, 2] = 0.0
    B = torch.from_numpy(Bh).to(DEV)
    X = torch.zeros_like(B)
    df = device_factors(f)
    res = A.block_solve(B, X, df, 1e-9, 1000)
    assert res.converged and res.iters[2] == 0
    assert float(X[:, 2].abs().max()) == 0.0
    X.zero_()
    res = A.block_solve(B, X, df, 1e-12, 3)
    assert res.info == 4104 and res.status[2] == 0 and res.status[0] == 4104
    assert res.iters[0] == 3


def test_block_cg_unpreconditioned():
    irp, ja, val = ainv.pde.gen_pde3d(10, "poisson")
    n = len(irp) - 1
    A = ainv.DeviceOperator(irp, ja, val)
    Bh = _rhs(n, 3, 50)
    B = torch.from_numpy(Bh).to(DEV)
    X = torch.zeros_like(B)
    res = A.block_solve(B, X, None, 1e-9, 2000)
    assert res.converged
    a = O.CSR(n, irp, ja, val)
    for l in range(3):
        assert _relres(a, X.cpu().numpy()[:, l], Bh[:, l]) <= 1.05e-9
        x1 = torch.zeros(n, dtype=torch.float64, device=DEV)
        single = A.solve(torch.from_numpy(Bh[:, l].copy()).to(DEV), x1, None, "CG", 1e-9, 2000)
        assert abs(res.iters[l] - single.iter) <= max(1, int(np.ceil(0.05 * single.iter)))

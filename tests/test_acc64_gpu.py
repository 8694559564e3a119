"""FP32 / BF16 factor storage with FP64 accumulation (AINV_PREC_FP32_ACC64,
AINV_PREC_BF16_ACC64): the same factor bytes as FP32 / BF16, but the apply's
products, sums and intermediate are FP64.  So the result equals the FP64
oracle apply on the *rounded* factors to 1e-12 (not just the 5e-6 / 3e-2
of FP32 accumulation), and solves follow the FP64 recurrence closely."""
import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, device_factors, oracle_factors, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _round(v, prec):
    f = np.asarray(v, np.float64).astype(np.float32)
    if prec == "FP32_ACC64":
        return f.astype(np.float64)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000          # round to nearest even
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("prec", ["FP32_ACC64", "BF16_ACC64"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_is_fp64_arithmetic_on_rounded_factors(prec, trans):
    irp, ja, val = ainv.pde.gen_pde3d(30, "convdiff", (10 / np.sqrt(3),) * 3)
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    q = dict(f)
    for k in ("wt_val", "z_val", "d"):
        q[k] = _round(f[k], prec)
    x, y0 = ainv.pde.rand_uniform(3, n), ainv.pde.rand_uniform(4, n)
    df = device_factors(f, prec)
    assert df.prec == prec
    xd, yd = torch.from_numpy(x).to(DEV), torch.from_numpy(y0).to(DEV)
    df.apply(xd, yd, 1.25, -0.5, trans)
    torch.cuda.synchronize()
    ref = O.ainv_apply(oracle_factors(q), x, 1.25, -0.5, y0, trans)
    assert relerr(yd.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("prec", ["FP32_ACC64", "BF16_ACC64"])
def test_solve_and_block_solve(prec):
    irp, ja, val = ainv.pde.gen_pde3d(40, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    df = device_factors(f, prec)
    A = ainv.DeviceOperator(irp, ja, val)
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(torch.from_numpy(b).to(DEV), x, df, "BICGSTAB", 1e-9, 2000)
    assert res.converged, res
    r = b - O.spmv(O.CSR(n, irp, ja, val), x.cpu().numpy())
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05e-9
    irp, ja, val = ainv.pde.gen_pde3d(16, "poisson")
    n = len(irp) - 1
    g = build_factors(irp, ja, val)
    dg = device_factors(g, prec)
    A = ainv.DeviceOperator(irp, ja, val)
    B = torch.from_numpy(np.stack([ainv.pde.rand_normal(k, n) for k in range(8)], 1)).to(DEV)
    X = torch.zeros_like(B)
    assert A.block_solve(B, X, dg, 1e-9, 1000).converged

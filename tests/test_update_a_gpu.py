"""update_a on the device (ainv_gpu_update_a, mld_d_solver_update_a)
against the oracle: bit-identical new d for FP64 factors (same sorted-dot
order, no fused multiply-add), close for FP32 factors; the apply after the
update matches the oracle apply with the new d to 1e-12."""
import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, build_inverse_factors, device_factors, oracle_factors, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _factors(kind):
    irp, ja, val = ainv.pde.gen_pde3d(30, "convdiff", (10 / np.sqrt(3),) * 3)
    if kind == "AINV":
        return build_factors(irp, ja, val)
    return build_inverse_factors(kind, irp, ja, val)


@pytest.mark.parametrize("kind", ["AINV", "INVK", "INVT"])
def test_fp64_update_is_bit_identical(kind):
    f = _factors(kind)
    n = len(f["d"])
    x = ainv.pde.rand_uniform(17, n, 0.0, 3.0)
    df = device_factors(f)
    d_out = torch.zeros(n, dtype=torch.float64, device=DEV)
    df.update_a(torch.from_numpy(x).to(DEV), d_out)
    torch.cuda.synchronize()
    ref = O.update_a(oracle_factors(f), x)
    np.testing.assert_array_equal(d_out.cpu().numpy(), ref)
    # the apply now uses the new d
    of = oracle_factors(f)
    of = O.Factors(of.wt, of.z, ref)
    v = ainv.pde.rand_uniform(18, n)
    for trans in ("N", "T"):
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        df.apply(torch.from_numpy(v).to(DEV), y, 1.0, 0.0, trans)
        torch.cuda.synchronize()
        assert relerr(y.cpu().numpy(), O.ainv_apply(of, v, trans=trans)) <= 1e-12


def test_fp32_update_close():
    f = _factors("AINV")
    n = len(f["d"])
    x = ainv.pde.rand_uniform(19, n, 0.0, 3.0)
    df = device_factors(f, "FP32")
    d_out = torch.zeros(n, dtype=torch.float64, device=DEV)
    df.update_a(torch.from_numpy(x).to(DEV), d_out)
    torch.cuda.synchronize()
    ref = O.update_a(oracle_factors(f), x)
    assert relerr(d_out.cpu().numpy(), ref) <= 1e-6


def test_solver_type_update_and_shifted_solve():
    irp, ja, val = ainv.pde.gen_pde3d(24, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val, amold="FP64") == 0
    f0 = sv.factors()
    shift = np.full(n, 0.5 * float(np.max(val)))
    assert sv.update_a(shift) == 0
    f1 = sv.factors()
    np.testing.assert_array_equal(f1["d"], O.update_a(oracle_factors(f0), shift))
    # a solve of the shifted system with the refreshed preconditioner
    import scipy.sparse as sp
    As = sp.csr_matrix((val, ja, irp), shape=(n, n)) + sp.diags(shift)
    As.sort_indices()
    A = ainv.DeviceOperator(As.indptr.astype(np.int32), As.indices.astype(np.int32), As.data)
    b = torch.from_numpy(As @ ainv.pde.rand_uniform(0, n)).to(DEV)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    res = A.solve(b, x, sv.device, "BICGSTAB", 1e-9, 1000)
    assert res.converged, res
    assert ainv.mld_d_ainv_solver_type().update_a(shift) == ainv._lib.ERR_NOT_BUILT


def test_reduced_precision_update_keeps_fp64_host_d():
    """With FP32 factors on the device the solver type still forms the new
    d in FP64 from its FP64 host d, so repeated updates track the oracle's
    FP64 recurrence (only the device factors' rounding enters, through e)."""
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val, amold="FP32") == 0
    of = oracle_factors(sv.factors())
    d_ref = of.d
    for k in range(3):
        shift = ainv.pde.rand_uniform(60 + k, n, 0.0, 2.0)
        assert sv.update_a(shift) == 0
        d_ref = O.update_a(O.Factors(of.wt, of.z, d_ref), shift)
        assert relerr(sv.factors()["d"], d_ref) <= 1e-6
    assert sv.update_a(np.zeros(n - 1)) == ainv._lib.ERR_ARG

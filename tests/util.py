"""Shared helpers for the GPU parity tests (oracle = CPU restatement)."""
import numpy as np

import ainv
import oracle as O


def build_factors(irp, ja, val, fill=20, thresh=0.1, alg="LLK"):
    """Product host build (mld_d_ainv_solver_type) -> dict of CSR arrays."""
    sv = ainv.mld_d_ainv_solver_type()
    sv.csetc("AINV_ALG", alg)
    sv.cseti("SUB_FILLIN", fill)
    sv.csetr("SUB_ILUTHRS", thresh)
    assert sv.build(irp, ja, val) == 0, ainv.last_error()
    return sv.factors()


def oracle_factors(f):
    n = len(f["d"])
    return O.Factors(O.CSR(n, f["wt_irp"], f["wt_ja"], f["wt_val"]),
                     O.CSR(n, f["z_irp"], f["z_ja"], f["z_val"]), f["d"])


def device_factors(f, prec="FP64"):
    return ainv.DeviceFactors((f["wt_irp"], f["wt_ja"], f["wt_val"]),
                              (f["z_irp"], f["z_ja"], f["z_val"]), f["d"], prec=prec)


def relerr(y, ref):
    """Norm-wise relative error ||y - ref||_inf / ||ref||_inf."""
    y = np.asarray(y)
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


# The 200^3 convection-diffusion variants: INVK (fill level 1) and INVT
# (threshold 0.05, fill cap 20), the sub / inverse settings taken alike.
INVK_SETTINGS = {"SUB_FILLIN": 1, "INV_FILLIN": 1}
INVT_SETTINGS = {"SUB_FILLIN": 20, "SUB_ILUTHRS": 0.05, "INV_FILLIN": 20, "INV_THRESH": 0.05}


def build_inverse_factors(solver, irp, ja, val, settings=None):
    """Product host build of INVK / INVT (mld_d_inv[kt]_solver_type)."""
    sv = ainv.mld_d_invk_solver_type() if solver == "INVK" else ainv.mld_d_invt_solver_type()
    if settings is None:
        settings = INVK_SETTINGS if solver == "INVK" else INVT_SETTINGS
    for k, v in settings.items():
        (sv.csetr if isinstance(v, float) else sv.cseti)(k, v)
    assert sv.build(irp, ja, val) == 0, ainv.last_error()
    return sv.factors()


def oracle_spread(method, a, of, b, eps, itmax, k=6):
    """Iteration counts of the oracle solve on b and on k copies of b
    perturbed at rounding level (1e-15 relative): (min, max).  Used where a
    device loop sums its dots in an order of its own (the multi-RHS CG and
    the server), so its count is judged against this spread widened by 5%."""
    rng = np.random.default_rng(7)
    its = []
    for j in range(k + 1):
        bj = b if j == 0 else b * (1.0 + 1e-15 * rng.standard_normal(len(b)))
        _, it, _, rc = O.solve(method, a, of, bj, eps=eps, itmax=itmax)
        assert rc == 0
        its.append(it)
    return min(its), max(its)


def within_spread(gpu_it, lo, hi):
    return lo - max(1, np.ceil(0.05 * lo)) <= gpu_it <= hi + max(1, np.ceil(0.05 * hi))

"""ainv_gpu_apply_csr_noalloc: the apply for callers that cannot allocate
device memory while applying (memory owned by an outside pool, or a
latency-critical section where cudaMalloc/cudaFree are not allowed).

Called through the C-ABI with caller-owned device CSR arrays, it must match
the regular entry point (ainv_gpu_create + ainv_gpu_apply) within the FP64
apply tolerance used by the other tests (1e-12 norm-wise relative), on two
calls in a row -- the second call reuses the built-in scratch array that the
first one left filled.  Collected last so a failure here does not hide the
other tests' results."""
import ctypes as C

import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, device_factors, oracle_factors, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).to(DEV)


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_apply_matches_regular_apply_twice():
    irp, ja, val = ainv.pde.gen_pde3d(48, "convdiff", (10 / np.sqrt(3),) * 3)
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    arrs = {k: _dev(f[k], np.int32 if k.endswith(("irp", "ja")) else np.float64)
            for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]}
    df = device_factors(f)
    lib = ainv.lib()
    for call, (seed, alpha, beta) in enumerate([(21, 1.0, 0.0), (22, -0.5, 2.0)]):
        x = _dev(ainv.pde.rand_uniform(seed, n), np.float64)
        y0 = ainv.pde.rand_uniform(seed + 100, n)
        y_ref = _dev(y0, np.float64)
        y_new = _dev(y0, np.float64)
        df.apply(x, y_ref, alpha, beta, "N")
        info = lib.ainv_gpu_apply_csr_noalloc(
            n, _p(arrs["wt_irp"]), _p(arrs["wt_ja"]), _p(arrs["wt_val"]), len(f["wt_ja"]),
            _p(arrs["z_irp"]), _p(arrs["z_ja"]), _p(arrs["z_val"]), len(f["z_ja"]),
            _p(arrs["d"]), alpha, _p(x), beta, _p(y_new), None)
        assert info == 0, ainv.last_error()
        torch.cuda.synchronize()
        err = relerr(y_new.cpu().numpy(), y_ref.cpu().numpy())
        assert err <= 1e-12, (call, err)


def _noalloc(f, x, alpha, beta, y0):
    """One call of the entry point on device copies of the CSR factors f."""
    n = len(f["d"])
    arrs = {k: _dev(f[k], np.int32 if k.endswith(("irp", "ja")) else np.float64)
            for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]}
    xd, yd = _dev(x, np.float64), _dev(y0, np.float64)
    info = ainv.lib().ainv_gpu_apply_csr_noalloc(
        n, _p(arrs["wt_irp"]), _p(arrs["wt_ja"]), _p(arrs["wt_val"]), len(f["wt_ja"]),
        _p(arrs["z_irp"]), _p(arrs["z_ja"]), _p(arrs["z_val"]), len(f["z_ja"]),
        _p(arrs["d"]), alpha, _p(xd), beta, _p(yd), None)
    assert info == 0, ainv.last_error()
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def test_noalloc_apply_matches_oracle_on_golden_factors():
    """The committed golden factors (convection-diffusion 6^3, LLK) against
    the oracle's apply, alpha/beta both general."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "convdiff6_llk.npz"))
    f = {k: g[k] for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]}
    n = len(f["d"])
    for seed, alpha, beta in [(31, 1.0, 0.0), (32, 0.75, -1.5)]:
        x = ainv.pde.rand_uniform(seed, n)
        y0 = ainv.pde.rand_uniform(seed + 7, n)
        ref = O.ainv_apply(oracle_factors(f), x, alpha, beta, y0)
        assert relerr(_noalloc(f, x, alpha, beta, y0), ref) <= 1e-12


def _random_triangular(n, per_row, lower, rng):
    """Unit-diagonal triangular CSR whose off-diagonal columns are drawn at
    random per row (no two rows share a pattern, unlike a stencil)."""
    irp, ja, val = [0], [], []
    for i in range(n):
        span = np.arange(0, i) if lower else np.arange(i + 1, n)
        k = min(len(span), int(rng.integers(0, per_row + 1)))
        cols = np.sort(rng.choice(span, size=k, replace=False)) if k else np.array([], int)
        cols = np.concatenate([cols, [i]]) if lower else np.concatenate([[i], cols])
        ja += cols.tolist()
        val += [1.0 if c == i else float(rng.uniform(-0.5, 0.5)) for c in cols]
        irp.append(len(ja))
    return np.array(irp, np.int32), np.array(ja, np.int32), np.array(val)


def test_noalloc_apply_scattered_pattern_twice():
    """Rows with different, scattered column sets (a non-stencil pattern),
    checked against the oracle and the regular entry point on two calls."""
    rng = np.random.default_rng(5)
    n = 3000
    wi, wj, wv = _random_triangular(n, 12, True, rng)
    zi, zj, zv = _random_triangular(n, 12, False, rng)
    f = dict(wt_irp=wi, wt_ja=wj, wt_val=wv, z_irp=zi, z_ja=zj, z_val=zv,
             d=rng.uniform(0.5, 2.0, n))
    df = device_factors(f)
    for seed, alpha, beta in [(41, 1.0, 0.0), (42, -2.0, 0.5)]:
        x = ainv.pde.rand_uniform(seed, n)
        y0 = ainv.pde.rand_uniform(seed + 9, n)
        got = _noalloc(f, x, alpha, beta, y0)
        ref = O.ainv_apply(oracle_factors(f), x, alpha, beta, y0)
        assert relerr(got, ref) <= 1e-12
        y_reg = _dev(y0, np.float64)
        df.apply(_dev(x, np.float64), y_reg, alpha, beta, "N")
        torch.cuda.synchronize()
        assert relerr(got, y_reg.cpu().numpy()) <= 1e-12


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = ainv.lib()
    dummy = torch.zeros(4, dtype=torch.float64, device=DEV)
    idx = torch.zeros(4, dtype=torch.int32, device=DEV)
    info = lib.ainv_gpu_apply_csr_noalloc(
        (1 << 20) + 1, _p(idx), _p(idx), _p(dummy), 0, _p(idx), _p(idx), _p(dummy), 0,
        _p(dummy), 1.0, _p(dummy), 0.0, _p(dummy), None)
    assert info == ainv._lib.ERR_ARG
    assert "1048576" in ainv.last_error()

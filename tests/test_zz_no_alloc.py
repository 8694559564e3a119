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
from util import build_factors, device_factors, relerr

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


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = ainv.lib()
    dummy = torch.zeros(4, dtype=torch.float64, device=DEV)
    idx = torch.zeros(4, dtype=torch.int32, device=DEV)
    info = lib.ainv_gpu_apply_csr_noalloc(
        (1 << 20) + 1, _p(idx), _p(idx), _p(dummy), 0, _p(idx), _p(idx), _p(dummy), 0,
        _p(dummy), 1.0, _p(dummy), 0.0, _p(dummy), None)
    assert info == ainv._lib.ERR_ARG
    assert "1048576" in ainv.last_error()

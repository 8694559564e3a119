"""Argument checks on the Python side of the C-ABI: every path that hands a
raw address to the library first checks dtype, contiguity and length, so a
short or single-precision buffer is rejected before any call reaches the
library (a kernel would otherwise read or write past its end).  Runs on the
CPU: the library calls are replaced by a recorder."""
import numpy as np
import pytest

import ainv
import ainv.device as D
import ainv.solver as S

torch = pytest.importorskip("torch")


class _Recorder:
    """Stand-in for the loaded library: answers n, records compute calls."""

    def __init__(self, n):
        self.n, self.calls = n, []

    def ainv_gpu_get_n(self, h):
        return self.n

    def mld_d_solver_handle(self, h):
        return 1234

    def __getattr__(self, name):
        def call(*args):
            self.calls.append(name)
            return 0
        return call


@pytest.fixture
def rec(monkeypatch):
    r = _Recorder(100)
    monkeypatch.setattr(D, "lib", lambda: r)
    monkeypatch.setattr(S, "lib", lambda: r)
    return r


def test_host_pointer_checks():
    n = 10
    assert D.hptr(np.zeros(n), n).value is not None
    assert D.hptr(np.zeros(n + 3), n).value is not None  # n_col >= n, as apply_v allows
    with pytest.raises(ValueError):
        D.hptr(np.zeros(n - 1), n)
    with pytest.raises(TypeError):
        D.hptr(np.zeros(n, np.float32), n)
    with pytest.raises(TypeError):
        D.hptr(np.zeros(2 * n)[::2], n)
    with pytest.raises(ValueError):
        D.hptr(torch.zeros(n - 1, dtype=torch.float64), n)
    with pytest.raises(TypeError):
        D.hptr([0.0] * n, n)


def test_device_pointer_checks_reject_host_buffers():
    with pytest.raises(TypeError):
        D.dptr(torch.zeros(10, dtype=torch.float64), 10)  # not on a GPU
    with pytest.raises(TypeError):
        D.dptr(np.zeros(10), 10)


def test_factors_host_apply_rejects_short_arrays(rec):
    f = D.DeviceFactors(None, None, None, _borrow=object())
    with pytest.raises(ValueError):
        f.apply_host(np.zeros(99))
    with pytest.raises(ValueError):
        f.apply_host(np.zeros(100), y=np.zeros(50))
    with pytest.raises(ValueError):
        f.apply_host(torch.zeros(100, dtype=torch.float64), y=torch.zeros(99, dtype=torch.float64))
    with pytest.raises(TypeError):
        f.apply_host(torch.zeros(100, dtype=torch.float32), y=torch.zeros(100, dtype=torch.float32))
    assert rec.calls == []
    f.apply_host(np.zeros(100))
    assert rec.calls == ["ainv_gpu_apply_host"]


def test_factors_device_calls_reject_cpu_tensors(rec):
    f = D.DeviceFactors(None, None, None, _borrow=object())
    x = torch.zeros(100, dtype=torch.float64)
    for call in (lambda: f.apply(x, x), lambda: f.apply_stage(1, x, x),
                 lambda: f.update_a(x)):
        with pytest.raises(TypeError):
            call()
    assert rec.calls == []


def test_solver_apply_a_rejects_short_arrays(rec):
    sv = S.mld_d_ainv_solver_type.__new__(S.mld_d_ainv_solver_type)
    sv._h = None
    with pytest.raises(ValueError):
        sv.apply_a(1.0, np.zeros(100), 0.0, np.zeros(99))
    with pytest.raises(ValueError):
        sv.apply_a(1.0, np.zeros(90), 0.0, np.zeros(100))
    with pytest.raises(ValueError):
        sv.apply_a(1.0, torch.zeros(100, dtype=torch.float64), 0.0,
                   torch.zeros(99, dtype=torch.float64))
    with pytest.raises(TypeError):
        sv.apply(1.0, torch.zeros(100, dtype=torch.float64), 0.0,
                 torch.zeros(100, dtype=torch.float64))
    assert rec.calls == []
    assert sv.apply_a(1.0, np.zeros(100), 0.0, np.zeros(100)) == 0
    assert rec.calls == ["mld_d_solver_apply_host"]


def test_update_a_short_x_is_an_argument_error():
    """mld_d_base_ainv_update_a.f90:54-58 returns info = -1 for size(x) <
    size(d); the solver type returns an argument error and reads nothing."""
    irp, ja, val = ainv.pde.gen_pde3d(6, "poisson")
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val) == 0
    assert sv.update_a(np.zeros(n - 1)) == ainv._lib.ERR_ARG
    assert "entries" in ainv.last_error()
    # the right length gets past the size check (no device factors here)
    assert sv.update_a(np.zeros(n)) == ainv._lib.ERR_NOT_BUILT

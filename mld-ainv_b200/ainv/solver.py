"""Python mirror of the plugin's solver types.

Names, keys and error convention follow the Fortran types
mld_d_ainv_solver_type (src/mld_d_ainv_solver.F90:46-67),
mld_d_invk_solver_type (src/mld_d_invk_solver.f90:47-57) and
mld_d_invt_solver_type (src/mld_d_invt_solver.f90:46-58): every procedure
returns `info` (0 = psb_success_) instead of raising, as the Fortran ones
set their `info` argument.  `build` runs the host factor construction;
`cnv` (or `build(..., amold=prec)`) converts the factors to the device
layout, after which `apply` (apply_v, device vectors) and `apply_a` (host
arrays) run on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PREC, SUCCESS, lib, last_error
from .device import DeviceFactors, _is_cpu_tensor, _stream, dptr, hptr


class _SolverType:
    _kind = "AINV"

    def __init__(self):
        h = C.c_void_p()
        info = lib().mld_d_solver_create(C.byref(h), self._kind.encode())
        if info != SUCCESS:
            raise RuntimeError(last_error())
        self._h = h

    # -- settings ---------------------------------------------------------
    def default(self) -> int:
        return lib().mld_d_solver_default(self._h)

    def cseti(self, what: str, val: int) -> int:
        return lib().mld_d_solver_cseti(self._h, what.encode(), int(val))

    def csetr(self, what: str, val: float) -> int:
        return lib().mld_d_solver_csetr(self._h, what.encode(), float(val))

    def csetc(self, what: str, val: str) -> int:
        return lib().mld_d_solver_csetc(self._h, what.encode(), val.encode())

    def set(self, what: str, val) -> int:
        """Generic set, dispatched on the value's type like prec%set."""
        if isinstance(val, str):
            return self.csetc(what, val)
        if isinstance(val, (int, np.integer)):
            return self.cseti(what, val)
        return self.csetr(what, val)

    def check(self) -> int:
        return lib().mld_d_solver_check(self._h)

    # -- build / convert ----------------------------------------------------
    def build(self, irp, ja, val, one_based: bool = False, amold: str | None = None) -> int:
        """Host factor construction from A (CSR).  amold: device precision
        ('FP64', 'FP32', 'BF16') to convert to once built."""
        if amold is not None:
            info = self.cnv(amold)
            if info != SUCCESS:
                return info
        irp = np.ascontiguousarray(irp, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        return lib().mld_d_solver_build(self._h, len(irp) - 1, C.c_void_p(irp.ctypes.data),
                                        C.c_void_p(ja.ctypes.data), C.c_void_p(val.ctypes.data),
                                        1 if one_based else 0)

    def cnv(self, prec: str = "FP64") -> int:
        return lib().mld_d_solver_cnv(self._h, PREC[prec.upper()])

    # -- apply --------------------------------------------------------------
    def load(self, prefix: str) -> int:
        """Factors from <prefix>_{wmat,diag,zmat}.mtx (a dump of this library
        or of the reference)."""
        return lib().mld_d_solver_load(self._h, prefix.encode())

    def save(self, path: str) -> int:
        """Binary factor cache (host factors and settings)."""
        return lib().mld_d_solver_save(self._h, path.encode())

    def restore(self, path: str) -> int:
        return lib().mld_d_solver_restore(self._h, path.encode())

    def update_a(self, x) -> int:
        """update(x) of the plugin type (shifted system A + diag(x)) on the
        uploaded factors; the host d follows.  Like the reference, x shorter
        than the factors' n is an argument error (info != 0)."""
        x = np.ascontiguousarray(x, np.float64)
        return lib().mld_d_solver_update_a(self._h, C.c_void_p(x.ctypes.data), x.size)

    def _n(self) -> int | None:
        """Rows of the factors: the device copy's, else the host build's,
        else None (nothing built)."""
        h = lib().mld_d_solver_handle(self._h)
        if h:
            return lib().ainv_gpu_get_n(C.c_void_p(h))
        n = C.c_int(0)
        if lib().mld_d_solver_get_factors(self._h, C.byref(n), None, None,
                                          *([None] * 7)) == SUCCESS:
            return n.value
        return None

    def apply(self, alpha, x, beta, y, trans: str = "N", stream=None) -> int:
        """apply_v: y = alpha * M x + beta * y on device tensors (float64,
        contiguous, at least n entries each)."""
        n = self._n() or 0
        return lib().mld_d_solver_apply(self._h, float(alpha), dptr(x, n, "x"), float(beta),
                                        dptr(y, n, "y"), trans.encode()[:1], _stream(stream))

    def apply_a(self, alpha, x, beta, y, trans: str = "N") -> int:
        """apply_a: host arrays; y (float64, contiguous) is updated in place.
        x and y are numpy arrays or CPU torch tensors of at least n entries;
        with page-locked tensors (``tensor.pin_memory()``) the transfers
        overlap the sweeps."""
        if _is_cpu_tensor(y):
            if not _is_cpu_tensor(x):
                raise TypeError("x must be a CPU tensor when y is one")
        elif isinstance(y, np.ndarray):
            x = np.ascontiguousarray(x, np.float64)
        else:
            raise TypeError("y must be a numpy array or a CPU tensor")
        n = self._n() or 0
        return lib().mld_d_solver_apply_host(self._h, float(alpha), hptr(x, n, "x"), float(beta),
                                             hptr(y, n, "y"), trans.encode()[:1])

    @property
    def device(self) -> DeviceFactors | None:
        h = lib().mld_d_solver_handle(self._h)
        return DeviceFactors(None, None, None, _borrow=C.c_void_p(h)) if h else None

    # -- inspection -----------------------------------------------------------
    def factors(self) -> dict:
        n, nw, nz = C.c_int(), C.c_longlong(), C.c_longlong()
        info = lib().mld_d_solver_get_factors(self._h, C.byref(n), C.byref(nw), C.byref(nz),
                                              *([None] * 7))
        if info != SUCCESS:
            raise RuntimeError(last_error())
        n, nw, nz = n.value, nw.value, nz.value
        out = dict(wt_irp=np.empty(n + 1, np.int32), wt_ja=np.empty(nw, np.int32),
                   wt_val=np.empty(nw), z_irp=np.empty(n + 1, np.int32),
                   z_ja=np.empty(nz, np.int32), z_val=np.empty(nz), d=np.empty(n))
        keys = ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]
        lib().mld_d_solver_get_factors(self._h, None, None, None,
                                       *[C.c_void_p(out[k].ctypes.data) for k in keys])
        return out

    def clone(self):
        h = C.c_void_p()
        info = lib().mld_d_solver_clone(self._h, C.byref(h))
        if info != SUCCESS:
            raise RuntimeError(last_error())
        obj = self.__class__.__new__(self.__class__)
        obj._h = h
        return obj

    def clone_settings(self, other: "_SolverType") -> int:
        return lib().mld_d_solver_clone_settings(self._h, other._h)

    def free(self) -> int:
        return lib().mld_d_solver_free(self._h)

    def sizeof(self) -> int:
        return int(lib().mld_d_solver_sizeof(self._h))

    def get_nzeros(self) -> int:
        return int(lib().mld_d_solver_get_nzeros(self._h))

    @staticmethod
    def get_wrksz() -> int:
        return lib().mld_d_solver_get_wrksz()

    def descr(self) -> str:
        buf = C.create_string_buffer(1024)
        lib().mld_d_solver_descr(self._h, buf, len(buf))
        return buf.value.decode()

    def dump(self, prefix: str) -> int:
        return lib().mld_d_solver_dump(self._h, prefix.encode())

    def __del__(self):
        try:
            if self._h:
                lib().mld_d_solver_destroy(self._h)
            self._h = None
        except Exception:
            pass


class mld_d_ainv_solver_type(_SolverType):  # noqa: N801 (reference name)
    _kind = "AINV"


class mld_d_invk_solver_type(_SolverType):  # noqa: N801
    _kind = "INVK"


class mld_d_invt_solver_type(_SolverType):  # noqa: N801
    _kind = "INVT"

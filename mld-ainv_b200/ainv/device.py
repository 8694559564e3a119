"""Device objects: the converted factors (W^T, Z, D^-1) and the operator A.

Vectors passed to the device entry points are CUDA tensors (torch is used
only as the owner of device memory and streams); host entry points take
numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import KRYLOV, PREC, SUCCESS, check, lib, last_error


def _np(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def dptr(t, n: int, name: str = "vector") -> C.c_void_p:
    """Device address of `t` once it is known to be a contiguous float64
    CUDA tensor of at least n entries.  The kernels read or write n entries
    through the raw address, so a strided or single-precision tensor
    (TypeError) or a short one (ValueError) is rejected here, before any
    call reaches the library."""
    if not (_is_tensor(t) and t.is_cuda):
        raise TypeError(f"{name}: expected a CUDA tensor")
    if t.dtype != _torch().float64 or not t.is_contiguous():
        raise TypeError(f"{name}: expected a contiguous float64 tensor")
    if t.numel() < n:
        raise ValueError(f"{name}: {t.numel()} entries, {n} needed")
    return C.c_void_p(t.data_ptr())


def hptr(a, n: int, name: str = "array") -> C.c_void_p:
    """Host address of a numpy array or CPU tensor once it is known to be
    contiguous float64 with at least n entries (the library reads or writes
    n entries through it, from the CPU or from a kernel over PCIe)."""
    if _is_cpu_tensor(a):
        if a.dtype != _torch().float64 or not a.is_contiguous():
            raise TypeError(f"{name}: expected a contiguous float64 tensor")
        size, addr = a.numel(), a.data_ptr()
    elif isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError(f"{name}: expected a contiguous float64 array")
        size, addr = a.size, a.ctypes.data
    else:
        raise TypeError(f"{name}: expected a numpy array or a CPU tensor, got {type(a)}")
    if size < n:
        raise ValueError(f"{name}: {size} entries, {n} needed")
    return C.c_void_p(addr)


def _stream(s):
    if s is None:
        return None
    return C.c_void_p(getattr(s, "cuda_stream", s))


def _torch():
    import torch
    return torch


def _is_tensor(a) -> bool:
    t = type(a)
    return t.__module__.startswith("torch") and t.__name__ in ("Tensor", "Parameter")


def _is_cpu_tensor(a) -> bool:
    return _is_tensor(a) and a.device.type == "cpu"


class DeviceFactors:
    """W^T (lower CSR), Z (upper CSR) and D^-1 uploaded to the device layout."""

    def __init__(self, wt, z, d, prec: str = "FP64", one_based: bool = False, *, _borrow=None):
        self._own = _borrow is None
        if _borrow is not None:
            self._h = _borrow
            return
        self._keep = [_np(wt[0], np.int32), _np(wt[1], np.int32), _np(wt[2], np.float64),
                      _np(z[0], np.int32), _np(z[1], np.int32), _np(z[2], np.float64),
                      _np(d, np.float64)]
        n = len(self._keep[6])
        h = C.c_void_p()
        check(lib().ainv_gpu_create(C.byref(h), n, *[C.c_void_p(a.ctypes.data) for a in self._keep],
                                    PREC[prec.upper()], 1 if one_based else 0))
        self._h = h
        del self._keep

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def n(self) -> int:
        return lib().ainv_gpu_get_n(self._h)

    @property
    def prec(self) -> str:
        p = lib().ainv_gpu_get_prec(self._h)
        return {v: k for k, v in PREC.items()}[p]

    def apply(self, x, y, alpha=1.0, beta=0.0, trans="N", stream=None) -> None:
        """y = alpha * Z D^-1 W^T x + beta * y (trans 'N'), device tensors."""
        n = self.n
        check(lib().ainv_gpu_apply(self._h, trans.encode()[:1], alpha, dptr(x, n, "x"), beta,
                                   dptr(y, n, "y"), _stream(stream)))

    def apply_stage(self, stage, x=None, y=None, alpha=1.0, beta=0.0, trans="N", stream=None):
        """Run sweep 1 (t = D^-1 W^T x) or sweep 2 (y = alpha Z t + beta y) alone."""
        n = self.n
        check(lib().ainv_gpu_apply_stage(self._h, trans.encode()[:1], int(stage), alpha,
                                         dptr(x, n, "x") if x is not None else None, beta,
                                         dptr(y, n, "y") if y is not None else None,
                                         _stream(stream)))

    def update_a(self, x, d_out=None, stream=None) -> None:
        """update_a on the device: d <- 1/(1/d + diag(W^T diag(x) Z)); x a
        CUDA float64 tensor of n entries, d_out (optional) receives the new d
        in FP64."""
        n = self.n
        check(lib().ainv_gpu_update_a(self._h, dptr(x, n, "x"),
                                      dptr(d_out, n, "d_out") if d_out is not None else None,
                                      _stream(stream)))

    def apply_host(self, x, alpha=1.0, beta=0.0, y=None, trans="N"):
        """y = alpha*op(M) x + beta*y on host arrays (the array form of the
        apply).  x and y are numpy arrays (a new y is returned) or contiguous
        float64 CPU torch tensors (y written in place and returned).  With
        page-locked tensors (``tensor.pin_memory()``) the copies overlap the
        sweeps chunk by chunk."""
        n = self.n
        if _is_cpu_tensor(x):
            if y is None or not _is_cpu_tensor(y):
                raise ValueError("apply_host: y must be a CPU tensor when x is one")
            check(lib().ainv_gpu_apply_host(self._h, trans.encode()[:1], alpha,
                                            hptr(x, n, "x"), beta, hptr(y, n, "y")))
            return y
        x = _np(x, np.float64)
        y = np.zeros_like(x) if y is None else _np(y, np.float64).copy()
        check(lib().ainv_gpu_apply_host(self._h, trans.encode()[:1], alpha, hptr(x, n, "x"), beta,
                                        hptr(y, n, "y")))
        return y

    def check(self) -> None:
        """Raise if a device-side wait of a kernel on these factors timed out."""
        check(lib().ainv_gpu_check(self._h))

    def sizeof(self) -> int:
        return int(lib().ainv_gpu_sizeof(self._h))

    def get_nzeros(self) -> int:
        return int(lib().ainv_gpu_get_nzeros(self._h))

    def layout_info(self, which: str = "wt") -> dict:
        """Device layout of one operand: 'wt', 'z' (trans 'N'), 'zt', 'w' (trans 'T')."""
        w = {"wt": 0, "z": 1, "zt": 2, "w": 3}[which]
        ll = [C.c_longlong() for _ in range(3)]
        ii = [C.c_int() for _ in range(2)]
        check(lib().ainv_gpu_layout_info(self._h, w, *[C.byref(x) for x in ll + ii]))
        return dict(nnz=ll[0].value, slots=ll[1].value, nidx=ll[2].value, nslices=ii[0].value,
                    offset_slices=ii[1].value)

    def close(self) -> None:
        if getattr(self, "_own", False) and self._h:
            lib().ainv_gpu_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolveResult:
    def __init__(self, info, iters, err, verify_fails=0, replacements=0):
        self.info, self.iter, self.err = info, iters, err
        self.verify_fails, self.replacements = verify_fails, replacements

    @property
    def converged(self) -> bool:
        return self.info == SUCCESS

    def __repr__(self):
        return (f"SolveResult(info={self.info}, iter={self.iter}, err={self.err:.3e}, "
                f"verify_fails={self.verify_fails}, replacements={self.replacements})")


class BlockSolveResult:
    def __init__(self, info, iters, errs, status):
        self.info, self.iters, self.errs, self.status = info, iters, errs, status

    @property
    def converged(self) -> bool:
        return self.info == SUCCESS and all(s == SUCCESS for s in self.status)

    def __repr__(self):
        return (f"BlockSolveResult(info={self.info}, iters={self.iters}, "
                f"max_err={max(self.errs):.3e})")


class DeviceOperator:
    """Sparse operator A (FP64) on the device, with the Krylov driver."""

    def __init__(self, irp, ja, val, one_based: bool = False):
        irp, ja, val = _np(irp, np.int32), _np(ja, np.int32), _np(val, np.float64)
        self.n = len(irp) - 1
        h = C.c_void_p()
        check(lib().ainv_csr_create(C.byref(h), self.n, C.c_void_p(irp.ctypes.data),
                                    C.c_void_p(ja.ctypes.data), C.c_void_p(val.ctypes.data),
                                    1 if one_based else 0))
        self._h = h

    @property
    def handle(self):
        return self._h

    def check(self) -> None:
        """Raise if a device-side wait of a kernel on A timed out."""
        check(lib().ainv_csr_check(self._h))

    def spmv(self, x, y, alpha=1.0, beta=0.0, stream=None) -> None:
        check(lib().ainv_csr_spmv(self._h, alpha, dptr(x, self.n, "x"), beta,
                                  dptr(y, self.n, "y"), _stream(stream)))

    def solve(self, b, x, factors: DeviceFactors | None = None, method="BICGSTAB", eps=1e-9,
              itmax=1000, stream=None) -> SolveResult:
        """psb_krylov(method, A, prec, b, x, eps, ..., istop=2) on the device.
        Returns the status instead of raising for NOCONV / breakdown."""
        it, err = C.c_int(0), C.c_double(0.0)
        info = lib().ainv_gpu_solve(factors.handle if factors is not None else None, self._h,
                                    dptr(b, self.n, "b"), dptr(x, self.n, "x"),
                                    KRYLOV[method.upper()], eps, itmax,
                                    C.byref(it), C.byref(err), _stream(stream))
        if info not in (SUCCESS, 4102, 4103, 4104):
            check(info)
        vf, rp = C.c_int(0), C.c_int(0)
        lib().ainv_csr_solve_info(self._h, C.byref(vf), C.byref(rp))
        return SolveResult(info, it.value, err.value, vf.value, rp.value)

    def history(self) -> np.ndarray:
        """||r_k||/||b|| after each iteration of the last solve on this
        operator (the first 8192 iterations)."""
        cnt = C.c_int(0)
        check(lib().ainv_csr_solve_history(self._h, None, 0, C.byref(cnt)))
        out = np.zeros(cnt.value)
        if cnt.value:
            check(lib().ainv_csr_solve_history(self._h, C.c_void_p(out.ctypes.data), cnt.value,
                                               C.byref(cnt)))
        return out

    def block_solve(self, B, X, factors: DeviceFactors | None = None, eps=1e-9, itmax=1000,
                    stream=None) -> "BlockSolveResult":
        """CG on the m columns of B (a CUDA float64 tensor of shape (n, m),
        m <= 32, row-major): one SpMM per product for all columns, each column
        with its own recurrence.  X (same shape) holds x0 and receives the
        solutions.  Statuses are returned per column instead of raised."""
        if B.dim() != 2 or B.shape != X.shape or B.shape[0] != self.n:
            raise ValueError("B and X must both have shape (n, m)")
        if factors is not None and factors.n != self.n:
            raise ValueError("block_solve: preconditioner and operator sizes differ")
        m = B.shape[1]
        it = (C.c_int * m)()
        err = (C.c_double * m)()
        st = (C.c_int * m)()
        info = lib().ainv_gpu_block_solve(factors.handle if factors is not None else None,
                                          self._h, m, dptr(B, self.n * m, "B"), m,
                                          dptr(X, self.n * m, "X"), m, eps, itmax, it,
                                          err, st, _stream(stream))
        if info not in (SUCCESS, 4102, 4103, 4104):
            check(info)
        return BlockSolveResult(info, list(it), list(err), list(st))

    def close(self) -> None:
        if self._h:
            lib().ainv_csr_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

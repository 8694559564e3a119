"""Solve server: continuous batching of BiCGSTAB solves on resident operators.

Mirror of the ainv_server_* C-ABI (include/ainv_b200.h).  Requests are
queued with `submit` (host right-hand side, host solution buffer) and
collected with `wait`; the native engine thread admits them first-come
first-served as slots and device memory free up, advances all admitted
requests together through one captured CUDA graph per step, and writes each
solution back as soon as it has converged.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import Result, ServerInfo, check, lib
from .device import DeviceFactors, DeviceOperator, hptr


@dataclass
class Completed:
    id: int
    op: int
    status: int
    iter: int
    err: float
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit

    @property
    def converged(self) -> bool:
        return self.status == 0


def request_bytes(n: int) -> int:
    """Device bytes a request of n rows holds while admitted."""
    return int(lib().ainv_server_request_bytes(n))


def plan(rows, grid: int):
    """Block plan for requests of the given row counts: (b0, nb) arrays."""
    rows = np.ascontiguousarray(rows, np.int32)
    b0 = np.zeros(len(rows), np.int32)
    nb = np.zeros(len(rows), np.int32)
    check(lib().ainv_server_plan(len(rows), C.c_void_p(rows.ctypes.data), grid,
                                 C.c_void_p(b0.ctypes.data), C.c_void_p(nb.ctypes.data)))
    return b0, nb


class SolveServer:
    def __init__(self, max_slots: int = 16, hbm_bytes: int = 0, iters_per_launch: int = 4):
        h = C.c_void_p()
        check(lib().ainv_server_create(C.byref(h), max_slots, hbm_bytes, iters_per_launch))
        self._h = h
        self._keep = []       # operators / factors referenced by the server
        self._buffers = {}    # id -> (b, x) kept alive until wait
        self._rows = {}       # operator -> rows (length of its b and x)

    def add_operator(self, a: DeviceOperator, f: DeviceFactors) -> int:
        op = C.c_int(0)
        check(lib().ainv_server_add_operator(self._h, a.handle, f.handle, C.byref(op)))
        self._keep.append((a, f))
        self._rows[op.value] = a.n
        return op.value

    def submit(self, op: int, b, x, eps: float = 1e-8, itmax: int = 1000) -> int:
        """Queue A_op x = b.  b and x are host float64 buffers (numpy arrays
        or pinned torch tensors) kept alive here until `wait`."""
        rid = C.c_longlong(0)
        n = self._rows.get(op, 0)  # an unknown operator is the library's argument error
        check(lib().ainv_server_submit(self._h, op, hptr(b, n, "b"), hptr(x, n, "x"), eps,
                                       itmax, C.byref(rid)))
        self._buffers[rid.value] = (b, x)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> Completed:
        """The request's outcome; its status (NOCONV, breakdown, ...) is in
        the result, while an unknown id or a timeout raises."""
        r = Result()
        info = lib().ainv_server_wait(self._h, rid, timeout, C.byref(r))
        if info in (30, 4106):  # unknown id, or still running: a call error
            check(info)
        self._buffers.pop(rid, None)
        return Completed(r.id, r.op, r.status, r.iter, r.err, r.t_submit, r.t_admit, r.t_done)

    def stats(self) -> dict:
        s = ServerInfo()
        lib().ainv_server_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in ServerInfo._fields_}

    def close(self) -> None:
        if self._h:
            lib().ainv_server_destroy(self._h)
        self._h = None
        self._buffers.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



"""ctypes front end for the CPU oracle (libainv_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or the timed CPU reference --
never by the product.  Parity with the Fortran reference is UNPINNED (the
reference cannot be built here); see ainv_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libainv_oracle.so")
_lib = None

ALG = {"LLK": 0, "SYM-LLK": 1, "LLK-NOTH": 2, "STAB-LLK": 3, "MLK": 4}

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_gen_pde3d.restype = C.c_long
        L.orc_gen_pde3d.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, _i32p, _i32p, _f64p]
        L.orc_rand_uniform.argtypes = [C.c_uint64, C.c_long, C.c_double,
                                       C.c_double, _f64p]
        L.orc_rand_normal.argtypes = [C.c_uint64, C.c_long, _f64p]
        L.orc_ainv_build.restype = C.c_int
        L.orc_ainv_build.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p,
                                     C.c_int, C.c_double,
                                     _i32p, _i32p, _f64p, C.POINTER(C.c_long),
                                     _i32p, _i32p, _f64p, C.POINTER(C.c_long),
                                     _f64p]
        L.orc_csr_spmv.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double,
                                   _f64p, C.c_double, _f64p]
        L.orc_csr_spmv_t.argtypes = L.orc_csr_spmv.argtypes
        L.orc_ainv_apply.restype = C.c_int
        L.orc_ainv_apply.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p,
                                     _i32p, _f64p, _f64p, C.c_char, C.c_double,
                                     _f64p, C.c_double, _f64p, _f64p]
        kry = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i32p, _i32p,
               _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_int,
               C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_cg.restype = C.c_int
        L.orc_cg.argtypes = kry
        L.orc_bicgstab.restype = C.c_int
        L.orc_bicgstab.argtypes = kry
        pp_i = C.POINTER(C.POINTER(C.c_int))
        pp_d = C.POINTER(C.POINTER(C.c_double))
        outs = [pp_i, pp_i, pp_d, C.POINTER(C.c_long),
                pp_i, pp_i, pp_d, C.POINTER(C.c_long), _f64p]
        L.orc_invk_build.restype = C.c_int
        L.orc_invk_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int,
                                     C.c_int] + outs
        L.orc_invt_build.restype = C.c_int
        L.orc_invt_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int,
                                     C.c_double, C.c_int, C.c_double] + outs
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_update_a.restype = C.c_int
        L.orc_update_a.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p,
                                   _f64p, _f64p, _f64p]
        L.orc_set_dot_order.argtypes = [C.c_int]
        L.orc_dot_device_order.restype = C.c_double
        L.orc_dot_device_order.argtypes = [C.c_int, _f64p, _f64p]
        L.orc_set_history.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _lib = L
    return _lib


@dataclass
class CSR:
    n: int
    irp: np.ndarray
    ja: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.irp[-1])


@dataclass
class Factors:
    wt: CSR
    z: CSR
    d: np.ndarray


def gen_pde3d(idim: int, kind: str = "poisson", beta=(0.0, 0.0, 0.0)) -> CSR:
    """kind 'poisson' (6/-1) or 'convdiff' (upwind, h = 1/(idim+1))."""
    n = idim ** 3
    irp = np.zeros(n + 1, np.int32)
    ja = np.zeros(7 * n, np.int32)
    val = np.zeros(7 * n, np.float64)
    k = 0 if kind == "poisson" else 1
    nnz = lib().orc_gen_pde3d(idim, k, float(beta[0]), float(beta[1]),
                              float(beta[2]), irp, ja, val)
    return CSR(n, irp, ja[:nnz].copy(), val[:nnz].copy())


def rand_uniform(seed: int, n: int, lo=-1.0, hi=1.0) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_rand_uniform(seed, n, lo, hi, out)
    return out


def rand_normal(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_rand_normal(seed, n, out)
    return out


def ainv_build(a: CSR, alg: str = "LLK", fill_in: int = 20,
               thresh: float = 0.1) -> Factors:
    n = a.n
    cap = n * fill_in
    wi = np.zeros(n + 1, np.int32); wj = np.zeros(cap, np.int32)
    wv = np.zeros(cap, np.float64)
    zi = np.zeros(n + 1, np.int32); zj = np.zeros(cap, np.int32)
    zv = np.zeros(cap, np.float64)
    d = np.zeros(n, np.float64)
    nw = C.c_long(0); nz = C.c_long(0)
    rc = lib().orc_ainv_build(ALG[alg], n, a.irp, a.ja, a.val, fill_in,
                              float(thresh), wi, wj, wv, C.byref(nw), zi, zj,
                              zv, C.byref(nz), d)
    if rc != 0:
        raise RuntimeError(f"orc_ainv_build failed: {rc}")
    return Factors(CSR(n, wi, wj[:nw.value].copy(), wv[:nw.value].copy()),
                   CSR(n, zi, zj[:nz.value].copy(), zv[:nz.value].copy()), d)


def _owned_factors(n, call) -> Factors:
    """Run an oracle builder that allocates its factor arrays; copy and free."""
    ptrs = [C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)(),
            C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()]
    nw, nz = C.c_long(), C.c_long()
    d = np.zeros(n, np.float64)
    rc = call(C.byref(ptrs[0]), C.byref(ptrs[1]), C.byref(ptrs[2]), C.byref(nw),
              C.byref(ptrs[3]), C.byref(ptrs[4]), C.byref(ptrs[5]), C.byref(nz), d)
    try:
        if rc != 0:
            raise RuntimeError(f"oracle factor build failed: {rc}")
        sizes = [n + 1, nw.value, nw.value, n + 1, nz.value, nz.value]
        arrs = [np.ctypeslib.as_array(p, shape=(k,)).copy() if k else
                np.zeros(0, np.int32 if i % 3 < 2 else np.float64)
                for i, (p, k) in enumerate(zip(ptrs, sizes))]
    finally:
        for p in ptrs:
            if p:
                lib().orc_free(C.cast(p, C.c_void_p))
    return Factors(CSR(n, *arrs[:3]), CSR(n, *arrs[3:]), d)


def invk_build(a: CSR, fill1: int = 1, fill2: int = 1) -> Factors:
    """INVK factors: ILU(fill1), then level-fill2 sparse inverses."""
    return _owned_factors(a.n, lambda *o: lib().orc_invk_build(
        a.n, a.irp, a.ja, a.val, fill1, fill2, *o))


def invt_build(a: CSR, fillin: int = 20, thresh: float = 0.05,
               invfill: int = 20, invthresh: float = 0.05) -> Factors:
    """INVT factors: ILUT(fillin, thresh), then (invfill, invthresh) inverses."""
    return _owned_factors(a.n, lambda *o: lib().orc_invt_build(
        a.n, a.irp, a.ja, a.val, fillin, float(thresh), invfill,
        float(invthresh), *o))


def update_a(f: Factors, x) -> np.ndarray:
    """New d after update_a(x): 1 / (1/d + diag(W^T diag(x) Z))."""
    n = f.d.shape[0]
    out = np.empty(n)
    rc = lib().orc_update_a(n, f.wt.irp, f.wt.ja, f.wt.val, f.z.irp, f.z.ja, f.z.val,
                            np.ascontiguousarray(f.d, np.float64),
                            np.ascontiguousarray(x, np.float64), out)
    if rc != 0:
        raise RuntimeError(f"orc_update_a failed: {rc}")
    return out


def spmv(a: CSR, x, alpha=1.0, beta=0.0, y=None, trans="N") -> np.ndarray:
    y = np.zeros(a.n) if y is None else np.ascontiguousarray(y, np.float64).copy()
    x = np.ascontiguousarray(x, np.float64)
    f = lib().orc_csr_spmv if trans == "N" else lib().orc_csr_spmv_t
    f(a.n, a.irp, a.ja, a.val, alpha, x, beta, y)
    return y


def ainv_apply(f: Factors, x, alpha=1.0, beta=0.0, y=None, trans="N") -> np.ndarray:
    n = f.d.shape[0]
    y = np.zeros(n) if y is None else np.ascontiguousarray(y, np.float64).copy()
    x = np.ascontiguousarray(x, np.float64)
    work = np.zeros(n)
    rc = lib().orc_ainv_apply(n, f.wt.irp, f.wt.ja, f.wt.val, f.z.irp, f.z.ja,
                              f.z.val, f.d, trans.encode(), alpha, x, beta, y,
                              work)
    if rc != 0:
        raise ValueError(f"invalid trans {trans!r}")
    return y


DOT_ORDERS = {"device": 0, "sequential": 1}


def solve(method: str, a: CSR, f: Factors, b, x0=None, eps=1e-9, itmax=1000,
          order: str = "device", history: bool = False):
    """Returns (x, iterations, relative residual, status), plus the
    per-iteration ||r_k||/||b|| when history is set.  order: the summation
    order of the dots, "device" (the device library's canonical order) or
    "sequential" (reference BLAS ddot)."""
    x = np.zeros(a.n) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
    b = np.ascontiguousarray(b, np.float64)
    it = C.c_int(0); err = C.c_double(0.0)
    fn = lib().orc_cg if method.upper() == "CG" else lib().orc_bicgstab
    hist = np.zeros(max(itmax, 1)) if history else None
    L = lib()
    L.orc_set_dot_order(DOT_ORDERS[order])
    L.orc_set_history(hist.ctypes.data if history else None, len(hist) if history else 0)
    try:
        rc = fn(a.n, a.irp, a.ja, a.val, f.wt.irp, f.wt.ja, f.wt.val, f.z.irp,
                f.z.ja, f.z.val, f.d, b, x, eps, itmax, C.byref(it), C.byref(err))
    finally:
        L.orc_set_history(None, 0)
        L.orc_set_dot_order(0)
    if history:
        return x, it.value, err.value, rc, hist[:it.value].copy()
    return x, it.value, err.value, rc


def dot_device_order(a, b) -> float:
    """The device library's canonical-order dot of two float64 vectors."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return lib().orc_dot_device_order(len(a), a, b)


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def get_threads() -> int:
    return lib().orc_get_threads()

"""INVK / INVT host builders (product C++ through the C-ABI) on the CPU.

The product restates MLD2P4's ILU(k) / ILUT and the plugin's sparse
inverses (src/impl/mld_d_invk_bld.f90, src/impl/mld_d_invt_bld.f90,
src/impl/mld_dsparse_invk.f90, src/impl/mld_dsparse_invt.f90 and their
copyin / inv / copyout routines).  It must agree bit for bit with the C
oracle's independent restatement; the known-answer tests pin the
mathematics (exact factorisation + exact inverse = A^-1, level-of-fill
patterns, caps).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import ainv
import oracle as O


def _build(kind, a_irp, a_ja, a_val, **kw):
    sv = ainv.mld_d_invk_solver_type() if kind == "INVK" else ainv.mld_d_invt_solver_type()
    for k, v in kw.items():
        (sv.csetr if isinstance(v, float) else sv.cseti)(k, v)
    rc = sv.build(a_irp, a_ja, a_val)
    return sv, rc


def _mat(f, pre, n):
    return sp.csr_matrix((f[pre + "_val"], f[pre + "_ja"], f[pre + "_irp"]), shape=(n, n))


def _same(f, of):
    pairs = [("wt_irp", of.wt.irp), ("wt_ja", of.wt.ja), ("wt_val", of.wt.val),
             ("z_irp", of.z.irp), ("z_ja", of.z.ja), ("z_val", of.z.val), ("d", of.d)]
    for k, v in pairs:
        np.testing.assert_array_equal(f[k], v, err_msg=k)


CASES = [
    (14, "convdiff", (10 / np.sqrt(3),) * 3),
    (11, "convdiff", (80.0, -30.0, 15.0)),
    (12, "poisson", (0.0, 0.0, 0.0)),
]


@pytest.mark.parametrize("idim,kind,beta", CASES)
@pytest.mark.parametrize("fill1,fill2", [(1, 1), (0, 2), (2, 0)])
def test_invk_matches_oracle(idim, kind, beta, fill1, fill2):
    irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
    sv, rc = _build("INVK", irp, ja, val, SUB_FILLIN=fill1, INV_FILLIN=fill2)
    assert rc == 0
    _same(sv.factors(), O.invk_build(O.CSR(len(irp) - 1, irp, ja, val), fill1, fill2))


@pytest.mark.parametrize("idim,kind,beta", CASES)
@pytest.mark.parametrize("p", [(20, 0.05, 20, 0.05), (2, 0.01, 1, 0.02), (0, 0.001, 4, 0.0)])
def test_invt_matches_oracle(idim, kind, beta, p):
    irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
    sv, rc = _build("INVT", irp, ja, val, SUB_FILLIN=p[0], SUB_ILUTHRS=float(p[1]),
                    INV_FILLIN=p[2], INV_THRESH=float(p[3]))
    assert rc == 0
    _same(sv.factors(), O.invt_build(O.CSR(len(irp) - 1, irp, ja, val), *p))


@pytest.mark.parametrize("solver", ["INVK", "INVT"])
@pytest.mark.parametrize("kind,beta", [("poisson", (0, 0, 0)), ("convdiff", (25.0, -5.0, 12.0))])
def test_exact_limits_invert_a(solver, kind, beta):
    """No dropping: exact LDU and exact triangular inverses, Z D W^T = A^-1."""
    irp, ja, val = ainv.pde.gen_pde3d(4, kind, beta)
    n = len(irp) - 1
    if solver == "INVK":
        sv, rc = _build(solver, irp, ja, val, SUB_FILLIN=n, INV_FILLIN=n)
    else:
        sv, rc = _build(solver, irp, ja, val, SUB_FILLIN=n, SUB_ILUTHRS=0.0,
                        INV_FILLIN=n, INV_THRESH=0.0)
    assert rc == 0
    f = sv.factors()
    M = (_mat(f, "z", n) @ sp.diags(f["d"]) @ _mat(f, "wt", n)).toarray()
    A = sp.csr_matrix((val, ja, irp), shape=(n, n)).toarray()
    assert np.abs(M @ A - np.eye(n)).max() < 1e-12


def test_tridiagonal_ilu0_is_exact():
    """ILU(0) of a tridiagonal matrix is its exact LU; the unbounded-level
    inverses of the bidiagonal factors are then exact as well."""
    n = 12
    rows = []
    for i in range(n):
        e = [(i - 1, -1.0 - 0.1 * i)] if i > 0 else []
        e.append((i, 4.0 + 0.5 * i))
        if i < n - 1:
            e.append((i + 1, -2.0 + 0.05 * i))
        rows.append(e)
    irp = np.cumsum([0] + [len(e) for e in rows]).astype(np.int32)
    ja = np.array([c for e in rows for c, _ in e], np.int32)
    val = np.array([v for e in rows for _, v in e])
    sv, rc = _build("INVK", irp, ja, val, SUB_FILLIN=0, INV_FILLIN=n)
    assert rc == 0
    f = sv.factors()
    M = (_mat(f, "z", n) @ sp.diags(f["d"]) @ _mat(f, "wt", n)).toarray()
    A = sp.csr_matrix((val, ja, irp), shape=(n, n)).toarray()
    np.testing.assert_allclose(M, np.linalg.inv(A), rtol=1e-12, atol=1e-14)
    # the inverse of a bidiagonal factor is dense upper: level j - i - 1
    for fill2 in range(4):
        sv, _ = _build("INVK", irp, ja, val, SUB_FILLIN=0, INV_FILLIN=fill2)
        Z = _mat(sv.factors(), "z", n).toarray()
        for i in range(n - 1):
            cols = np.nonzero(Z[i])[0]
            assert list(cols) == list(range(i, min(n, i + fill2 + 2)))


def test_invk_level0_keeps_factor_pattern():
    """INVK(0, 0): the inverse keeps the pattern of U (level 0) plus the
    diagonal, so Z's pattern is the upper triangle of A's pattern."""
    irp, ja, val = ainv.pde.gen_pde3d(6, "convdiff", (7.0, -3.0, 2.0))
    n = len(irp) - 1
    sv, rc = _build("INVK", irp, ja, val, SUB_FILLIN=0, INV_FILLIN=0)
    assert rc == 0
    f = sv.factors()
    A = sp.csr_matrix((val, ja, irp), shape=(n, n))
    Zp = (_mat(f, "z", n) != 0).astype(int)
    Up = (sp.triu(A) != 0).astype(int)
    assert (Zp != Up).nnz == 0
    Wp = (_mat(f, "wt", n) != 0).astype(int)
    assert (Wp != (sp.tril(A) != 0).astype(int)).nnz == 0
    assert np.all(_mat(f, "z", n).diagonal() == 1.0)
    assert np.all(_mat(f, "wt", n).diagonal() == 1.0)


def test_invt_row_caps():
    """Each row of Z keeps at most nnz(U row) + inv_fill entries (diagonal
    included), checked against the oracle's ILUT U (same restatement)."""
    irp, ja, val = ainv.pde.gen_pde3d(9, "convdiff", (40.0, 10.0, -20.0))
    sv, rc = _build("INVT", irp, ja, val, SUB_FILLIN=2, SUB_ILUTHRS=0.01,
                    INV_FILLIN=1, INV_THRESH=0.0)
    assert rc == 0
    f = sv.factors()
    zl = np.diff(f["z_irp"])
    assert zl[-1] == 1 and f["z_val"][-1] == 1.0
    # with INV_THRESH = 0 and a fill cap of 1, rows are short
    assert zl.max() <= 2 + 2 + 3 + 1
    assert np.all(f["z_ja"][f["z_irp"][:-1]] >= np.arange(len(irp) - 1))


def test_build_is_independent_of_thread_count():
    irp, ja, val = ainv.pde.gen_pde3d(24, "convdiff", (10.0, 10.0, 10.0))  # n = 13824
    out = []
    old = os.environ.get("AINV_BUILD_THREADS")
    try:
        for t in ("1", "5"):
            os.environ["AINV_BUILD_THREADS"] = t
            sv, rc = _build("INVT", irp, ja, val, SUB_FILLIN=20, SUB_ILUTHRS=0.05,
                            INV_FILLIN=20, INV_THRESH=0.05)
            assert rc == 0
            out.append(sv.factors())
    finally:
        if old is None:
            os.environ.pop("AINV_BUILD_THREADS", None)
        else:
            os.environ["AINV_BUILD_THREADS"] = old
    for k in out[0]:
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)


def test_zero_pivot_is_reported():
    """A structurally zero diagonal gives a zero ILU pivot: breakdown."""
    irp = np.array([0, 2, 4, 6], np.int32)
    ja = np.array([1, 2, 0, 2, 0, 1], np.int32)
    val = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    for solver in ("INVK", "INVT"):
        sv, rc = _build(solver, irp, ja, val)
        assert rc == ainv._lib.ERR_BREAKDOWN
        assert "pivot" in ainv.last_error()


def test_negative_levels_rejected_and_check_resets():
    irp, ja, val = ainv.pde.gen_pde3d(4, "poisson")
    sv, rc = _build("INVK", irp, ja, val, SUB_FILLIN=-1)
    assert rc == ainv._lib.ERR_ARG
    assert sv.check() == 0               # mld_check_def: back to the default 0
    assert sv.build(irp, ja, val) == 0
    t, rc = _build("INVT", irp, ja, val, INV_THRESH=-0.5)
    assert rc == ainv._lib.ERR_ARG
    assert t.check() == 0 and t.build(irp, ja, val) == 0


def test_invk_factors_are_unit_triangles_usable_by_create():
    """W^T lower and Z upper, as ainv_gpu_create requires; d finite."""
    irp, ja, val = ainv.pde.gen_pde3d(8, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    sv, rc = _build("INVK", irp, ja, val, SUB_FILLIN=1, INV_FILLIN=1)
    assert rc == 0
    f = sv.factors()
    W, Z = _mat(f, "wt", n).tocoo(), _mat(f, "z", n).tocoo()
    assert np.all(W.col <= W.row) and np.all(Z.col >= Z.row)
    assert np.all(np.isfinite(f["d"])) and sv.get_nzeros() == n + W.nnz + Z.nnz

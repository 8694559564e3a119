"""The C oracle against the golden fixtures and known-answer tests.

Fixtures come from tests/golden/make_golden.py, an independent pure-Python
restatement of the reference (src/impl/mld_dsparse_biconjg_llk.F90,
src/impl/mld_d_sparsify.f90, src/impl/mld_d_ainv_bld.F90,
src/impl/mld_d_base_ainv_solver_apply_vect.f90, and for INVK / INVT
src/impl/mld_dsparse_invk.f90, src/impl/mld_dsparse_invt.f90 with their
copyin / inv / copyout routines over a restated MLD2P4 ILU(k) / ILUT).  Integer patterns and
factor values must match bit for bit; applies to 1e-13 relative.
"""
import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLD, "*.npz")))


def _csr(irp, ja, val, n):
    return sp.csr_matrix((val, ja, irp), shape=(n, n))


def _oracle_factors(g, a):
    """The oracle's factors for a fixture: AINV, or INVK / INVT when the
    fixture names its solver and parameters."""
    solver = str(g["solver"]) if "solver" in g.files else "AINV"
    if solver == "INVK":
        p = g["params"]
        return O.invk_build(a, int(p[0]), int(p[1]))
    if solver == "INVT":
        p = g["params"]
        return O.invt_build(a, int(p[0]), float(p[1]), int(p[2]), float(p[3]))
    return O.ainv_build(a, str(g["alg"]), int(g["meta"][2]), float(g["thresh"]))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_golden(path):
    g = np.load(path)
    a = O.CSR(len(g["a_irp"]) - 1, g["a_irp"], g["a_ja"], g["a_val"])
    kind = str(g["kind"])
    if kind in ("poisson", "convdiff"):
        idim = int(g["meta"][0])
        b = tuple(float(v) for v in g["beta"])
        gen = O.gen_pde3d(idim, kind, b)
        np.testing.assert_array_equal(gen.irp, a.irp)
        np.testing.assert_array_equal(gen.ja, a.ja)
        np.testing.assert_array_equal(gen.val, a.val)
    f = _oracle_factors(g, a)
    np.testing.assert_array_equal(f.wt.irp, g["wt_irp"])
    np.testing.assert_array_equal(f.wt.ja, g["wt_ja"])
    np.testing.assert_array_equal(f.wt.val, g["wt_val"])
    np.testing.assert_array_equal(f.z.irp, g["z_irp"])
    np.testing.assert_array_equal(f.z.ja, g["z_ja"])
    np.testing.assert_array_equal(f.z.val, g["z_val"])
    np.testing.assert_array_equal(f.d, g["d"])
    yN = O.ainv_apply(f, g["x"], 1.5, 0.5, g["y0"], "N")
    yT = O.ainv_apply(f, g["x"], -0.75, 2.0, g["y0"], "T")
    np.testing.assert_allclose(yN, g["yN"], rtol=1e-13, atol=1e-13 * np.abs(g["yN"]).max())
    np.testing.assert_allclose(yT, g["yT"], rtol=1e-13, atol=1e-13 * np.abs(g["yT"]).max())


def test_rng_matches_fixture_generator():
    g = np.load(os.path.join(GOLD, "poisson5_llk.npz"))
    np.testing.assert_array_equal(O.rand_uniform(7, 125), g["x"])


@pytest.mark.parametrize("kind", ["poisson", "convdiff"])
def test_exact_biconjugation_inverts(kind):
    """No dropping (thresh 0, fill n): Z D^-1 W^T = A^-1."""
    a = O.gen_pde3d(4, kind, (3.0, -2.0, 1.0))
    n = a.n
    f = O.ainv_build(a, "LLK", n, 0.0)
    M = (_csr(f.z.irp, f.z.ja, f.z.val, n) @ sp.diags(f.d)
         @ _csr(f.wt.irp, f.wt.ja, f.wt.val, n)).toarray()
    A = _csr(a.irp, a.ja, a.val, n).toarray()
    assert np.abs(M @ A - np.eye(n)).max() < 1e-12


def test_hand4_exact():
    g = np.load(os.path.join(GOLD, "hand4.npz"))
    n = 4
    M = (_csr(g["z_irp"], g["z_ja"], g["z_val"], n) @ sp.diags(g["d"])
         @ _csr(g["wt_irp"], g["wt_ja"], g["wt_val"], n)).toarray()
    A = _csr(g["a_irp"], g["a_ja"], g["a_val"], n).toarray()
    np.testing.assert_allclose(M, np.linalg.inv(A), rtol=1e-13, atol=1e-15)


def test_symmetric_matrix_gives_w_equal_z():
    a = O.gen_pde3d(8, "poisson")
    f = O.ainv_build(a, "LLK", 20, 0.1)
    Wt = _csr(f.wt.irp, f.wt.ja, f.wt.val, a.n)
    Z = _csr(f.z.irp, f.z.ja, f.z.val, a.n)
    assert (Wt.T != Z).nnz == 0


def test_factor_shape_invariants():
    a = O.gen_pde3d(9, "convdiff", (30.0, -10.0, 5.0))
    f = O.ainv_build(a, "LLK", 5, 0.05)
    n = a.n
    wl = np.diff(f.wt.irp)
    assert wl.max() <= 5  # per-column cap (Wt rows are W columns)
    for i in range(n):  # unit lower Wt, diagonal last
        cols = f.wt.ja[f.wt.irp[i]:f.wt.irp[i + 1]]
        assert cols[-1] == i and np.all(np.diff(cols) > 0)
        assert f.wt.val[f.wt.irp[i + 1] - 1] == 1.0
    Zc = _csr(f.z.irp, f.z.ja, f.z.val, n).tocsc()
    assert np.diff(Zc.indptr).max() <= 5
    assert np.all(_csr(f.z.irp, f.z.ja, f.z.val, n).diagonal() == 1.0)


def test_apply_transpose_identity():
    """<M x, y> = <x, M^T y> with M = Z D^-1 W^T."""
    a = O.gen_pde3d(7, "convdiff", (20.0, 5.0, -8.0))
    f = O.ainv_build(a, "LLK", 20, 0.1)
    x = O.rand_uniform(1, a.n)
    y = O.rand_uniform(2, a.n)
    lhs = O.ainv_apply(f, x) @ y
    rhs = x @ O.ainv_apply(f, y, trans="T")
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_invalid_trans_rejected():
    a = O.gen_pde3d(3, "poisson")
    f = O.ainv_build(a, "LLK", 20, 0.1)
    with pytest.raises(ValueError):
        O.ainv_apply(f, np.ones(a.n), trans="X")


@pytest.mark.parametrize("method,kind", [("CG", "poisson"), ("BICGSTAB", "convdiff")])
def test_oracle_krylov_converges(method, kind):
    a = O.gen_pde3d(16, kind, (10 / np.sqrt(3),) * 3)
    f = O.ainv_build(a, "LLK", 20, 0.1)
    xs = O.rand_uniform(0, a.n)
    b = O.spmv(a, xs)
    x, it, err, rc = O.solve(method, a, f, b, eps=1e-9, itmax=500)
    assert rc == 0 and err <= 1e-9
    r = b - O.spmv(a, x)
    assert np.linalg.norm(r) <= 1.01e-9 * np.linalg.norm(b)

"""update_a (src/impl/mld_d_base_ainv_update_a.f90:53-79) in the oracle:
known answers that pin the formula d <- 1/(1/d + diag(W^T diag(x) Z))."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O


def _m(c, n):
    return sp.csr_matrix((c.val, c.ja, c.irp), shape=(n, n))


@pytest.mark.parametrize("kind,beta", [("poisson", (0, 0, 0)), ("convdiff", (20.0, -5.0, 8.0))])
def test_exact_factors_give_the_shifted_diagonal(kind, beta):
    """With no dropping W^T A Z = diag(1/d), so after update_a(x) the new d
    is the inverse diagonal of W^T (A + diag(x)) Z."""
    a = O.gen_pde3d(4, kind, beta)
    n = a.n
    f = O.ainv_build(a, "LLK", n, 0.0)
    x = O.rand_uniform(3, n, 0.0, 2.0)
    dn = O.update_a(f, x)
    A = _m(a, n).toarray()
    Wt, Z = _m(f.wt, n).toarray(), _m(f.z, n).toarray()
    np.testing.assert_allclose(np.diag(Wt @ A @ Z), 1.0 / f.d, rtol=1e-12)
    np.testing.assert_allclose(np.diag(Wt @ (A + np.diag(x)) @ Z), 1.0 / dn, rtol=1e-12)


def test_matches_dense_restatement_and_zero_shift():
    a = O.gen_pde3d(7, "convdiff", (10.0, 3.0, -6.0))
    n = a.n
    f = O.ainv_build(a, "LLK", 20, 0.1)
    x = O.rand_uniform(5, n, -0.5, 1.5)
    Wt, Z = _m(f.wt, n), _m(f.z, n)
    e = np.asarray((Wt @ sp.diags(x) @ Z).diagonal())
    np.testing.assert_allclose(O.update_a(f, x), 1.0 / (1.0 / f.d + e), rtol=1e-13)
    np.testing.assert_allclose(O.update_a(f, np.zeros(n)), f.d, rtol=1e-15)


def test_inverse_factors_too():
    """update_a is a method of the common base type: INVK / INVT factors too."""
    a = O.gen_pde3d(6, "convdiff", (4.0, 4.0, 4.0))
    n = a.n
    for f in (O.invk_build(a, 1, 1), O.invt_build(a, 20, 0.05, 20, 0.05)):
        x = O.rand_uniform(9, n, 0.0, 1.0)
        e = np.asarray((_m(f.wt, n) @ sp.diags(x) @ _m(f.z, n)).diagonal())
        np.testing.assert_allclose(O.update_a(f, x), 1.0 / (1.0 / f.d + e), rtol=1e-13)

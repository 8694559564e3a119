"""CPU-only checks of the product library: it loads, exports every symbol
the public header declares, and its host side (solver-type plumbing and the
host factor build) behaves like the reference's plugin types.  No compute
call here touches a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import ainv
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(ainv.LIB_PATH)
    declared = _declared_functions()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    bound = {name for name, _, _ in ainv._lib.SIGNATURES}
    assert set(_declared_functions()) <= bound


def _factors_equal(f, of):
    pairs = [("wt_irp", of.wt.irp), ("wt_ja", of.wt.ja), ("wt_val", of.wt.val),
             ("z_irp", of.z.irp), ("z_ja", of.z.ja), ("z_val", of.z.val), ("d", of.d)]
    for k, v in pairs:
        np.testing.assert_array_equal(f[k], v, err_msg=k)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_host_build_matches_golden(path):
    """Product host build == golden restatement, bit for bit."""
    g = np.load(path)
    solver = str(g["solver"]) if "solver" in g.files else "AINV"
    if solver != "AINV":
        p = g["params"]
        sv = (ainv.mld_d_invk_solver_type() if solver == "INVK"
              else ainv.mld_d_invt_solver_type())
        sv.cseti("SUB_FILLIN", int(p[0]))
        if solver == "INVK":
            sv.cseti("INV_FILLIN", int(p[1]))
        else:
            sv.csetr("SUB_ILUTHRS", float(p[1]))
            sv.cseti("INV_FILLIN", int(p[2]))
            sv.csetr("INV_THRESH", float(p[3]))
        assert sv.build(g["a_irp"], g["a_ja"], g["a_val"]) == 0
        f = sv.factors()
        for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]:
            np.testing.assert_array_equal(f[k], g[k], err_msg=k)
        return
    alg = str(g["alg"])
    sv = ainv.mld_d_ainv_solver_type()
    if alg == "LLK-NOTH":
        assert sv.cseti("AINV_ALG", ainv.AINV_ALG["LLK-NOTH"]) == 0
    else:
        assert sv.csetc("AINV_ALG", alg) == 0
    sv.cseti("SUB_FILLIN", int(g["meta"][2]))
    sv.csetr("SUB_ILUTHRS", float(g["thresh"]))
    assert sv.build(g["a_irp"], g["a_ja"], g["a_val"]) == 0
    f = sv.factors()
    for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]:
        np.testing.assert_array_equal(f[k], g[k], err_msg=k)


@pytest.mark.parametrize("alg", ["LLK", "STAB-LLK", "MLK"])
@pytest.mark.parametrize("idim,kind,beta,fill,thr", [
    (14, "convdiff", (10 / np.sqrt(3),) * 3, 20, 0.1),
    (11, "convdiff", (80.0, -30.0, 15.0), 6, 0.02),
    (12, "poisson", (0, 0, 0), 3, 0.01),
    (10, "convdiff", (-50.0, 20.0, -70.0), 20, 0.0),
])
def test_host_build_matches_oracle(idim, kind, beta, fill, thr, alg):
    irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
    sv = ainv.mld_d_ainv_solver_type()
    assert sv.csetc("AINV_ALG", alg) == 0
    sv.cseti("SUB_FILLIN", fill)
    sv.csetr("SUB_ILUTHRS", thr)
    assert sv.build(irp, ja, val) == 0
    of = O.ainv_build(O.CSR(len(irp) - 1, irp, ja, val), alg, fill, thr)
    _factors_equal(sv.factors(), of)


def _dense(irp, ja, val, n):
    m = np.zeros((n, n))
    for r in range(n):
        for k in range(irp[r], irp[r + 1]):
            m[r, ja[k]] += val[k]
    return m


@pytest.mark.parametrize("kind,beta", [("convdiff", (25.0, -10.0, 5.0)), ("poisson", (0, 0, 0))])
def test_stab_llk_known_answers(kind, beta):
    """STAB-LLK without dropping is an exact biconjugation, Z D^-1 W^T = A^-1;
    on a symmetric A its W equals Z; with dropping its pivots differ from
    LLK's (they come from w_i^T A z_i)."""
    irp, ja, val = ainv.pde.gen_pde3d(5, kind, beta)
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    assert sv.csetc("AINV_ALG", "STAB-LLK") == 0
    sv.cseti("SUB_FILLIN", n)
    sv.csetr("SUB_ILUTHRS", 0.0)
    assert sv.build(irp, ja, val) == 0
    f = sv.factors()
    wt = _dense(f["wt_irp"], f["wt_ja"], f["wt_val"], n)
    z = _dense(f["z_irp"], f["z_ja"], f["z_val"], n)
    m = z @ np.diag(f["d"]) @ wt
    assert np.abs(m @ _dense(irp, ja, val, n) - np.eye(n)).max() < 1e-12
    if kind == "poisson":
        np.testing.assert_array_equal(wt.T, z)
    llk, stab = ainv.mld_d_ainv_solver_type(), ainv.mld_d_ainv_solver_type()
    assert stab.csetc("AINV_ALG", "STAB-LLK") == 0
    for s in (llk, stab):
        s.cseti("SUB_FILLIN", 8)
        s.csetr("SUB_ILUTHRS", 0.05)
        assert s.build(irp, ja, val) == 0
    assert not np.array_equal(llk.factors()["d"], stab.factors()["d"])


def test_generators_match_oracle():
    for idim, kind, b in [(9, "poisson", (0, 0, 0)), (8, "convdiff", (3.0, -7.0, 11.0))]:
        irp, ja, val = ainv.pde.gen_pde3d(idim, kind, b)
        g = O.gen_pde3d(idim, kind, b)
        np.testing.assert_array_equal(irp, g.irp)
        np.testing.assert_array_equal(ja, g.ja)
        np.testing.assert_array_equal(val, g.val)
    np.testing.assert_array_equal(ainv.pde.rand_uniform(0, 5000), O.rand_uniform(0, 5000))
    np.testing.assert_allclose(ainv.pde.rand_normal(5, 5000), O.rand_normal(5, 5000),
                               rtol=0, atol=1e-14)


def test_one_based_build_equals_zero_based():
    irp, ja, val = ainv.pde.gen_pde3d(6, "convdiff", (5.0, 1.0, -2.0))
    a, b = ainv.mld_d_ainv_solver_type(), ainv.mld_d_ainv_solver_type()
    for s in (a, b):
        s.cseti("SUB_FILLIN", 20)
        s.csetr("SUB_ILUTHRS", 0.1)
    assert a.build(irp, ja, val) == 0
    assert b.build(irp + 1, ja + 1, val, one_based=True) == 0
    fa, fb = a.factors(), b.factors()
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k])


def test_solver_settings_and_defaults():
    """Keys, defaults and check() like the Fortran types."""
    sv = ainv.mld_d_ainv_solver_type()
    assert "Fill level             : 0" in sv.descr()   # default fill_in = 0
    assert sv.cseti("sub_fillin", 7) == 0                # keys are case-insensitive
    assert sv.csetr("SUB_ILUTHRS", 0.25) == 0
    assert sv.csetc("ainv_alg", "sym-llk") == 0
    assert sv.cseti("UNKNOWN_KEY", 3) == 0               # base-solver fallthrough
    d = sv.descr()
    assert "Symmetric Left-looking" in d and ": 7" in d and "0.25" in d
    sv2 = ainv.mld_d_ainv_solver_type()
    sv2.cseti("SUB_FILLIN", -4)
    sv2.csetr("SUB_ILUTHRS", -1.0)
    assert sv2.check() == 0                              # reset with a warning
    assert "Fill level             : 1" in sv2.descr()
    assert "Fill threshold         : 0" in sv2.descr()
    assert sv.get_wrksz() == 2
    t = ainv.mld_d_invt_solver_type()
    t.cseti("INV_FILLIN", 20)
    t.csetr("INV_THRESH", 0.05)
    assert "Inverse fill threshold :0.05" in t.descr()
    k = ainv.mld_d_invk_solver_type()
    k.cseti("SUB_FILLIN", 1)
    k.cseti("INV_FILLIN", 1)
    assert "Inverse fill level     :1" in k.descr()


def test_clone_settings_and_clone():
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 5)
    sv.csetr("SUB_ILUTHRS", 0.05)
    other = ainv.mld_d_ainv_solver_type()
    assert sv.clone_settings(other) == 0
    assert other.descr() == sv.descr()
    assert sv.clone_settings(ainv.mld_d_invk_solver_type()) != 0
    irp, ja, val = ainv.pde.gen_pde3d(5, "poisson")
    assert sv.build(irp, ja, val) == 0
    c = sv.clone()
    fa, fc = sv.factors(), c.factors()
    for k in fa:
        np.testing.assert_array_equal(fa[k], fc[k])
    assert c.get_nzeros() == sv.get_nzeros() == 125 + len(fa["wt_ja"]) + len(fa["z_ja"])
    assert sv.free() == 0 and sv.get_nzeros() == 0
    assert c.get_nzeros() > 0


def test_build_errors():
    irp, ja, val = ainv.pde.gen_pde3d(4, "poisson")
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 0)
    assert sv.build(irp, ja, val) == ainv._lib.ERR_ARG        # fill_in < 1 without check()
    sv.cseti("SUB_FILLIN", 4)
    sv.csetc("AINV_ALG", "NOPE")
    assert sv.build(irp, ja, val) == ainv._lib.ERR_ARG        # 'Invalid alg'
    bad = ja.copy()
    bad[3] = 10_000
    sv.csetc("AINV_ALG", "LLK")
    assert sv.build(irp, bad, val) == ainv._lib.ERR_ARG       # column out of range
    assert "out of range" in ainv.last_error()
    unsorted = ja.copy()
    unsorted[[0, 1]] = unsorted[[1, 0]]
    assert sv.build(irp, unsorted, val) == ainv._lib.ERR_ARG
    assert sv.build(irp, ja, val) == 0


def test_apply_requires_device_factors():
    irp, ja, val = ainv.pde.gen_pde3d(4, "poisson")
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    assert sv.build(irp, ja, val) == 0
    y = np.zeros(64)
    assert sv.apply_a(1.0, np.ones(64), 0.0, y) == ainv._lib.ERR_NOT_BUILT
    torch = pytest.importorskip("torch")
    xt, yt = torch.ones(64, dtype=torch.float64), torch.zeros(64, dtype=torch.float64)
    assert sv.apply_a(1.0, xt, 0.0, yt) == ainv._lib.ERR_NOT_BUILT
    with pytest.raises(TypeError):
        sv.apply_a(1.0, np.ones(64), 0.0, yt)               # mixed array kinds
    with pytest.raises(TypeError):
        sv.apply_a(1.0, xt.float(), 0.0, yt)                # not float64
    with pytest.raises(ValueError):
        sv.apply_a(1.0, xt[:32], 0.0, yt)                   # x shorter than n


def test_dump_writes_matrix_market(tmp_path):
    irp, ja, val = ainv.pde.gen_pde3d(3, "convdiff", (1.0, 2.0, 3.0))
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.01)
    assert sv.build(irp, ja, val) == 0
    prefix = str(tmp_path / "dump_ainv_d")
    assert sv.dump(prefix) == 0
    import scipy.io
    f = sv.factors()
    W = scipy.io.mmread(prefix + "_wmat.mtx").tocsr()
    Z = scipy.io.mmread(prefix + "_zmat.mtx").tocsr()
    D = scipy.io.mmread(prefix + "_diag.mtx").ravel()
    np.testing.assert_array_equal(W.indptr, f["wt_irp"])
    np.testing.assert_array_equal(Z.data, f["z_val"])
    np.testing.assert_array_equal(D, f["d"])


def _tie_matrix(seed, n, density=0.25):
    rng = np.random.default_rng(seed)
    m = np.where(rng.random((n, n)) < density, rng.choice([-1.0, 1.0, -0.5, 0.5], (n, n)), 0.0)
    np.fill_diagonal(m, 4.0)
    irp, ja, val = [0], [], []
    for r in range(n):
        c = np.nonzero(m[r])[0]
        ja += c.tolist()
        val += m[r, c].tolist()
        irp.append(len(ja))
    return np.array(irp, np.int32), np.array(ja, np.int32), np.array(val)


def test_mlk_differs_from_llk_only_at_ties():
    """MLK (src/impl/mld_dsparse_biconjg_mlk.F90) walks the same steps as LLK
    through sorted linked lists; only its sparsify (mld_d_sparsify_list with
    psb_hsort) orders equal magnitudes differently.  On the PDE grid the two
    agree; on matrices built from {+-1, +-0.5} they differ, and the product's
    MLK still equals the oracle's literal linked-list restatement."""
    irp, ja, val = ainv.pde.gen_pde3d(10, "convdiff", (-50.0, 20.0, -70.0))
    f = {}
    for alg in ("LLK", "MLK"):
        sv = ainv.mld_d_ainv_solver_type()
        assert sv.csetc("AINV_ALG", alg) == 0
        sv.cseti("SUB_FILLIN", 20)
        sv.csetr("SUB_ILUTHRS", 0.1)
        assert sv.build(irp, ja, val) == 0
        f[alg] = sv.factors()
    for k in f["LLK"]:
        np.testing.assert_array_equal(f["LLK"][k], f["MLK"][k], err_msg=k)
    gm = np.load(os.path.join(GOLD, "mlk_ties20.npz"))
    gl = np.load(os.path.join(GOLD, "llk_ties20.npz"))
    assert not np.array_equal(gm["z_ja"], gl["z_ja"])
    differ = 0
    for seed in (1, 3, 4, 5, 6):
        irp, ja, val = _tie_matrix(seed, 14 + seed)
        n = len(irp) - 1
        for fill, thr in ((2, 0.0), (3, 0.01)):
            sv = ainv.mld_d_ainv_solver_type()
            assert sv.csetc("AINV_ALG", "MLK") == 0
            sv.cseti("SUB_FILLIN", fill)
            sv.csetr("SUB_ILUTHRS", thr)
            assert sv.build(irp, ja, val) == 0
            om = O.ainv_build(O.CSR(n, irp, ja, val), "MLK", fill, thr)
            ol = O.ainv_build(O.CSR(n, irp, ja, val), "LLK", fill, thr)
            _factors_equal(sv.factors(), om)
            differ += not np.array_equal(om.z.ja, ol.z.ja) or not np.array_equal(om.wt.ja, ol.wt.ja)
    assert differ > 0

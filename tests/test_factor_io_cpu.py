"""Factor interchange (no GPU): MatrixMarket load of a dump, in this
library's and in the reference's file layout
(src/impl/mld_d_base_ainv_solver_dmp.f90:82-108), and the binary cache."""
import os

import numpy as np
import pytest

import ainv

KEYS = ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]


def _built(kind="AINV"):
    irp, ja, val = ainv.pde.gen_pde3d(7, "convdiff", (12.0, -4.0, 3.0))
    sv = {"AINV": ainv.mld_d_ainv_solver_type, "INVK": ainv.mld_d_invk_solver_type,
          "INVT": ainv.mld_d_invt_solver_type}[kind]()
    sv.cseti("SUB_FILLIN", 20 if kind != "INVK" else 1)
    sv.csetr("SUB_ILUTHRS", 0.1)
    sv.cseti("INV_FILLIN", 1)
    assert sv.build(irp, ja, val) == 0
    return sv


def _same(a, b):
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("kind", ["AINV", "INVK", "INVT"])
def test_dump_then_load_round_trips(tmp_path, kind):
    sv = _built(kind)
    prefix = str(tmp_path / "f")
    assert sv.dump(prefix) == 0
    other = ainv.mld_d_ainv_solver_type()
    assert other.load(prefix) == 0
    _same(sv.factors(), other.factors())
    assert other.get_nzeros() == sv.get_nzeros()


def test_load_reference_style_files(tmp_path):
    """PSBLAS-style output: comment lines after the banner, entries in any
    order, 1-based, 19 significant digits."""
    p = str(tmp_path / "dump_ainv_d_p000_l001")
    open(p + "_wmat.mtx", "w").write(
        "%%MatrixMarket matrix coordinate real general\n% INVK\n%\n3 3 4\n"
        "3 3  1.000000000000000000E+00\n2 1 -2.500000000000000000E-01\n"
        "1 1  1.000000000000000000E+00\n2 2  1.000000000000000000E+00\n")
    open(p + "_zmat.mtx", "w").write(
        "%%MatrixMarket matrix coordinate real general\n3 3 4\n"
        "1 1 1.0\n1 2 -0.5\n2 2 1.0\n3 3 1.0\n")
    open(p + "_diag.mtx", "w").write(
        "%%MatrixMarket matrix array real general\n% d\n3 1\n0.25\n0.5\n0.125\n")
    sv = ainv.mld_d_invk_solver_type()
    assert sv.load(p) == 0
    f = sv.factors()
    assert list(f["wt_irp"]) == [0, 1, 3, 4] and list(f["wt_ja"]) == [0, 0, 1, 2]
    assert list(f["wt_val"]) == [1.0, -0.25, 1.0, 1.0]
    assert list(f["z_ja"]) == [0, 1, 1, 2] and list(f["d"]) == [0.25, 0.5, 0.125]


def test_load_errors(tmp_path):
    sv = ainv.mld_d_ainv_solver_type()
    assert sv.load(str(tmp_path / "missing")) == ainv._lib.ERR_ARG
    p = str(tmp_path / "bad")
    open(p + "_wmat.mtx", "w").write("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n")
    open(p + "_zmat.mtx", "w").write("%%MatrixMarket matrix coordinate real general\n2 2 0\n")
    open(p + "_diag.mtx", "w").write("%%MatrixMarket matrix array real general\n2 1\n1\n1\n")
    assert sv.load(p) == ainv._lib.ERR_ARG and "bad entry" in ainv.last_error()


def test_cache_round_trip_and_checks(tmp_path):
    sv = _built("INVT")
    path = str(tmp_path / "f.bin")
    assert sv.save(path) == 0
    other = ainv.mld_d_invt_solver_type()
    assert other.restore(path) == 0
    _same(sv.factors(), other.factors())
    assert other.descr() == sv.descr()                      # settings travel too
    assert ainv.mld_d_ainv_solver_type().restore(path) == ainv._lib.ERR_ARG   # other type
    raw = bytearray(open(path, "rb").read())
    raw[len(raw) // 2] ^= 0xFF
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(bytes(raw))
    assert other.restore(bad) == ainv._lib.ERR_ARG and "corrupt" in ainv.last_error()
    open(bad, "wb").write(bytes(raw[:100]))
    assert other.restore(bad) == ainv._lib.ERR_ARG
    assert ainv.mld_d_ainv_solver_type().save(path) == ainv._lib.ERR_NOT_BUILT


@pytest.mark.parametrize("alg", ["STAB-LLK", "MLK"])
def test_cache_keeps_the_biconjugation_variant(tmp_path, alg):
    """AINV factors of the STAB-LLK / MLK variants: the cache restores the
    factors bit for bit and the variant with them (descr names it)."""
    irp, ja, val = ainv.pde.gen_pde3d(7, "convdiff", (12.0, -4.0, 3.0))
    sv = ainv.mld_d_ainv_solver_type()
    assert sv.csetc("AINV_ALG", alg) == 0
    sv.cseti("SUB_FILLIN", 6)
    sv.csetr("SUB_ILUTHRS", 0.05)
    assert sv.build(irp, ja, val) == 0
    path = str(tmp_path / "f.bin")
    assert sv.save(path) == 0
    other = ainv.mld_d_ainv_solver_type()
    assert other.restore(path) == 0
    _same(sv.factors(), other.factors())
    assert other.descr() == sv.descr()
    assert {"STAB-LLK": "Stabilized", "MLK": "list merge"}[alg] in other.descr()

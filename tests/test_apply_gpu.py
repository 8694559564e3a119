"""GPU parity of the AINV apply (src/impl/mld_d_base_ainv_solver_apply_vect.f90)
against the CPU oracle on the same factors and inputs, through the C-ABI.

Tolerances (norm-wise relative, ||y - y_oracle||_inf / ||y_oracle||_inf):
  FP64 factors: 1e-12 (the north-star bound for the FP64 apply); the 'N'
                apply is moreover bit-identical to the oracle's: both sum
                each row in column order with every product and sum
                rounded once, and form alpha*acc + beta*y alike
  FP32 factors: 5e-6   (float32 storage and accumulation)
  BF16 factors: 3e-2   (bfloat16 storage, float32 accumulation)
"""
import glob
import os

import numpy as np
import pytest

import ainv
import oracle as O
from util import build_factors, device_factors, oracle_factors, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {"FP64": 1e-12, "FP32": 5e-6, "BF16": 3e-2}


def _gpu_apply(df, x, alpha, beta, y0, trans):
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(DEV)
    yd = torch.from_numpy(np.ascontiguousarray(y0)).to(DEV)
    df.apply(xd, yd, alpha, beta, trans)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_apply_matches_golden(path):
    g = np.load(path)
    f = {k: g[k] for k in ["wt_irp", "wt_ja", "wt_val", "z_irp", "z_ja", "z_val", "d"]}
    df = device_factors(f)
    yN = _gpu_apply(df, g["x"], 1.5, 0.5, g["y0"], "N")
    yT = _gpu_apply(df, g["x"], -0.75, 2.0, g["y0"], "T")
    assert relerr(yN, g["yN"]) <= 1e-12
    assert relerr(yT, g["yT"]) <= 1e-12


@pytest.mark.parametrize("idim,kind,beta", [
    (40, "poisson", (0, 0, 0)),                  # the 40^3 Poisson workload
    (50, "convdiff", (10 / np.sqrt(3),) * 3),    # convection-diffusion, upwind
    (23, "convdiff", (90.0, -40.0, 25.0)),       # strong convection, ragged rows
])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_fp64_parity(idim, kind, beta, trans):
    irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
    f = build_factors(irp, ja, val)
    of = oracle_factors(f)
    n = len(f["d"])
    x, y0 = ainv.pde.rand_uniform(11, n), ainv.pde.rand_uniform(12, n)
    df = device_factors(f)
    for alpha, beta_ in [(1.0, 0.0), (1.5, 0.5), (-2.0, 1.0)]:
        y = _gpu_apply(df, x, alpha, beta_, y0, trans)
        ref = O.ainv_apply(of, x, alpha, beta_, y0, trans)
        assert relerr(y, ref) <= 1e-12, (alpha, beta_)
        if trans == "N":
            np.testing.assert_array_equal(y, ref)


def test_apply_full_size_convdiff_200():
    """The 200^3 convection-diffusion factors (8M rows): GPU vs oracle apply
    on the same product-built factors, plus linearity of the device apply."""
    irp, ja, val = ainv.pde.gen_pde3d(200, "convdiff", (10 / np.sqrt(3),) * 3)
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    x = ainv.pde.rand_uniform(0, n)
    df = device_factors(f)
    y = _gpu_apply(df, x, 1.0, 0.0, np.zeros(n), "N")
    ref = O.ainv_apply(oracle_factors(f), x, 1.0, 0.0, None, "N")
    assert relerr(y, ref) <= 1e-12
    np.testing.assert_array_equal(y, ref)
    x2 = ainv.pde.rand_uniform(1, n)
    y2 = _gpu_apply(df, x2, 1.0, 0.0, np.zeros(n), "N")
    y12 = _gpu_apply(df, 2.0 * x - 3.0 * x2, 1.0, 0.0, np.zeros(n), "N")
    assert relerr(y12, 2.0 * y - 3.0 * y2) <= 1e-12


@pytest.mark.parametrize("prec", ["FP32", "BF16"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_mixed_precision(prec, trans):
    irp, ja, val = ainv.pde.gen_pde3d(30, "convdiff", (10 / np.sqrt(3),) * 3)
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    x, y0 = ainv.pde.rand_uniform(3, n), ainv.pde.rand_uniform(4, n)
    df = device_factors(f, prec)
    assert df.prec == prec
    y = _gpu_apply(df, x, 1.25, -0.5, y0, trans)
    ref = O.ainv_apply(oracle_factors(f), x, 1.25, -0.5, y0, trans)
    assert relerr(y, ref) <= TOL[prec]


def test_beta_zero_ignores_y_contents():
    irp, ja, val = ainv.pde.gen_pde3d(12, "poisson")
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    x = ainv.pde.rand_uniform(5, n)
    y = _gpu_apply(device_factors(f), x, 1.0, 0.0, np.full(n, np.nan), "N")
    assert np.isfinite(y).all()
    assert relerr(y, O.ainv_apply(oracle_factors(f), x)) <= 1e-12


@pytest.mark.parametrize("n_side", [1, 2, 3])
def test_tiny_and_ragged_sizes(n_side):
    """n = 1, 8, 27: a single partial slice of 32 rows."""
    irp, ja, val = ainv.pde.gen_pde3d(n_side, "convdiff", (3.0, -2.0, 1.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    x = ainv.pde.rand_uniform(6, n)
    for trans in "NT":
        y = _gpu_apply(device_factors(f), x, 0.5, 0.0, np.zeros(n), trans)
        assert relerr(y, O.ainv_apply(oracle_factors(f), x, 0.5, 0.0, None, trans)) <= 1e-12


def test_host_array_form_equals_device_form():
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (4.0, 5.0, 6.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df = device_factors(f)
    x, y0 = ainv.pde.rand_uniform(7, n), ainv.pde.rand_uniform(8, n)
    yh = df.apply_host(x, 2.0, 0.25, y0, "N")
    yd = _gpu_apply(df, x, 2.0, 0.25, y0, "N")
    np.testing.assert_array_equal(yh, yd)


def test_apply_is_deterministic():
    irp, ja, val = ainv.pde.gen_pde3d(32, "convdiff", (10.0, 0.0, -3.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df = device_factors(f)
    x = ainv.pde.rand_uniform(9, n)
    a = _gpu_apply(df, x, 1.0, 0.0, np.zeros(n), "N")
    b = _gpu_apply(df, x, 1.0, 0.0, np.zeros(n), "N")
    np.testing.assert_array_equal(a, b)


def test_invalid_arguments_are_rejected():
    irp, ja, val = ainv.pde.gen_pde3d(4, "poisson")
    f = build_factors(irp, ja, val)
    df = device_factors(f)
    x = torch.ones(64, dtype=torch.float64, device=DEV)
    y = torch.zeros(64, dtype=torch.float64, device=DEV)
    with pytest.raises(ainv.AinvError) as e:
        df.apply(x, y, 1.0, 0.0, "X")
    assert e.value.info == ainv._lib.ERR_ARG
    with pytest.raises(ainv.AinvError):   # factors swapped: W^T must be lower
        ainv.DeviceFactors((f["z_irp"], f["z_ja"], f["z_val"]),
                           (f["wt_irp"], f["wt_ja"], f["wt_val"]), f["d"])


def test_one_based_upload():
    irp, ja, val = ainv.pde.gen_pde3d(9, "convdiff", (1.0, 2.0, 3.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df1 = ainv.DeviceFactors((f["wt_irp"] + 1, f["wt_ja"] + 1, f["wt_val"]),
                             (f["z_irp"] + 1, f["z_ja"] + 1, f["z_val"]), f["d"], one_based=True)
    x = ainv.pde.rand_uniform(10, n)
    np.testing.assert_array_equal(_gpu_apply(df1, x, 1.0, 0.0, np.zeros(n), "N"),
                                  _gpu_apply(device_factors(f), x, 1.0, 0.0, np.zeros(n), "N"))


def test_solver_type_build_cnv_apply():
    """The plugin type end to end: precset, build with a device mold, apply_v,
    apply_a, clone, free."""
    irp, ja, val = ainv.pde.gen_pde3d(16, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.set("AINV_ALG", "LLK")
    sv.set("SUB_FILLIN", 20)
    sv.set("SUB_ILUTHRS", 0.1)
    assert sv.check() == 0
    assert sv.build(irp, ja, val, amold="FP64") == 0
    of = oracle_factors(sv.factors())
    x = ainv.pde.rand_uniform(13, n)
    xd = torch.from_numpy(x).to(DEV)
    yd = torch.zeros(n, dtype=torch.float64, device=DEV)
    assert sv.apply(1.0, xd, 0.0, yd, "N") == 0
    torch.cuda.synchronize()
    assert relerr(yd.cpu().numpy(), O.ainv_apply(of, x)) <= 1e-12
    yh = np.zeros(n)
    assert sv.apply_a(1.0, x, 0.0, yh, "T") == 0
    assert relerr(yh, O.ainv_apply(of, x, trans="T")) <= 1e-12
    c = sv.clone()
    yc = np.zeros(n)
    assert c.apply_a(1.0, x, 0.0, yc, "N") == 0
    np.testing.assert_array_equal(yc, yd.cpu().numpy())
    assert sv.device.get_nzeros() == sv.get_nzeros()
    assert sv.sizeof() > sv.device.sizeof() > 0
    assert sv.free() == 0
    assert sv.apply_a(1.0, x, 0.0, yh, "N") == ainv._lib.ERR_NOT_BUILT
    assert c.apply_a(1.0, x, 0.0, yc, "N") == 0


def test_cnv_changes_precision():
    irp, ja, val = ainv.pde.gen_pde3d(10, "poisson")
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val) == 0
    assert sv.device is None
    for p in ["BF16", "FP32", "FP64"]:
        assert sv.cnv(p) == 0
        assert sv.device.prec == p


def _random_unit_triangular(n, per_row, lower, seed):
    """Random unit-triangular CSR with scattered columns (no shared offsets)."""
    rng = np.random.default_rng(seed)
    irp, ja, val = [0], [], []
    for i in range(n):
        pool = np.arange(0, i) if lower else np.arange(i + 1, n)
        k = min(len(pool), int(rng.integers(0, per_row + 1)))
        cols = sorted(rng.choice(pool, size=k, replace=False).tolist()) if k else []
        row = (cols + [i]) if lower else ([i] + cols)
        vals = [1.0 if c == i else float(rng.uniform(-0.5, 0.5)) for c in row]
        ja += row
        val += vals
        irp.append(len(ja))
    return np.array(irp, np.int32), np.array(ja, np.int32), np.array(val)


@pytest.mark.parametrize("trans", ["N", "T"])
def test_apply_column_mode_random_factors(trans):
    """Scattered patterns force the per-entry column encoding."""
    n = 3000
    wt = _random_unit_triangular(n, 9, True, 1)
    z = _random_unit_triangular(n, 9, False, 2)
    d = ainv.pde.rand_uniform(3, n, 0.5, 2.0)
    f = dict(wt_irp=wt[0], wt_ja=wt[1], wt_val=wt[2], z_irp=z[0], z_ja=z[1], z_val=z[2], d=d)
    df = device_factors(f)
    for which in ("wt", "z", "zt", "w"):
        lay = df.layout_info(which)
        assert lay["offset_slices"] < lay["nslices"] // 4, lay   # mostly column mode
    x, y0 = ainv.pde.rand_uniform(4, n), ainv.pde.rand_uniform(5, n)
    y = _gpu_apply(df, x, 0.75, -1.5, y0, trans)
    ref = O.ainv_apply(oracle_factors(f), x, 0.75, -1.5, y0, trans)
    assert relerr(y, ref) <= 1e-12


def test_stencil_factors_use_offset_mode():
    irp, ja, val = ainv.pde.gen_pde3d(40, "convdiff", (10 / np.sqrt(3),) * 3)
    f = build_factors(irp, ja, val)
    df = device_factors(f)
    for which in ("wt", "z", "zt", "w"):
        lay = df.layout_info(which)
        assert lay["offset_slices"] == lay["nslices"]
        assert lay["nidx"] <= 8 * lay["nslices"]          # a few offsets per slice
        assert lay["slots"] <= 1.02 * 4 * 64000 + 32 * 4   # ~4 slots per row


def _scattered_factors(n, per_row=5, seed=11):
    """Unit triangular W^T (lower) and Z (upper) whose off-diagonal entries sit
    anywhere in their triangle: every chunk of the host-array pipeline then
    depends on far-away chunks."""
    rng = np.random.default_rng(seed)

    def tri(lower):
        irp, ja, va = [0], [], []
        for i in range(n):
            lo, hi = (0, i) if lower else (i + 1, n)
            cols = rng.integers(lo, hi, per_row) if hi > lo else np.zeros(0, np.int64)
            cols = np.unique(np.append(cols, i))
            ja.extend(cols.tolist())
            va.extend(np.where(cols == i, 1.0, rng.uniform(-0.3, 0.3, len(cols))).tolist())
            irp.append(len(ja))
        return np.array(irp, np.int32), np.array(ja, np.int32), np.array(va)

    wt, z = tri(True), tri(False)
    return dict(wt_irp=wt[0], wt_ja=wt[1], wt_val=wt[2], z_irp=z[0], z_ja=z[1], z_val=z[2],
                d=rng.uniform(0.5, 2.0, n))


@pytest.mark.parametrize("fused", ["1", "0"])
@pytest.mark.parametrize("kind", ["stencil", "scattered"])
def test_pipelined_host_apply_equals_device_form(kind, fused, monkeypatch):
    """Page-locked host arrays go through the chunked pipeline: copies of x
    with one persistent sweep kernel writing y to the host (fused), or the
    event-driven stream form; FP64 results are bit-identical to the
    device-array apply for both trans and beta = 0 / != 0."""
    monkeypatch.setenv("AINV_HOST_FUSED", fused)
    if kind == "stencil":
        irp, ja, val = ainv.pde.gen_pde3d(22, "convdiff", (4.0, -5.0, 6.0))
        f = build_factors(irp, ja, val)
    else:
        f = _scattered_factors(9000)
    n = len(f["d"])
    df = device_factors(f)
    x, y0 = ainv.pde.rand_uniform(17, n), ainv.pde.rand_uniform(18, n)
    # nominal chunks of 512 rows (ramped: 29 chunks at 22^3), 1024 and 4000 rows
    for rows in ("512", "1024", "4000"):
        monkeypatch.setenv("AINV_HOST_CHUNK_ROWS", rows)
        for trans in "NT":
            for alpha, beta in ((1.0, 0.0), (2.0, -0.75)):
                xp = torch.from_numpy(x.copy()).pin_memory()
                yp = torch.from_numpy(y0.copy()).pin_memory()
                df.apply_host(xp, alpha, beta, yp, trans)
                yd = _gpu_apply(df, x, alpha, beta, y0, trans)
                np.testing.assert_array_equal(yp.numpy(), yd, err_msg=f"{rows} {trans} {beta}")
                # the pageable form takes the serial path: same numbers
                np.testing.assert_array_equal(df.apply_host(x, alpha, beta, y0, trans), yd)


@pytest.mark.parametrize("prec", ["FP32", "BF16", "FP32_ACC64", "BF16_ACC64"])
def test_pipelined_host_apply_reduced_precision(prec, monkeypatch):
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (1.0, 2.0, 3.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df = device_factors(f, prec)
    x, y0 = ainv.pde.rand_uniform(21, n), ainv.pde.rand_uniform(22, n)
    monkeypatch.setenv("AINV_HOST_CHUNK_ROWS", "640")
    tol = {"FP32": 5e-6, "BF16": 3e-2, "FP32_ACC64": 5e-6, "BF16_ACC64": 3e-2}[prec]
    for trans in "NT":
        xp = torch.from_numpy(x.copy()).pin_memory()
        yp = torch.from_numpy(y0.copy()).pin_memory()
        df.apply_host(xp, 1.5, 0.5, yp, trans)
        ref = O.ainv_apply(oracle_factors(f), x, 1.5, 0.5, y0, trans)
        assert relerr(yp.numpy(), ref) <= tol, (prec, trans)


def test_repeated_host_apply_on_the_same_arrays(monkeypatch):
    """The same page-locked arrays on repeated calls (the fused pipeline's
    chunk flags carry a new epoch per call): every call reads the arrays'
    current contents, with scalars and trans changing between calls."""
    irp, ja, val = ainv.pde.gen_pde3d(21, "convdiff", (3.0, 1.0, -2.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df = device_factors(f)
    monkeypatch.setenv("AINV_HOST_CHUNK_ROWS", "1024")
    xp = torch.zeros(n, dtype=torch.float64).pin_memory()
    yp = torch.zeros(n, dtype=torch.float64).pin_memory()
    y0 = ainv.pde.rand_uniform(40, n)
    calls = [("N", 1.0, 0.0)] * 4 + [("N", 0.5, 0.0)] * 3 + [("T", 1.0, 0.25)] * 3 + \
            [("N", 1.0, 0.0)] * 3
    for k, (trans, alpha, beta) in enumerate(calls):
        x = ainv.pde.rand_uniform(100 + k, n)
        xp.copy_(torch.from_numpy(x))
        yp.copy_(torch.from_numpy(y0))
        df.apply_host(xp, alpha, beta, yp, trans)
        np.testing.assert_array_equal(yp.numpy(), _gpu_apply(df, x, alpha, beta, y0, trans),
                                      err_msg=f"call {k}")


def test_host_apply_in_place(monkeypatch):
    """x and y the same page-locked array (y = op(M) y): the call copies all
    of x before writing y, so the result equals the out-of-place apply."""
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (2.0, -1.0, 3.0))
    f = build_factors(irp, ja, val)
    n = len(f["d"])
    df = device_factors(f)
    monkeypatch.setenv("AINV_HOST_CHUNK_ROWS", "512")
    x = ainv.pde.rand_uniform(31, n)
    for trans in "NT":
        ref = _gpu_apply(df, x, 1.25, 0.0, np.zeros(n), trans)
        buf = torch.from_numpy(x.copy()).pin_memory()
        df.apply_host(buf, 1.25, 0.0, buf, trans)
        np.testing.assert_array_equal(buf.numpy(), ref)


def test_solver_apply_a_on_pinned_tensors(monkeypatch):
    """The solver type's array-form apply with page-locked CPU tensors takes
    the pipelined path and gives the same bits as with numpy arrays."""
    irp, ja, val = ainv.pde.gen_pde3d(18, "convdiff", (6.0, -2.0, 4.0))
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val, amold="FP64") == 0
    monkeypatch.setenv("AINV_HOST_CHUNK_ROWS", "512")
    x, y0 = ainv.pde.rand_uniform(51, n), ainv.pde.rand_uniform(52, n)
    for trans in "NT":
        yn = y0.copy()
        assert sv.apply_a(0.5, x, 1.5, yn, trans) == 0
        xp = torch.from_numpy(x.copy()).pin_memory()
        yp = torch.from_numpy(y0.copy()).pin_memory()
        assert sv.apply_a(0.5, xp, 1.5, yp, trans) == 0
        np.testing.assert_array_equal(yp.numpy(), yn)

"""Inputs the benchmark builds for its general-pattern leg: the scattered
factors keep every row's diagonal and values, stay unit triangular with
strictly increasing columns (the device layout's contract), keep their
columns within the stated band, and apply like the oracle says they should
(checked against a dense product on a small case)."""
import os
import sys

import numpy as np

import ainv
import oracle as O

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_scattered_factors_contract():
    irp, ja, val = ainv.pde.gen_pde3d(14, "convdiff", bench.BETA)
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val) == 0
    f = sv.factors()
    n = len(f["d"])
    band = 200
    g = bench.scattered_factors(f, band=band, seed=3)
    np.testing.assert_array_equal(g["d"], f["d"])
    for k, lower in (("wt", True), ("z", False)):
        ip, j, v = g[k + "_irp"], g[k + "_ja"], g[k + "_val"]
        row = np.repeat(np.arange(n), np.diff(ip))
        assert ((j <= row) if lower else (j >= row)).all()
        assert (np.abs(j - row) <= band).all()
        same_row = row[1:] == row[:-1]
        assert (np.diff(j)[same_row] > 0).all()                 # strictly increasing
        np.testing.assert_array_equal(v[j == row], 1.0)         # unit diagonal kept
        assert len(j) >= 0.97 * len(f[k + "_ja"])               # few collisions dropped
        patterns = {tuple(j[ip[i]:ip[i + 1]] - i) for i in range(0, n, 7)}
        assert len(patterns) > n // 14                          # rows do not share patterns
    x = O.rand_uniform(4, n)
    of = O.Factors(O.CSR(n, g["wt_irp"], g["wt_ja"], g["wt_val"]),
                   O.CSR(n, g["z_irp"], g["z_ja"], g["z_val"]), g["d"])
    W = np.zeros((n, n))
    Z = np.zeros((n, n))
    for M, k in ((W, "wt"), (Z, "z")):
        ip = g[k + "_irp"]
        for i in range(n):
            M[i, g[k + "_ja"][ip[i]:ip[i + 1]]] = g[k + "_val"][ip[i]:ip[i + 1]]
    np.testing.assert_allclose(O.ainv_apply(of, x), Z @ (g["d"] * (W @ x)), rtol=1e-12,
                               atol=1e-12)

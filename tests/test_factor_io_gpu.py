"""Factors loaded from a dump or restored from the cache apply on the GPU
exactly as the factors they were saved from (bit-identical y)."""
import numpy as np
import pytest

import ainv

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def test_loaded_factors_apply_identically(tmp_path):
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (10.0, 2.0, -3.0))
    n = len(irp) - 1
    sv = ainv.mld_d_ainv_solver_type()
    sv.cseti("SUB_FILLIN", 20)
    sv.csetr("SUB_ILUTHRS", 0.1)
    assert sv.build(irp, ja, val, amold="FP64") == 0
    prefix, cache = str(tmp_path / "f"), str(tmp_path / "f.bin")
    assert sv.dump(prefix) == 0 and sv.save(cache) == 0
    a, b = ainv.mld_d_ainv_solver_type(), ainv.mld_d_ainv_solver_type()
    assert a.cnv("FP64") == 0 and b.cnv("FP64") == 0
    assert a.load(prefix) == 0 and b.restore(cache) == 0      # uploaded on arrival
    x = torch.from_numpy(ainv.pde.rand_uniform(1, n)).to(DEV)
    ys = []
    for s in (sv, a, b):
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        assert s.apply(1.0, x, 0.0, y, "N") == 0
        ys.append(y.cpu().numpy())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ys[0], ys[1])
    np.testing.assert_array_equal(ys[0], ys[2])

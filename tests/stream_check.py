"""Parity of the kernels a process uses under AINV_STREAM=<0|1> (set by the
caller before this module runs): apply 'N'/'T' for FP64/FP32/BF16 factors,
the A product and a BiCGSTAB solve, against the CPU oracle.  Prints one JSON
line; exits nonzero on a violation.  Driven by tests/test_stream_gpu.py."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "mld-ainv_b200")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import ainv  # noqa: E402
import oracle as O  # noqa: E402
from util import build_factors, device_factors, oracle_factors, relerr  # noqa: E402

TOL = {"FP64": 1e-12, "FP32": 5e-6, "BF16": 3e-2}


def main(idim):
    out = {"stream": os.environ.get("AINV_STREAM"), "idim": idim}
    irp, ja, val = ainv.pde.gen_pde3d(idim, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    f = build_factors(irp, ja, val)
    of = oracle_factors(f)
    x, y0 = ainv.pde.rand_uniform(1, n), ainv.pde.rand_uniform(2, n)
    ok = True
    for prec in ("FP64", "FP32", "BF16"):
        df = device_factors(f, prec)
        for trans, beta in (("N", 0.0), ("N", 0.5), ("T", 0.5)):
            xd = torch.from_numpy(x).cuda()
            yd = torch.from_numpy(y0).cuda()
            df.apply(xd, yd, 1.25, beta, trans)
            torch.cuda.synchronize()
            e = relerr(yd.cpu().numpy(), O.ainv_apply(of, x, 1.25, beta, y0, trans))
            out[f"{prec}_{trans}_{beta}"] = e
            ok &= e <= TOL[prec]
        df.check()
    A = ainv.DeviceOperator(irp, ja, val)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0).cuda()
    A.spmv(xd, yd, 2.0, -1.0)
    torch.cuda.synchronize()
    e = relerr(yd.cpu().numpy(), O.spmv(O.CSR(n, irp, ja, val), x, 2.0, -1.0, y0))
    out["spmv"] = e
    ok &= e <= 1e-12
    b = O.spmv(O.CSR(n, irp, ja, val), ainv.pde.rand_uniform(0, n))
    for prec in ("FP64", "BF16"):
        xx = torch.zeros(n, dtype=torch.float64, device="cuda")
        res = A.solve(torch.from_numpy(b).cuda(), xx, device_factors(f, prec), "BICGSTAB", 1e-9, 3000)
        true = np.linalg.norm(b - O.spmv(O.CSR(n, irp, ja, val), xx.cpu().numpy())) / np.linalg.norm(b)
        out[f"solve_{prec}"] = [res.info, res.iter, true]
        ok &= res.converged and true <= 1.05e-9
    A.check()
    out["ok"] = bool(ok)
    print(json.dumps(out))
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]) if len(sys.argv) > 1 else 48))

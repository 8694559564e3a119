"""Solve server on the GPU: continuous batching of BiCGSTAB solves against
resident operators, through the ainv_server_* C-ABI.

The central properties: a request's result is the same alone and in a mix,
and it is the single-solve result.  The server sums every dot in the
canonical order of the single-solve loop (slice sums folded in fixed
groups and ranges), and its operator kernels compute each member's rows
with the single-solve arithmetic, so the iterates depend neither on the
other requests nor on the blocks a request gets: the tests assert
bit-identical solutions and iteration counts, against a request's solo run
and against ainv_gpu_solve.  Converged results meet the FP64 relative
residual on b - A x (tolerance 1e-8, as the serving workload asks).
"""
import numpy as np
import pytest

import ainv
import oracle as O
from ainv import serve, workload
from util import build_factors, device_factors, oracle_factors, oracle_spread, within_spread

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
EPS = 1e-8

SPECS = [
    (12, "poisson", (0.0, 0.0, 0.0)),
    (17, "convdiff", (8.0, -3.0, 5.0)),
    (21, "convdiff", (-2.0, 15.0, 1.0)),
    (9, "convdiff", (0.5, 0.5, 19.0)),
]


def _operators(prec="FP32"):
    ops = []
    for idim, kind, beta in SPECS:
        irp, ja, val = ainv.pde.gen_pde3d(idim, kind, beta)
        f = build_factors(irp, ja, val)
        ops.append(dict(a=ainv.DeviceOperator(irp, ja, val), f=device_factors(f, prec),
                        csr=O.CSR(len(irp) - 1, irp, ja, val), fac=f))
    return ops


def _requests(ops, count):
    out = []
    for rid in range(count):
        k = rid % len(ops)
        out.append((k, workload.request_rhs(1000 + rid, ops[k]["csr"].n)))
    return out


def _run(ops, reqs, max_slots, iters, order=None, alone=False):
    with serve.SolveServer(max_slots=max_slots, iters_per_launch=iters) as srv:
        ids = [srv.add_operator(o["a"], o["f"]) for o in ops]
        xs = [np.zeros(len(b)) for _, b in reqs]
        res = [None] * len(reqs)
        order = range(len(reqs)) if order is None else order
        if alone:
            for j in order:
                rid = srv.submit(ids[reqs[j][0]], reqs[j][1], xs[j], EPS, 2000)
                res[j] = srv.wait(rid)
        else:
            rids = {j: srv.submit(ids[reqs[j][0]], reqs[j][1], xs[j], EPS, 2000) for j in order}
            for j in order:
                res[j] = srv.wait(rids[j])
        stats = srv.stats()
    return xs, res, stats


def _true_relres(csr, x, b):
    return np.linalg.norm(b - O.spmv(csr, x)) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["FP32", "FP64"])
def test_alone_equals_mixed(prec):
    ops = _operators(prec)
    reqs = _requests(ops, 12)
    x1, r1, s1 = _run(ops, reqs, max_slots=1, iters=4, alone=True)
    order = list(np.random.default_rng(3).permutation(len(reqs)))
    x2, r2, s2 = _run(ops, reqs, max_slots=8, iters=3, order=order)
    assert s1["peak_active"] == 1 and s2["peak_active"] > 1
    for j, (k, b) in enumerate(reqs):
        assert r1[j].converged and r2[j].converged, (j, r1[j], r2[j])
        assert r1[j].iter == r2[j].iter, j
        assert np.array_equal(x1[j], x2[j]), j            # bit-identical
        assert _true_relres(ops[k]["csr"], x2[j], b) <= 1.05 * EPS
        assert r2[j].err <= EPS


def test_fp64_iterations_within_oracle_spread():
    ops = _operators("FP64")
    reqs = _requests(ops, 4)
    xs, res, _ = _run(ops, reqs, max_slots=4, iters=4)
    for j, (k, b) in enumerate(reqs):
        lo, hi = oracle_spread("BICGSTAB", ops[k]["csr"], oracle_factors(ops[k]["fac"]), b,
                                EPS, 2000)
        assert res[j].converged
        assert within_spread(res[j].iter, lo, hi), (j, res[j].iter, lo, hi)


def test_admission_is_bounded_by_device_memory():
    ops = _operators("FP32")[1:2]          # one operator: every request the same size
    budget = int(2.5 * serve.request_bytes(ops[0]["csr"].n))
    reqs = _requests(ops, 10)
    with serve.SolveServer(max_slots=8, hbm_bytes=budget, iters_per_launch=2) as srv:
        ids = [srv.add_operator(o["a"], o["f"]) for o in ops]
        xs = [np.zeros(len(b)) for _, b in reqs]
        rids = [srv.submit(ids[k], b, xs[j], EPS, 2000) for j, (k, b) in enumerate(reqs)]
        res = [srv.wait(r) for r in rids]
        st = srv.stats()
    assert all(r.converged for r in res)
    assert st["arena_bytes"] <= budget and st["arena_peak"] <= st["arena_bytes"]
    assert st["peak_active"] == 2                # two fit, a third never does
    assert st["completed"] == len(reqs)
    # first come, first served: admission order follows submission order
    admits = [r.t_admit for r in res]
    assert admits == sorted(admits)


def test_oversized_request_is_rejected():
    ops = _operators("FP32")[:1]
    n = ops[0]["csr"].n
    with serve.SolveServer(max_slots=2, hbm_bytes=serve.request_bytes(n) // 2) as srv:
        op = srv.add_operator(ops[0]["a"], ops[0]["f"])
        with pytest.raises(ainv.AinvError) as e:
            srv.submit(op, np.ones(n), np.zeros(n))
        assert e.value.info == 4025


def test_status_codes_and_special_cases():
    ops = _operators("FP32")[:2]
    with serve.SolveServer(max_slots=4, iters_per_launch=4) as srv:
        ids = [srv.add_operator(o["a"], o["f"]) for o in ops]
        n0, n1 = ops[0]["csr"].n, ops[1]["csr"].n
        b = workload.request_rhs(5, n1)
        x_short, x_zero, x_ok = np.zeros(n1), np.full(n0, 7.0), np.zeros(n1)
        r_short = srv.submit(ids[1], b, x_short, EPS, 2)           # itmax too small
        r_zero = srv.submit(ids[0], np.zeros(n0), x_zero, EPS, 50)  # b = 0
        r_ok = srv.submit(ids[1], b, x_ok, EPS, 2000)
        a, z, c = srv.wait(r_short), srv.wait(r_zero), srv.wait(r_ok)
        assert a.status == 4104 and a.iter == 2                      # NOCONV
        assert z.status == 0 and z.iter == 0 and np.all(x_zero == 0.0)
        assert c.converged and _true_relres(ops[1]["csr"], x_ok, b) <= 1.05 * EPS
        with pytest.raises(ainv.AinvError):
            srv.submit(99, b, x_ok)
        with pytest.raises(ainv.AinvError):
            srv.wait(123456)
        assert srv.stats()["completed"] == 3


def test_many_requests_stream_through_few_slots():
    """More requests than slots, submitted from a second thread while the
    engine runs: every request completes and matches its solo result."""
    import threading
    ops = _operators("FP32")
    reqs = _requests(ops, 24)
    x_alone, r_alone, _ = _run(ops, reqs[:4], max_slots=1, iters=4, alone=True)
    with serve.SolveServer(max_slots=3, iters_per_launch=2) as srv:
        ids = [srv.add_operator(o["a"], o["f"]) for o in ops]
        xs = [np.zeros(len(b)) for _, b in reqs]
        rids = [None] * len(reqs)

        def producer():
            for j, (k, b) in enumerate(reqs):
                rids[j] = srv.submit(ids[k], b, xs[j], EPS, 2000)

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        res = [srv.wait(r) for r in rids]
        st = srv.stats()
    assert all(r.converged for r in res) and st["peak_active"] <= 3
    for j in range(4):
        assert np.array_equal(xs[j], x_alone[j]) and res[j].iter == r_alone[j].iter


def test_both_precision_families_in_one_server():
    """FP32 and FP32_ACC64 operators side by side: the server re-captures its
    graph with both kernel families, and each result still equals its solo
    run bit for bit."""
    ops = _operators("FP32")[:2] + _operators("FP32_ACC64")[2:]
    reqs = _requests(ops, 8)
    x1, r1, _ = _run(ops, reqs, max_slots=1, iters=4, alone=True)
    x2, r2, st = _run(ops, reqs, max_slots=8, iters=4, order=list(reversed(range(8))))
    assert st["peak_active"] > 1
    for j, (k, b) in enumerate(reqs):
        assert r1[j].converged and r2[j].converged
        assert r1[j].iter == r2[j].iter and np.array_equal(x1[j], x2[j]), j
        assert _true_relres(ops[k]["csr"], x2[j], b) <= 1.05 * EPS


def test_requests_on_one_operator_share_reads():
    """Ten concurrent requests on one operator: the operator kernels serve
    them as groups (8 + 2 members) that read each chunk of A and of the
    factors once for all members; each result equals its solo run bit for
    bit and meets the tolerance."""
    ops = _operators("FP32")[2:3]
    reqs = _requests(ops, 10)
    x1, r1, _ = _run(ops, reqs, max_slots=1, iters=4, alone=True)
    x2, r2, st = _run(ops, reqs, max_slots=10, iters=3)
    assert st["peak_active"] == 10
    for j, (k, b) in enumerate(reqs):
        assert r1[j].converged and r2[j].converged
        assert r1[j].iter == r2[j].iter and np.array_equal(x1[j], x2[j]), j
        assert _true_relres(ops[k]["csr"], x2[j], b) <= 1.05 * EPS


@pytest.mark.parametrize("prec", ["FP64", "FP32_ACC64", "FP32", "BF16"])
def test_served_equals_single_solve(prec):
    """Six concurrent requests on two operators (groups of members that share
    the operator's reads): each solution and iteration count equals
    ainv_gpu_solve's on the same right-hand side, bit for bit."""
    ops = _operators(prec)[1:3]
    reqs = _requests(ops, 6)
    xs, res, st = _run(ops, reqs, max_slots=6, iters=3)
    assert st["peak_active"] == 6
    for j, (k, b) in enumerate(reqs):
        bd = torch.tensor(b, device="cuda")
        xd = torch.zeros_like(bd)
        r = ops[k]["a"].solve(bd, xd, ops[k]["f"], eps=EPS, itmax=2000)
        assert res[j].converged and r.info == 0
        assert res[j].iter == r.iter, (j, res[j].iter, r.iter)
        assert np.array_equal(xs[j], xd.cpu().numpy()), j


def test_served_fp64_equals_oracle():
    """With FP64 factors a served request's iterates are the oracle's
    ordered-dot BiCGSTAB iterates: same count, same solution bits."""
    ops = _operators("FP64")[1:2]
    reqs = _requests(ops, 3)
    xs, res, _ = _run(ops, reqs, max_slots=3, iters=4)
    for j, (k, b) in enumerate(reqs):
        x, it, err, rc = O.solve("BICGSTAB", ops[k]["csr"], oracle_factors(ops[k]["fac"]), b,
                                 eps=EPS, itmax=2000, order="device")
        assert rc == 0 and res[j].iter == it, (j, res[j].iter, it)
        assert np.array_equal(xs[j], x), j


_CHUNK_SCRIPT = """
import sys, numpy as np, torch
sys.path[:0] = {paths!r}
import ainv
from ainv import serve, workload
from util import build_factors, device_factors
irp, ja, val = ainv.pde.gen_pde3d(17, "convdiff", (8.0, -3.0, 5.0))
f = build_factors(irp, ja, val)
a = ainv.DeviceOperator(irp, ja, val)
fd = device_factors(f, "FP32_ACC64")
out = []
with serve.SolveServer(max_slots=3, iters_per_launch=2) as srv:
    op = srv.add_operator(a, fd)
    bs = [workload.request_rhs(1000 + j, a.n) for j in range(3)]
    xs = [np.zeros(a.n) for _ in bs]
    ids = [srv.submit(op, b, x, 1e-8, 2000) for b, x in zip(bs, xs)]
    res = [srv.wait(i) for i in ids]
for b, x, r in zip(bs, xs, res):
    bd = torch.tensor(b, device="cuda"); xd = torch.zeros_like(bd)
    s = a.solve(bd, xd, fd, eps=1e-8, itmax=2000)
    assert r.converged and r.iter == s.iter, (r.iter, s.iter)
    assert np.array_equal(x, xd.cpu().numpy())
print("OK")
"""


def test_streamed_operator_kernels_equal_single_solve():
    """With streaming selected for every kind (AINV_SERVER_STREAM=15) the
    server's streamed operator kernels run instead of the slice-shared ones
    and give the same bits."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    paths = [here, root, os.path.join(root, "oracle"), os.path.join(root, "mld-ainv_b200")]
    env = dict(os.environ, AINV_SERVER_STREAM="15")
    out = subprocess.run([sys.executable, "-c", _CHUNK_SCRIPT.format(paths=paths)],
                         env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and "OK" in out.stdout, out.stderr[-3000:]

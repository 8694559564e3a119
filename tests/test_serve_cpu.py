"""Host logic of the solve server (no GPU): the block plan, request sizes,
and the serving workload generator."""
import numpy as np
import pytest

import ainv
from ainv import serve, workload


@pytest.mark.parametrize("rows,grid", [
    ([13824, 2097152, 512, 1], 1184),
    ([100000] * 64, 1184),
    ([2097152] * 3, 64),
    ([1, 2, 3], 3),
    ([], 10),
])
def test_plan_invariants(rows, grid):
    b0, nb = serve.plan(rows, grid)
    chunks = [max(1, (r + 511) // 512) for r in rows]
    assert np.all(nb >= 1) and np.all(nb <= chunks)
    assert nb.sum() <= grid
    assert np.all(b0 == np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int32)[:len(rows)])


def test_plan_is_proportional():
    rows = [2097152, 262144, 13824]
    b0, nb = serve.plan(rows, 1184)
    assert nb[0] > nb[1] > nb[2] >= 1
    assert nb.sum() >= 1184 - len(rows)


def test_plan_rejects_more_slots_than_blocks():
    with pytest.raises(ainv.AinvError):
        serve.plan([10] * 5, 4)


def test_request_bytes():
    """A request's device bytes: 11 FP64 vectors and the apply intermediate
    (rows rounded up to 32), then the slice sums of 3 dots (one per 32-row
    slice, rounded up to 32) and their range sums (one per 256 groups of 8
    slices, rounded up to 32), the whole rounded up to 256 bytes."""
    def up(x, m):
        return -(-x // m) * m
    for n in (1, 31, 33, 1000, 13824, 2097152, 8000000):
        ns = -(-n // 32)
        nr = -(-(-(-ns // 8)) // 256)
        want = up((12 * up(n, 32) + 3 * (up(ns, 32) + up(nr, 32))) * 8, 256)
        b = serve.request_bytes(n)
        assert b == want, (n, b, want)
        assert b % 256 == 0 and b >= 12 * 8 * n
    assert serve.request_bytes(2097152) > serve.request_bytes(13824)


def test_serving_operators_are_deterministic_and_in_range():
    a = workload.serving_operators()
    b = workload.serving_operators()
    assert a == b and len(a) == 16
    assert all(24 <= s.idim <= 128 for s in a)
    kinds = {s.kind for s in a}
    assert kinds == {"poisson", "convdiff"}
    for s in a:
        mag = float(np.linalg.norm(s.beta))
        assert (mag == 0.0) if s.kind == "poisson" else (0.0 <= mag <= 20.0 + 1e-12)


def test_poisson_arrivals():
    t = workload.poisson_arrivals(500.0, 20000)
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 500.0) < 0.05 / 500.0
    assert abs(gaps.std() - 1 / 500.0) < 0.05 / 500.0   # exponential: sd = mean
    np.testing.assert_array_equal(t, workload.poisson_arrivals(500.0, 20000))


def test_request_ops_and_rhs():
    ops = workload.request_ops(2000, 16)
    assert ops.min() == 0 and ops.max() == 15
    np.testing.assert_array_equal(workload.request_rhs(7, 100), ainv.pde.rand_normal(7, 100))

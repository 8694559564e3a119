"""The canonical summation order of the Krylov dots.

The device library sums every dot in one fixed order (32-row slice trees,
groups of 8 slices added in order, 256-group ranges folded by 256 threads
and the same trees, then the ranges folded alike) so that its Krylov iterates do not depend on the grid
or the device; the oracle's ordered dot restates that order so that its
iterates equal the device's bit for bit.  Here the oracle's C form is
checked against a second, independent numpy restatement, and the two
orders the oracle offers (device, sequential) are compared on a solve."""
import numpy as np
import pytest

import ainv
import oracle as O


def _tree32(u):
    u = u.copy()
    o = 16
    while o > 0:
        u[..., :o] = u[..., :o] + u[..., o:2 * o]
        o //= 2
    return u[..., 0]


def _fold256(src):
    t = np.zeros(256)
    for j in range(256):
        a = 0.0
        for s in range(j, len(src), 256):
            a = a + src[s]
        t[j] = a
    w = _tree32(t.reshape(8, 32))
    tot = 0.0
    for k in range(8):
        tot = tot + w[k]
    return tot


def _canonical_dot(a, b):
    n = len(a)
    ns = -(-n // 32)
    p = np.zeros(ns * 32)
    p[:n] = a * b
    S = _tree32(p.reshape(ns, 32))
    G = []
    for g in range(0, ns, 8):
        t = 0.0
        for v in S[g:g + 8]:
            t = t + v
        G.append(t)
    G = np.array(G)
    R = np.array([_fold256(G[j:j + 256]) for j in range(0, len(G), 256)])
    return _fold256(R)


@pytest.mark.parametrize("n", [1, 31, 32, 33, 1000, 256 * 1024, 256 * 1024 + 5, 300_003])
def test_device_order_dot_matches_numpy_restatement(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n) * np.exp(rng.uniform(-20, 20, n))
    b = rng.standard_normal(n)
    got = O.dot_device_order(a, b)
    assert got == _canonical_dot(a, b)
    assert got == pytest.approx(float(np.dot(a, b)), rel=1e-9, abs=1e-300)


def test_device_order_is_not_the_sequential_sum():
    """On ill-conditioned data the orders differ in the last bits: the order
    is a real choice, which is why both sides must share it."""
    rng = np.random.default_rng(3)
    a = rng.standard_normal(200_000) * np.exp(rng.uniform(-10, 10, 200_000))
    b = rng.standard_normal(200_000)
    s = 0.0
    for v in a * b:
        s = s + v
    assert O.dot_device_order(a, b) != s


def test_oracle_orders_and_history():
    """Both dot orders converge; the recorded history ends at the returned
    residual and decreases overall; the two orders' counts are close."""
    irp, ja, val = ainv.pde.gen_pde3d(20, "convdiff", (10 / np.sqrt(3),) * 3)
    n = len(irp) - 1
    a = O.CSR(n, irp, ja, val)
    of = O.ainv_build(a, "LLK", 20, 0.1)
    b = O.spmv(a, O.rand_uniform(0, n, -1.0, 1.0))
    res = {}
    for order in ("device", "sequential"):
        x, it, err, rc, hist = O.solve("BICGSTAB", a, of, b, eps=1e-9, itmax=500, order=order,
                                       history=True)
        assert rc == 0 and err <= 1e-9
        assert len(hist) == it and hist[-1] == err
        res[order] = it
    assert abs(res["device"] - res["sequential"]) <= max(2, 0.1 * res["sequential"])

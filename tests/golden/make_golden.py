"""Generate the golden fixtures under tests/golden/.

The reference (Fortran on PSBLAS/MLD2P4) cannot be built in this
environment and ships no golden vectors, so these fixtures come from an
independent pure-Python restatement of the reference algorithm, written
separately from the C oracle and following the Fortran line by line:

  - maxval scaling and d = weight/p   src/impl/mld_d_ainv_bld.F90:115-184
  - left-looking biconjugation        src/impl/mld_dsparse_biconjg_llk.F90:35-366
  - SYM-LLK (W = Z)                   src/impl/mld_dsparse_biconjg_s_llk.F90:246
  - LLK without the alpha test        src/impl/mld_dsparse_biconjg_llk_noth.F90
  - STAB-LLK (stabilised pivots)      src/impl/mld_dsparse_biconjg_s_ft_llk.F90
  - MLK (sparsify_list, psb_hsort)    src/impl/mld_dsparse_biconjg_mlk.F90,
                                      src/impl/mld_d_sparsify.f90:152-230
  - sparsify (diag + nzrmax-1 largest, PSBLAS magnitude-heap tie order)
                                      src/impl/mld_d_sparsify.f90:35-149
  - Z CSC->CSR, W CSC->transpose      src/mld_d_biconjg_mod.F90:131-135
  - apply 'N' / 'T'                   src/impl/mld_d_base_ainv_solver_apply_vect.f90:112-127

Cases are tiny (pure-Python loops).  Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import heapq
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EPSTOL = 1.1e-16


# ---------------------------------------------------------------- inputs --
def pde3d(idim, kind, beta):
    """7-point operator, x fastest; kind 'poisson' (6/-1) or 'convdiff'."""
    m = idim
    h = 1.0 / (idim + 1)
    ih2 = 1.0 / (h * h)
    if kind == "poisson":
        lo = [-1.0] * 3
        up = [-1.0] * 3
        diag = 6.0
    else:
        lo, up = [0.0] * 3, [0.0] * 3
        diag = 6.0 * ih2
        for a in range(3):
            lo[a] = -ih2 - (beta[a] if beta[a] > 0 else 0.0) / h
            up[a] = -ih2 + (beta[a] if beta[a] < 0 else 0.0) / h
            diag += abs(beta[a]) / h
    rows = []
    for iz in range(m):
        for iy in range(m):
            for ix in range(m):
                r = ix + m * (iy + m * iz)
                e = []
                if iz > 0: e.append((r - m * m, lo[2]))
                if iy > 0: e.append((r - m, lo[1]))
                if ix > 0: e.append((r - 1, lo[0]))
                e.append((r, diag))
                if ix < m - 1: e.append((r + 1, up[0]))
                if iy < m - 1: e.append((r + m, up[1]))
                if iz < m - 1: e.append((r + m * m, up[2]))
                rows.append(e)
    return rows


def rows_to_csr(rows):
    irp = [0]
    ja, va = [], []
    for e in rows:
        for c, v in e:
            ja.append(c)
            va.append(v)
        irp.append(len(ja))
    return (np.array(irp, np.int32), np.array(ja, np.int32), np.array(va, np.float64))


# ------------------------------------------------ PSBLAS magnitude heap --
class MagHeapDown:
    """psb_d_idx_heap with dir=psb_asort_down_ (1-based binary heap)."""

    def __init__(self):
        self.k = [None]
        self.i = [None]

    def insert(self, key, idx):
        self.k.append(key)
        self.i.append(idx)
        c = len(self.k) - 1
        while c > 1:
            p = c // 2
            if abs(self.k[c]) <= abs(self.k[p]):
                break
            self.k[c], self.k[p] = self.k[p], self.k[c]
            self.i[c], self.i[p] = self.i[p], self.i[c]
            c = p

    def get_first(self):
        last = len(self.k) - 1
        if last <= 0:
            return None
        key, idx = self.k[1], self.i[1]
        self.k[1], self.i[1] = self.k[last], self.i[last]
        self.k.pop()
        self.i.pop()
        last -= 1
        c = 1
        while c <= last // 2:
            if 2 * c == last or abs(self.k[2 * c]) > abs(self.k[2 * c + 1]):
                j = 2 * c
            else:
                j = 2 * c + 1
            if abs(self.k[c]) < abs(self.k[j]):
                self.k[c], self.k[j] = self.k[j], self.k[c]
                self.i[c], self.i[j] = self.i[j], self.i[c]
                c = j
            else:
                break
        return key, idx


def sparsify(idiag, nzrmax, thresh, zw, nzset):
    xw = [0.0]
    xwid = [idiag]
    h = MagHeapDown()
    for i in sorted(nzset):
        if i == idiag:
            xw[0] = zw[i]
        elif abs(zw[i]) >= thresh:
            h.insert(zw[i], i)
        zw[i] = 0.0
    k = 1
    while k != nzrmax:
        got = h.get_first()
        if got is None:
            break
        xw.append(got[0])
        xwid.append(got[1])
        k += 1
    order = sorted(range(len(xwid)), key=lambda t: xwid[t])
    return [xwid[t] for t in order], [xw[t] for t in order]


def hsort_abs_down(x, ix):
    """PSBLAS psb_hsort(dir=psb_asort_down_): the entries inserted in order
    into a 1-based heap with the smallest |x| at the root (rise while
    strictly smaller than the parent); the root taken out len-1 times into
    the last free position (the last entry sinks toward the smaller child --
    left only when strictly smaller or the last one -- while strictly
    larger); the first position keeps the last root."""
    hk, hv = [None], [None]
    for key, idx in zip(x, ix):
        hk.append(key)
        hv.append(idx)
        c = len(hk) - 1
        while c > 1 and abs(hk[c]) < abs(hk[c // 2]):
            hk[c], hk[c // 2] = hk[c // 2], hk[c]
            hv[c], hv[c // 2] = hv[c // 2], hv[c]
            c //= 2
    m = len(x)
    ox, oi = [None] * m, [None] * m
    for j in range(m - 1, 0, -1):
        ox[j], oi[j] = hk[1], hv[1]
        hk[1], hv[1] = hk[-1], hv[-1]
        hk.pop()
        hv.pop()
        last, c = len(hk) - 1, 1
        while 2 * c <= last:
            l = 2 * c
            ch = l if (l == last or abs(hk[l]) < abs(hk[l + 1])) else l + 1
            if not abs(hk[c]) > abs(hk[ch]):
                break
            hk[c], hk[ch] = hk[ch], hk[c]
            hv[c], hv[ch] = hv[ch], hv[c]
            c = ch
    if m:
        ox[0], oi[0] = hk[1], hv[1]
    return ox, oi


def sparsify_list(idiag, nzrmax, thresh, zw, nzset):
    """mld_d_sparsify_list (src/impl/mld_d_sparsify.f90:152-230), used by MLK:
    entries in index order with the diagonal swapped into slot 0, the rest
    by descending magnitude (psb_hsort), cut at the first value below
    thresh and at nzrmax entries, survivors sorted by index."""
    xw, xi = [], []
    for r in sorted(nzset):
        xw.append(zw[r])
        xi.append(r)
        if r == idiag:
            xw[0], xw[-1] = xw[-1], xw[0]
            xi[0], xi[-1] = xi[-1], xi[0]
        zw[r] = 0.0
    m = len(xw)
    if m > 2:
        xw[1:], xi[1:] = hsort_abs_down(xw[1:], xi[1:])
    k = 1
    while k < m and not abs(xw[k]) < thresh:
        k += 1
    nz = max(1, min(k, nzrmax))
    order = sorted(range(nz), key=lambda t: xi[t])
    return [xi[t] for t in order], [xw[t] for t in order]


# --------------------------------------------------------- biconjugation --
def biconjg_half(n, dot_rows, cand_rows, nzrmax, thresh, piv0, noth, keep=sparsify):
    """dot_rows[j]: list of (k, a) giving the dot vector j; cand_rows[kr]:
    indices j whose dot vector touches position kr; the starting candidates
    for column i are cand_rows[i] filtered to j < i."""
    piv = [0.0] * n
    piv[0] = piv0
    cols = [([0], [1.0])]
    zw = [0.0] * n
    for i in range(1, n):
        zw[i] = 1.0
        nzset = {i}
        rh = []
        flagged = set()
        for j in cand_rows[i]:
            if j < i:
                heapq.heappush(rh, j)
                flagged.add(j)
        lastj = -1
        while True:
            j = None
            while rh:
                c = heapq.heappop(rh)
                if c > lastj:
                    lastj = c
                    j = c
                    break
            if j is None:
                break
            flagged.discard(j)
            if j >= i:
                continue
            s = 0.0
            for k, a in dot_rows[j]:
                s = s + zw[k] * a
            alpha = -s / piv[j]
            if noth or abs(alpha) > thresh:
                ci, cv = cols[j]
                for kr, v in zip(ci, cv):
                    zw[kr] = zw[kr] + alpha * v
                    if kr not in nzset:
                        nzset.add(kr)
                        for nj in cand_rows[kr]:
                            if nj not in flagged and j < nj < i:
                                heapq.heappush(rh, nj)
                                flagged.add(nj)
        s = 0.0
        for k, a in dot_rows[i]:
            s = s + zw[k] * a
        if abs(s) < EPSTOL:
            s = 1.0e-3
        piv[i] = s
        cols.append(keep(i, nzrmax, thresh, zw, nzset))
    return piv, cols


def sp_x_mat(xi, xv, mrows):
    """y = x^T M for a sparse index-sorted x and M given by rows: x's entries
    in order, each merged as x_k * M(k, :) into the sorted result (psb_d_spvspm
    with M = A, psb_d_spmspv with M = A's columns giving A x;
    src/mld_d_biconjg_mod.F90:145-296, through PSBLAS psb_nspaxpby)."""
    acc = {}
    for k, xk in zip(xi, xv):
        for c, a in mrows[k]:
            acc[c] = acc.get(c, 0.0) + xk * a
    idx = sorted(acc)
    return idx, [acc[c] for c in idx]


def stab_llk(n, srows, scols, col_idx, row_idx, nzrmax, thresh, piv0):
    """mld_dsparse_biconjg_s_ft_llk (src/impl/mld_dsparse_biconjg_s_ft_llk.F90):
    for each i, column i of Z (step j: (w_j^T A) . z) and then of W (step j:
    (A z_j) . w), both divided by the common pivot of column j; the pivot of
    column i is (A z_i) . w_i over the kept entries, with the 1e-3 guard."""
    piv = [0.0] * n
    piv[0] = piv0
    zcols, wcols = [([0], [1.0])], [([0], [1.0])]
    zw = [0.0] * n
    for i in range(1, n):
        for half in (0, 1):
            cand = col_idx if half == 0 else row_idx
            own = zcols if half == 0 else wcols
            other = wcols if half == 0 else zcols
            mrows = srows if half == 0 else scols
            zw[i] = 1.0
            nzset = {i}
            rh = []
            flagged = set()
            for j in cand[i]:
                if j < i:
                    heapq.heappush(rh, j)
                    flagged.add(j)
            lastj = -1
            while True:
                j = None
                while rh:
                    c = heapq.heappop(rh)
                    if c > lastj:
                        lastj = c
                        j = c
                        break
                if j is None or j >= i:
                    break
                flagged.discard(j)
                yi, yv = sp_x_mat(*other[j], mrows)
                s = 0.0
                for k, y in zip(yi, yv):
                    s = s + y * zw[k]
                alpha = -s / piv[j]
                if abs(alpha) > thresh:
                    ci, cv = own[j]
                    for kr, v in zip(ci, cv):
                        zw[kr] = zw[kr] + alpha * v
                        if kr not in nzset:
                            nzset.add(kr)
                            for nj in cand[kr]:
                                if nj not in flagged and j < nj < i:
                                    heapq.heappush(rh, nj)
                                    flagged.add(nj)
            own.append(sparsify(i, nzrmax, thresh, zw, nzset))
        yi, yv = sp_x_mat(*zcols[i], scols)
        w = dict(zip(*wcols[i]))
        s = 0.0
        for k, y in zip(yi, yv):
            if k in w:
                s = s + y * w[k]
        if abs(s) < EPSTOL:
            s = 1.0e-3
        piv[i] = s
    return piv, zcols, wcols


def ainv_build(rows, alg, nzrmax, thresh):
    n = len(rows)
    mx = max(abs(v) for e in rows for _, v in e)
    w = 1.0 / mx
    srows = [[(c, v * w) for c, v in e if 0 <= c < n] for e in rows]
    scols = [[] for _ in range(n)]
    for r, e in enumerate(srows):
        for c, v in e:
            scols[c].append((r, v))
    a11 = 0.0
    for c, v in srows[0]:
        if c == 0:
            a11 = v
            break
    if abs(a11) < EPSTOL:
        a11 = 1.0e-3
    col_idx = [[r for r, _ in e] for e in scols]
    row_idx = [[c for c, _ in e] for e in srows]
    noth = alg == "LLK-NOTH"
    # MLK (src/impl/mld_dsparse_biconjg_mlk.F90) visits the same steps as LLK
    # through sorted linked lists; only its list form of sparsify differs
    keep = sparsify_list if alg == "MLK" else sparsify
    if alg == "STAB-LLK":
        p, zcols, wcols = stab_llk(n, srows, scols, col_idx, row_idx, nzrmax, thresh, a11)
    else:
        p, zcols = biconjg_half(n, srows, col_idx, nzrmax, thresh, a11, noth, keep)
    if alg == "SYM-LLK":
        wcols = zcols
    elif alg != "STAB-LLK":
        _, wcols = biconjg_half(n, scols, row_idx, nzrmax, thresh, a11, noth, keep)
    d = np.array([(1.0 if abs(v) < EPSTOL else 1.0 / v) * w for v in p])
    # Wt CSR: row i = column w_i
    wt = rows_to_csr([list(zip(ci, cv)) for ci, cv in wcols])
    # Z CSR: transpose of the CSC columns
    zrows = [[] for _ in range(n)]
    for c, (ci, cv) in enumerate(zcols):
        for r, v in zip(ci, cv):
            zrows[r].append((c, v))
    z = rows_to_csr(zrows)
    return wt, z, d


def csr_mv(csr, x, trans="N"):
    irp, ja, va = csr
    n = len(irp) - 1
    y = [0.0] * n
    if trans == "N":
        for i in range(n):
            s = 0.0
            for k in range(irp[i], irp[i + 1]):
                s = s + va[k] * x[ja[k]]
            y[i] = s
    else:
        for r in range(n):
            for k in range(irp[r], irp[r + 1]):
                y[ja[k]] = y[ja[k]] + va[k] * x[r]
    return y


def apply(wt, z, d, x, trans, alpha, beta, y0):
    if trans == "N":
        t = csr_mv(wt, x)
        t = [d[i] * t[i] for i in range(len(t))]
        u = csr_mv(z, t)
    else:
        t = csr_mv(z, x, "T")
        t = [d[i] * t[i] for i in range(len(t))]
        u = csr_mv(wt, t, "T")
    return np.array([alpha * u[i] + beta * y0[i] for i in range(len(u))])


def splitmix_uniform(seed, n, lo=-1.0, hi=1.0):
    M = (1 << 64) - 1
    out = np.empty(n)
    for i in range(n):
        x = ((seed << 40) + i) & M
        x = (x + 0x9E3779B97F4A7C15) & M
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
        x = x ^ (x >> 31)
        out[i] = lo + (hi - lo) * ((x >> 11) * (1.0 / 9007199254740992.0))
    return out


# ------------------------------------------------------ INVK / INVT ----
# MLD2P4's ILU(k) / ILUT (external to the reference; restated from their
# published IKJ row algorithm) and the plugin's sparse inverses
# (src/impl/mld_dsparse_invk.f90, mld_d_invk_{copyin,inv,copyout}.f90,
# src/impl/mld_dsparse_invt.f90, mld_d_invt_{copyin,inv,copyout}.f90).
# Rows are lists of (column, value); L and U carry no diagonal.

def dnrm2(xs):
    """Reference BLAS dnrm2 (one-pass scaled sum of squares)."""
    scale, ssq = 0.0, 1.0
    for x in xs:
        if x != 0.0:
            ax = abs(x)
            if scale < ax:
                ssq = 1.0 + ssq * ((scale / ax) * (scale / ax))
                scale = ax
            else:
                ssq = ssq + (ax / scale) * (ax / scale)
    return scale * math.sqrt(ssq)


def drain(h):
    """Pop an ascending index heap, skipping repeats (the lastk test)."""
    last = None
    while h:
        k = heapq.heappop(h)
        if k != last:
            last = k
            yield k


def iluk(rows, fill):
    n = len(rows)
    unset = -(n + 1)
    row, lev = [0.0] * n, [unset] * n
    L, U, Ulev, d = [], [], [], [0.0] * n
    for i in range(n):
        h = []
        for c, v in rows[i]:
            row[c], lev[c] = v, 0
            heapq.heappush(h, c)
        idxs = []
        for k in drain(h):
            idxs.append(k)
            if row[k] != 0.0 and lev[k] <= fill and k < i:
                rwk, lk = row[k], lev[k]
                row[k] = row[k] * d[k]
                for (j, uv), ul in zip(U[k], Ulev[k]):
                    if lev[j] < 0:
                        heapq.heappush(h, j)
                        lev[j] = -lev[j]
                    row[j] = row[j] - rwk * uv
                    lev[j] = min(lev[j], lk + ul + 1)
        lr, ur, ulv, piv = [], [], [], 0.0
        for j in idxs:
            if j < i and lev[j] <= fill:
                lr.append((j, row[j]))
            elif j == i:
                piv = row[j]
            elif j > i and lev[j] <= fill:
                ur.append((j, row[j]))
                ulv.append(lev[j])
            row[j], lev[j] = 0.0, unset
        if abs(piv) < EPSTOL:
            raise ZeroDivisionError(f"ILU(k) pivot at row {i}")
        d[i] = 1.0 / piv
        L.append(lr)
        U.append([(j, d[i] * v) for j, v in ur])
        Ulev.append(ulv)
    return L, U, d


def top_magnitude(items, cap):
    """Offer (index, value) pairs to the magnitude heap, pop `cap` of them."""
    h = MagHeapDown()
    for j, v in items:
        h.insert(v, j)
    out = []
    for _ in range(cap):
        v, j = h.get_first()
        out.append((j, v))
    return out


def ilut(rows, fill, thresh):
    n = len(rows)
    w = 1.0 / max(abs(v) for e in rows for _, v in e)
    row = [0.0] * n
    L, U, d = [], [], [0.0] * n
    for i in range(n):
        h, vals = [], []
        nlw = nup = 0
        jmaxup, dmaxup = None, 0.0
        for c, v in rows[i]:
            row[c] = w * v
            vals.append(row[c])
            heapq.heappush(h, c)
            if c < i:
                nlw += 1
            if c > i:
                nup += 1
                if abs(row[c]) > dmaxup:
                    jmaxup, dmaxup = c, abs(row[c])
        tol = thresh * dnrm2(vals)
        idxs = []
        for k in drain(h):
            idxs.append(k)
            if k < i:
                rwk = row[k]
                row[k] = row[k] * d[k]
                if abs(row[k]) < tol:
                    row[k] = 0.0
                    continue
                for j, uv in U[k]:
                    if row[j] == 0.0:
                        heapq.heappush(h, j)
                    row[j] = row[j] - rwk * uv
        low = [(j, row[j]) for j in idxs if j < i and not abs(row[j]) < tol]
        if len(low) > nlw + fill:
            low = top_magnitude(low, nlw + fill)
        L.append(sorted(low))
        if i not in idxs or abs(row[i]) < EPSTOL:
            raise ZeroDivisionError(f"ILUT pivot at row {i}")
        d[i] = 1.0 / row[i]
        up = [(j, row[j]) for j in idxs
              if j > i and (j == jmaxup or not abs(row[j]) < tol)]
        if len(up) > nup + fill:
            top = top_magnitude(up, nup + fill)
            if jmaxup is not None and jmaxup not in [j for j, _ in top]:
                top[-1] = (jmaxup, row[jmaxup])
            up = top
        U.append([(j, d[i] * v) for j, v in sorted(up)])
        for j in idxs:
            row[j] = 0.0
    return L, U, [v * w for v in d]


def sparse_invk(U, fill):
    n = len(U)
    Z = []
    for i in range(n - 1):
        row, lev = {i: 1.0}, {i: 0}
        h = []
        for c, v in U[i]:
            row[c], lev[c] = -1.0 * v, 0
            heapq.heappush(h, c)
        idxs = [i]
        for k in drain(h):
            if k == i:
                continue
            idxs.append(k)
            if row[k] != 0.0 and lev[k] <= fill:
                for j, uv in U[k]:
                    if j not in lev:
                        heapq.heappush(h, j)
                        lev[j], row[j] = n + 1, 0.0
                    row[j] = row[j] - row[k] * uv
                    lev[j] = min(lev[j], lev[k] + 1)
        Z.append([(j, row[j]) for j in idxs if lev[j] <= fill])
    Z.append([(n - 1, 1.0)])
    return Z


def sparse_invt(U, fill, thresh):
    n = len(U)
    Z = []
    for i in range(n - 1):
        row = {i: 1.0}
        queued = set()
        h = []
        for c, v in U[i]:
            row[c] = -1.0 * v
            heapq.heappush(h, c)
            queued.add(c)
        nup = sum(1 for c, _ in U[i] if c > i)
        nrmi = dnrm2([v for _, v in U[i]])
        if nrmi < 1.0:
            nrmi = math.sqrt(1.0 + nrmi * nrmi)
        else:
            nrmi = nrmi * math.sqrt(1.0 + 1.0 / (nrmi * nrmi))
        tol = thresh * nrmi
        idxs = [i]
        for k in drain(h):
            rwk = row[k]
            queued.discard(k)
            if abs(rwk) < tol:
                row[k] = 0.0
                continue
            for j, uv in U[k]:
                row[j] = row.get(j, 0.0) - rwk * uv
                if j not in queued:
                    if abs(row[j]) < tol:
                        row[j] = 0.0
                    else:
                        heapq.heappush(h, j)
                        queued.add(j)
            idxs.append(k)
        cap = nup + fill
        acc, wmin = [], sys.float_info.max
        for j in idxs:
            v = row[j]
            if j != i and abs(v) < tol:
                continue
            if len(acc) > cap and abs(v) < wmin:
                continue
            wmin = min(abs(v), wmin)
            acc.append((j, v))
        if len(acc) > cap:
            acc = top_magnitude(acc, cap)
        Z.append(sorted(acc))
    Z.append([(n - 1, 1.0)])
    return Z


def transpose_rows(R):
    T = [[] for _ in R]
    for r, e in enumerate(R):
        for c, v in e:
            T[c].append((r, v))
    return T


def inverse_build(rows, solver, p):
    """INVK p = (fill1, fill2); INVT p = (fill, thresh, invfill, invthresh)."""
    if solver == "INVK":
        L, U, d = iluk(rows, p[0])
        inv = lambda T: sparse_invk(T, p[1])  # noqa: E731
    else:
        L, U, d = ilut(rows, p[0], p[1])
        inv = lambda T: sparse_invt(T, p[2], p[3])  # noqa: E731
    z = rows_to_csr(inv(U))
    wt = rows_to_csr(transpose_rows(inv(transpose_rows(L))))
    return wt, z, np.array(d)


# ---------------------------------------------------------------- cases --
CASES = [
    # name, grid, kind, beta, alg, fill_in, thresh
    ("poisson5_llk", 5, "poisson", (0, 0, 0), "LLK", 20, 0.1),
    ("poisson5_cap3", 5, "poisson", (0, 0, 0), "LLK", 3, 0.01),
    ("poisson4_exact", 4, "poisson", (0, 0, 0), "LLK", 64, 0.0),
    ("convdiff6_llk", 6, "convdiff", (40.0, -25.0, 10.0), "LLK", 20, 0.1),
    ("convdiff6_cap4", 6, "convdiff", (40.0, -25.0, 10.0), "LLK", 4, 0.02),
    ("convdiff5_noth", 5, "convdiff", (30.0, 30.0, 30.0), "LLK-NOTH", 6, 0.05),
    ("convdiff5_sym", 5, "convdiff", (5.0, 5.0, 5.0), "SYM-LLK", 8, 0.05),
    ("convdiff6_stab", 6, "convdiff", (40.0, -25.0, 10.0), "STAB-LLK", 8, 0.05),
    ("convdiff4_stab_exact", 4, "convdiff", (20.0, 5.0, -15.0), "STAB-LLK", 64, 0.0),
    ("convdiff6_mlk", 6, "convdiff", (40.0, -25.0, 10.0), "MLK", 4, 0.02),
]

HAND_4x4 = [  # small nonsymmetric case worked by hand in the test
    [(0, 4.0), (1, -1.0), (3, -0.5)],
    [(0, -2.0), (1, 5.0), (2, -1.0)],
    [(1, -1.0), (2, 6.0), (3, -2.0)],
    [(0, -1.0), (2, -3.0), (3, 7.0)],
]


INV_CASES = [
    # name, grid, kind, beta, solver, params
    ("invk_poisson5_k1", 5, "poisson", (0, 0, 0), "INVK", (1, 1)),
    ("invk_convdiff5_k2", 5, "convdiff", (40.0, -25.0, 10.0), "INVK", (2, 1)),
    ("invk_convdiff4_k0", 4, "convdiff", (-15.0, 5.0, 30.0), "INVK", (0, 0)),
    ("invt_convdiff6", 6, "convdiff", (20.0, 20.0, 20.0), "INVT", (20, 0.05, 20, 0.05)),
    ("invt_poisson5_tight", 5, "poisson", (0, 0, 0), "INVT", (3, 0.01, 2, 0.02)),
    ("invt_convdiff5_cap", 5, "convdiff", (35.0, -12.0, 8.0), "INVT", (0, 0.002, 1, 0.005)),
]


def rand_rows(seed, n, density):
    """Unstructured nonsymmetric test matrix: diagonal 4 + U(-1,1), each
    off-diagonal present with probability `density`, values U(-1,1).  The
    ILUT rule that keeps the largest original upper entry only fires on
    matrices like this one, where fill can outgrow the original entries."""
    u = splitmix_uniform(seed, n * n, 0.0, 1.0)
    v = splitmix_uniform(seed + 1000, n * n, -1.0, 1.0)
    rows = []
    for i in range(n):
        e = []
        for j in range(n):
            if i == j:
                e.append((j, 4.0 + v[i * n + j]))
            elif u[i * n + j] < density:
                e.append((j, v[i * n + j]))
        rows.append(e)
    return rows


def tie_rows(seed, n, density):
    """Nonsymmetric matrix whose values come from {-1, 1, -0.5, 0.5} (diagonal
    4): equal magnitudes meet at the fill cap, where MLK's list sparsify
    (psb_hsort) and LLK's magnitude heap keep different entries."""
    u = splitmix_uniform(seed, n * n, 0.0, 1.0)
    v = splitmix_uniform(seed + 1000, n * n, 0.0, 1.0)
    vals = (-1.0, 1.0, -0.5, 0.5)
    rows = []
    for i in range(n):
        e = []
        for j in range(n):
            if i == j:
                e.append((j, 4.0))
            elif u[i * n + j] < density:
                e.append((j, vals[min(3, int(v[i * n + j] * 4))]))
        rows.append(e)
    return rows


# name, seed, n, density, alg, fill_in, thresh
TIE_CASES = [
    ("mlk_ties20", 1, 20, 0.25, "MLK", 2, 0.0),
    ("llk_ties20", 1, 20, 0.25, "LLK", 2, 0.0),
]

RAND_CASES = [
    # name, seed, n, density, solver, params
    ("invt_rand10_jmaxup", 5, 10, 0.35, "INVT", (0, 0.0, 2, 0.01)),
    ("invk_rand10", 5, 10, 0.35, "INVK", (1, 1)),
]


def save(name, rows, a, wt, z, d, extra):
    n = len(rows)
    x = splitmix_uniform(7, n)
    y0 = splitmix_uniform(8, n)
    yN = apply(wt, z, d, x, "N", 1.5, 0.5, y0)
    yT = apply(wt, z, d, x, "T", -0.75, 2.0, y0)
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        a_irp=a[0], a_ja=a[1], a_val=a[2],
        wt_irp=wt[0], wt_ja=wt[1], wt_val=wt[2],
        z_irp=z[0], z_ja=z[1], z_val=z[2], d=d,
        x=x, y0=y0, yN=yN, yT=yT, **extra)
    print(f"{name}: n={n} nnzA={len(a[1])} nnzWt={len(wt[1])} nnzZ={len(z[1])}")


def main_inverse():
    for name, idim, kind, beta, solver, p in INV_CASES:
        rows = pde3d(idim, kind, beta)
        a = rows_to_csr(rows)
        wt, z, d = inverse_build(rows, solver, p)
        save(name, rows, a, wt, z, d, dict(
            meta=np.array([idim, {"poisson": 0, "convdiff": 1}[kind], 0], np.int64),
            beta=np.array(beta, np.float64), kind=np.array(kind),
            solver=np.array(solver), params=np.array(p, np.float64)))
    for name, seed, n, dens, solver, p in RAND_CASES:
        rows = rand_rows(seed, n, dens)
        a = rows_to_csr(rows)
        wt, z, d = inverse_build(rows, solver, p)
        save(name, rows, a, wt, z, d, dict(
            meta=np.array([seed, 3, n], np.int64), beta=np.zeros(3),
            kind=np.array("rand"), density=np.array(dens),
            solver=np.array(solver), params=np.array(p, np.float64)))


def main_ties():
    for name, seed, n, dens, alg, fill, thr in TIE_CASES:
        rows = tie_rows(seed, n, dens)
        a = rows_to_csr(rows)
        wt, z, d = ainv_build(rows, alg, fill, thr)
        save(name, rows, a, wt, z, d, dict(
            meta=np.array([seed, 4, fill], np.int64), beta=np.zeros(3),
            kind=np.array("ties"), density=np.array(dens), alg=np.array(alg),
            thresh=np.array(thr)))


def main():
    main_inverse()
    main_ties()
    cases = [(c[0], pde3d(c[1], c[2], c[3]), c) for c in CASES]
    cases.append(("hand4", HAND_4x4, ("hand4", 0, "hand", (0, 0, 0), "LLK", 4, 0.0)))
    for name, rows, c in cases:
        alg, fill, thr = c[4], c[5], c[6]
        a = rows_to_csr(rows)
        wt, z, d = ainv_build(rows, alg, fill, thr)
        n = len(rows)
        x = splitmix_uniform(7, n)
        y0 = splitmix_uniform(8, n)
        yN = apply(wt, z, d, x, "N", 1.5, 0.5, y0)
        yT = apply(wt, z, d, x, "T", -0.75, 2.0, y0)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            a_irp=a[0], a_ja=a[1], a_val=a[2],
            wt_irp=wt[0], wt_ja=wt[1], wt_val=wt[2],
            z_irp=z[0], z_ja=z[1], z_val=z[2], d=d,
            x=x, y0=y0, yN=yN, yT=yT,
            meta=np.array([c[1], {"poisson": 0, "convdiff": 1, "hand": 2}[c[2]],
                           fill], np.int64),
            beta=np.array(c[3], np.float64), thresh=np.array(thr),
            alg=np.array(alg), kind=np.array(c[2]))
        print(f"{name}: n={n} nnzA={len(a[1])} nnzWt={len(wt[1])} nnzZ={len(z[1])}")


if __name__ == "__main__":
    main()

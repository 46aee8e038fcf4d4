"""Structures for neighbour-set parity (LIST, src/cell.c:82-185).

The list's only floating-point decision is the strict test r^2 < Rc^2 on the
displacement x_q = ((ic_0 L_0q + ic_1 L_1q) + ic_2 L_2q) + (X_jq - X_iq),
r^2 = ((x_0^2 + x_1^2) + x_2^2), each operation rounded (src/cell.c:115-123).
``planted_pairs`` places pairs whose r^2, evaluated in exactly that order,
is the largest double below Rc^2, Rc^2 itself and the smallest double above
it, so that a list which rounds differently, or tests <= instead of <,
disagrees with the reference.  Positions are chosen so that the wrap into
the cell is exact (cubic cells of a power-of-two edge), and pairs are
planted both inside the cell and across a periodic boundary.
"""
from __future__ import annotations

import math

import numpy as np


def r2_list_order(xi, xj, ic, L):
    """r^2 of atom j's image ic seen from atom i, rounded as LIST does."""
    r = 0.0
    for q in range(3):
        x = 0.0
        x = x + float(ic[0]) * L[0][q]
        x = x + float(ic[1]) * L[1][q]
        x = x + float(ic[2]) * L[2][q]
        x = x + (xj[q] - xi[q])
        r = r + x * x
    return r


def _tune(xi, xj, ic, L, target, rc2):
    """Move xj[2] by single ulps until r^2 hits `target` ('below': the largest
    r^2 < rc2, 'equal': r^2 == rc2, 'above': the smallest r^2 > rc2).  The
    displacement's z part is small, so one ulp of xj[2] moves r^2 by far
    less than one ulp of rc2 and every value near rc2 is reachable."""
    xj = [float(v) for v in xj]
    want = {"below": math.nextafter(rc2, 0.0), "equal": rc2, "above": math.nextafter(rc2, math.inf)}[target]
    for _ in range(200000):
        r2 = r2_list_order(xi, xj, ic, L)
        if r2 == want:
            return xj
        dz = xj[2] - xi[2] + ic[2] * L[2][2]
        grow = r2 < want
        xj[2] = math.nextafter(xj[2], math.inf if (dz >= 0) == grow else -math.inf)
    raise RuntimeError("could not plant the pair")


def planted_pairs(rc, periodic=True, filler=400, seed=0):
    """dict(X, LAT, atmn, ND, planted) with three boundary pairs (r^2 one ulp
    below Rc^2, equal, one ulp above) inside the cell and, for a periodic
    cell, three more across the x boundary; `filler` random atoms on a
    2^-20 grid keep N above the cell-list threshold.  `planted` lists
    (i, j, image of j, expected in i's list)."""
    rc2 = rc * rc
    edge = 32.0 if periodic else 64.0
    L = [[edge, 0.0, 0.0], [0.0, edge, 0.0], [0.0, 0.0, edge]]
    rng = np.random.default_rng(seed)
    X, planted = [], []
    spots = [(8.0, 8.0), (8.0, 24.0), (24.0, 8.0)] if periodic else [(40.0, 12.0), (40.0, 30.0), (40.0, 48.0)]
    for k, target in enumerate(("below", "equal", "above")):
        y, z = spots[k]
        # inside the cell: a displacement of about (5.2, 3.0, 0.05)
        xi = [10.0 + 0.37 * k, y, z]
        d = np.array([5.2, 3.0, 0.0])
        d[2] = 0.0
        d[:2] *= math.sqrt(rc2 - 0.0025) / np.linalg.norm(d[:2])
        xj = [xi[0] + d[0], xi[1] + d[1], xi[2] + 0.05]
        xj = _tune(xi, xj, (0, 0, 0), L, target, rc2)
        i = len(X)
        X += [xi, xj]
        planted.append((i, i + 1, (0, 0, 0), target == "below"))
        if periodic:
            # across the x boundary: j sits near x = edge, its image -1 is near i
            xi = [0.75 + 0.21 * k, y + 4.0, z + 4.0]
            xj = [edge - (d[0] - 0.75 - 0.21 * k), xi[1] + d[1], xi[2] + 0.05]
            xj = _tune(xi, xj, (-1, 0, 0), L, target, rc2)
            i = len(X)
            X += [xi, xj]
            planted.append((i, i + 1, (-1, 0, 0), target == "below"))
    grid = 2.0 ** -20
    lo = 14.0 if not periodic else 0.0
    while len(X) < len(planted) * 2 + filler:
        p = np.floor(rng.uniform([lo, 0, 0], [edge if periodic else 30.0, edge, edge]) / grid) * grid
        X.append([float(v) for v in p])
    X = np.array(X)
    return dict(X=X, LAT=np.array(L), atmn=np.zeros(len(X), np.int32), ND=3 if periodic else 0, planted=planted)


def skewed_cell(n_atoms, rc, seed, want_bins=3):
    """Random positions in a skewed cell (angles 60-120 deg) whose thinnest
    periodic direction holds exactly `want_bins` cell-list bins of width >= Rc
    (the smallest bin count the cell list accepts)."""
    rng = np.random.default_rng(seed)
    for _ in range(10000):
        ang = np.radians(rng.uniform(60.0, 120.0, 3))
        ca, cb, cg = np.cos(ang)
        sg = np.sin(ang[2])
        lens = rng.uniform(0.8, 1.25, 3)
        cx = lens[2] * cb
        cy = lens[2] * (ca - cb * cg) / sg
        cz2 = lens[2] ** 2 - cx * cx - cy * cy
        if cz2 <= 0.05:
            continue
        L = np.array([[lens[0], 0, 0], [lens[1] * cg, lens[1] * sg, 0], [cx, cy, np.sqrt(cz2)]])
        widths = 1.0 / np.linalg.norm(np.linalg.inv(L).T, axis=1)
        scale = want_bins * rc * (1.0 + 1e-6) / widths.min() * rng.uniform(1.0, 1.2)
        L = L * scale
        widths = widths * scale
        M = np.floor(widths / (rc * (1.0 + 1e-9)))
        if M.min() != want_bins:
            continue
        frac = rng.uniform(0, 1, (n_atoms, 3))
        return dict(X=frac @ L, LAT=L, atmn=np.zeros(n_atoms, np.int32), ND=3)
    raise RuntimeError("no skewed cell found")


def multiset(nn, nj, sh):
    """Per atom, the sorted list of (j, image) entries."""
    out = []
    for i in range(len(nn)):
        n = int(nn[i])
        rows = [(int(nj[i, t]), int(sh[i, t, 0]), int(sh[i, t, 1]), int(sh[i, t, 2])) for t in range(n)]
        out.append(sorted(rows))
    return out

"""Seeded synthetic structures for the benchmark configurations.

Each generator returns dict(X[N,3] Cartesian, LAT[3,3] rows, atmn[N], ND,
spcz) with atoms grouped by species (the reference's CAST_CELL counts
species by runs of ATMN, src/cmod.c:1090-1093).

  fcc_supercell       Cu fcc 2x2x2 conventional, a = 3.61, jitter 0.05
  random_alloy        Cu/Pd/Ag fcc 10x10x10, a = 3.8, equal fractions
  ea_population       EA-like random cells (Mg-Ca or Cu-Pd-Ag), 20 A^3/atom
                      +-15%, angles U(60,120), 2.0 A minimum distance
  fcc_particle        Au fcc sphere ~20000 atoms, 5% vacancies, 15 A vacuum
"""
from __future__ import annotations

import numpy as np

FCC = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])


def _group(X, atmn):
    order = np.argsort(atmn, kind="stable")
    return X[order], atmn[order]


def fcc_supercell(n=2, a=3.61, jitter=0.05, seed=0, species=(29,)):
    rng = np.random.default_rng(seed)
    cells = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    frac = ((FCC[None] + cells[:, None]).reshape(-1, 3)) / n
    LAT = np.eye(3) * (a * n)
    X = frac @ LAT + rng.normal(0.0, jitter, (len(frac), 3))
    atmn = np.zeros(len(X), np.int32)
    return dict(X=X, LAT=LAT, atmn=atmn, ND=3, spcz=list(species))


def random_alloy(n=10, a=3.8, seed=0, species=(29, 46, 47), jitter=0.0):
    rng = np.random.default_rng(seed)
    cells = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    frac = ((FCC[None] + cells[:, None]).reshape(-1, 3)) / n
    LAT = np.eye(3) * (a * n)
    N = len(frac)
    ns = len(species)
    atmn = np.arange(N) % ns
    rng.shuffle(atmn)
    X = frac @ LAT
    if jitter > 0:
        X = X + rng.normal(0.0, jitter, X.shape)
    X, atmn = _group(X, atmn.astype(np.int32))
    return dict(X=X, LAT=LAT, atmn=atmn, ND=3, spcz=list(species))


def lattice_from_params(a, b, c, alpha, beta, gamma):
    ca, cb, cg = np.cos(np.radians([alpha, beta, gamma]))
    sg = np.sin(np.radians(gamma))
    cx = c * cb
    cy = c * (ca - cb * cg) / sg
    cz2 = c * c - cx * cx - cy * cy
    if cz2 <= 0:
        return None
    return np.array([[a, 0, 0], [b * cg, b * sg, 0], [cx, cy, np.sqrt(cz2)]])


def _min_image_dist(L, xf_new, xf_old):
    d = xf_old - xf_new
    d -= np.round(d)
    best = np.inf
    for sh in np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], float):
        best = min(best, np.min(np.linalg.norm((d + sh) @ L, axis=1)))
    return best


def random_cell(N, rng, species_count, vol_per_atom=20.0, spread=0.15, dmin=2.0, max_tries=200, composition=None):
    """EA-style random structure (cf. RAND_CL, src/eutl.c:276-390).  Species
    are drawn at random unless `composition` gives integer ratios (N must be
    a multiple of their sum), as in an EA run at fixed stoichiometry."""
    for _ in range(max_tries):
        V = N * vol_per_atom * (1.0 + spread * rng.uniform(-1, 1))
        ang = rng.uniform(60.0, 120.0, 3)
        ratios = rng.uniform(0.75, 1.33, 3)
        L = lattice_from_params(*ratios, *ang)
        if L is None:
            continue
        vol0 = abs(np.linalg.det(L))
        if vol0 < 0.3 * np.prod(ratios):
            continue
        L = L * (V / vol0) ** (1.0 / 3.0)
        xf = np.zeros((0, 3))
        ok = True
        for _k in range(N):
            for _t in range(2000):
                cand = rng.uniform(0, 1, 3)
                if len(xf) == 0 or _min_image_dist(L, cand, xf) >= dmin:
                    xf = np.vstack([xf, cand])
                    break
            else:
                ok = False
                break
        if not ok:
            continue
        if composition is None:
            comp = rng.integers(0, species_count, N)
            if species_count > 1 and len(np.unique(comp)) < 2:
                comp[0] = (comp[0] + 1) % species_count
        else:
            unit = sum(composition)
            if N % unit:
                raise ValueError(f"{N} atoms do not fit composition {composition}")
            comp = rng.permutation(np.repeat(np.arange(len(composition)), np.asarray(composition) * (N // unit)))
        X, atmn = _group(xf @ L, comp.astype(np.int32))
        return X, L, atmn
    raise RuntimeError("could not place atoms")


def ea_population(count=256, nmin=8, nmax=64, seed=0, species=(12, 20), composition=None):
    """`count` random cells of nmin..nmax atoms (uniform); with a fixed
    `composition` the atom count is uniform over its multiples in range."""
    rng = np.random.default_rng(seed)
    out = []
    unit = sum(composition) if composition is not None else 1
    sizes = [n for n in range(nmin, nmax + 1) if n % unit == 0]
    for _ in range(count):
        if composition is None:
            N = int(rng.integers(nmin, nmax + 1))
        else:
            N = int(sizes[rng.integers(0, len(sizes))])
        X, L, atmn = random_cell(N, rng, len(species), composition=composition)
        out.append(dict(X=X, LAT=L, atmn=atmn, ND=3, spcz=list(species)))
    return out


def fcc_particle(n_target=20000, a=4.08, vacancy=0.05, jitter=0.05, pad=15.0, seed=0, species=(79,)):
    rng = np.random.default_rng(seed)
    R = (3.0 * n_target * a ** 3 / (16.0 * np.pi * (1.0 - vacancy))) ** (1.0 / 3.0)
    m = int(np.ceil(R / a)) + 1
    cells = np.array([[i, j, k] for i in range(-m, m) for j in range(-m, m) for k in range(-m, m)], float)
    pts = ((FCC[None] + cells[:, None]).reshape(-1, 3)) * a
    pts = pts[np.linalg.norm(pts, axis=1) <= R]
    keep = rng.uniform(0, 1, len(pts)) >= vacancy
    pts = pts[keep] + rng.normal(0.0, jitter, (keep.sum(), 3))
    box = 2.0 * R + 2.0 * pad
    X = pts + box / 2.0
    LAT = np.eye(3) * box
    atmn = np.zeros(len(X), np.int32)
    return dict(X=X, LAT=LAT, atmn=atmn, ND=0, spcz=list(species))

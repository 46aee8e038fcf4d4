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


_SHIFTS = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], float)


def _min_image_dist_batch(L, cands, xf_old):
    """_min_image_dist for a batch of candidates at once: [B] minimum image
    distances of cands[B, 3] (fractional) to the atoms xf_old[M, 3]."""
    d = xf_old[None, :, :] - cands[:, None, :]
    d -= np.round(d)
    v = (d[:, :, None, :] + _SHIFTS[None, None, :, :]) @ L
    return np.sqrt((v * v).sum(-1)).min(axis=(1, 2))


def _place(rng, L, xf, dmin, tries=2000, batch=64):
    """Next atom by rejection (uniform fractional candidates, minimum image
    distance >= dmin), scoring candidates in batches of 2, 4, ... up to
    `batch` (most atoms are accepted at the first candidate).  The random
    stream is consumed exactly as by one candidate at a time: after a batch
    the state is restored and only the candidates up to the accepted one are
    re-drawn.  Returns the accepted position or None."""
    if len(xf) == 0:
        return rng.uniform(0, 1, 3)
    done, size = 0, 2
    while done < tries:
        b = min(size, tries - done)
        size = min(2 * size, batch)
        saved = rng.bit_generator.state
        cands = rng.uniform(0, 1, (b, 3))
        ok = _min_image_dist_batch(L, cands, xf) >= dmin
        if ok.any():
            i = int(np.argmax(ok))
            rng.bit_generator.state = saved
            rng.uniform(0, 1, (i + 1, 3))
            return cands[i]
        done += b
    return None


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
            cand = _place(rng, L, xf, dmin)
            if cand is None:
                ok = False
                break
            xf = np.vstack([xf, cand])
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


def _population_chunk(args):
    count, seed, k, kw = args
    return ea_population(count=count, seed=[seed, k], **kw)


def ea_population_chunked(count, seed=0, chunk=256, workers=None, **kw):
    """ea_population in independent chunks: chunk k holds `chunk` structures
    drawn from the generator seeded by (seed, k), so the population depends
    on (count, seed, chunk) only, not on how many worker processes build it.
    Workers are started with `spawn` (safe next to a CUDA context)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os

    jobs = [(min(chunk, count - k * chunk), seed, k, kw) for k in range((count + chunk - 1) // chunk)]
    workers = workers or min(len(jobs), os.cpu_count() or 1)
    if workers <= 1:
        parts = [_population_chunk(j) for j in jobs]
    else:
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(_population_chunk, jobs))
    return [s for part in parts for s in part]

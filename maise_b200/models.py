"""Writers for MAISE 'model' files and random-initialised potentials.

A model file is the text format the reference reads (src/util.c:1233-1335,
src/nutl.c:502-633, src/nprs.c:75-257): a header table, the per-input range
table (minimum, maximum, 1/(maximum-minimum)), the weights in V2W order and
the appended basis.  ``write_model`` emits that layout; ``random_model``
draws N(0, 1/fan_in) weights and scales the inputs by the descriptor ranges
of a sample structure, as a trained model's range table does.
"""
from __future__ import annotations

import numpy as np

BOHR = 0.529177249  # Angstrom per bohr, the B2A unit of the basis files

_SYMBOLS = {12: "Mg", 20: "Ca", 29: "Cu", 46: "Pd", 47: "Ag", 79: "Au"}


def symbol(z: int) -> str:
    return _SYMBOLS.get(z, f"Z{z}")


# ---------------------------------------------------------------------------
# basis
# ---------------------------------------------------------------------------

def g4_table_51():
    """The 43 (eta4, zeta, lambda) index triples of the reference's 51-input
    layout (models/nn_Cu_d3_v1): eta 0-2 with zeta 0-1, eta 3-5 with zeta
    0-3, eta 6 with zeta 0-3 except the last (zeta 3, lambda +1)."""
    rows = []
    for e in range(3):
        rows += [(e, z, l) for z in range(2) for l in range(2)]
    for e in range(3, 6):
        rows += [(e, z, l) for z in range(4) for l in range(2)]
    rows += [(6, z, l) for z in range(4) for l in range(2)][:7]
    return rows


class Basis:
    """G2/G4 function table in the reference's units (Angstrom inputs)."""

    def __init__(self, rc=6.0, eta2=None, eta4=None, zetas=(1.0, 2.0, 4.0, 16.0), lambdas=(-1.0, 1.0),
                 g4_rows=None, rs=0.0):
        self.rc = float(rc)
        self.eta2 = np.asarray(eta2 if eta2 is not None else np.geomspace(0.003, 0.5, 8), float)
        self.eta4 = np.asarray(eta4 if eta4 is not None else np.geomspace(0.003, 0.03, 7), float)
        self.zetas = np.asarray(zetas, float)
        self.lambdas = np.asarray(lambdas, float)
        self.rs = float(rs)
        self.g4 = list(g4_rows if g4_rows is not None else g4_table_51())

    @property
    def ng2(self):
        return len(self.eta2)

    @property
    def ng4(self):
        return len(self.g4)

    def ncmp(self, nspc: int) -> int:
        return self.ng2 * nspc + self.ng4 * nspc * (nspc + 1) // 2

    def text(self) -> str:
        """The basis block as the reference parses it (B2A = 1 bohr)."""
        lines = ["  B2A          Scaling", f"  {BOHR:.9f}  1.0", "", "  N  GN  Rc  Rs   n1  n2  k   z   l", ""]
        n = 1
        for k in range(self.ng2):
            lines.append(f"{n:3d}   2   0   0   {k:d}   0   0   0   0")
            n += 1
        for (e, z, l) in self.g4:
            lines.append(f"{n:3d}   4   0   0   0   {e:d}   0   {z:d}   {l:d}")
            n += 1
        lines.append("")
        a2 = BOHR * BOHR

        def row(name, vals):
            return f" {name:<3s} {len(vals):2d} " + " ".join(f"{v:.12f}" for v in vals)

        lines.append(row("Rc", [self.rc / BOHR]))
        lines.append(row("Rs", [self.rs / BOHR]))
        lines.append(row("n1", list(self.eta2 * a2)))
        lines.append(row("n2", list(self.eta4 * a2)))
        lines.append(row("k", [1.0]))
        lines.append(row("z", list(self.zetas)))
        lines.append(row("l", list(self.lambdas)))
        return "\n".join(lines) + "\n"


# ---------------------------------------------------------------------------
# model file
# ---------------------------------------------------------------------------

def write_model(path, spcz, arch, nets, rmin, rmax, basis_text, model_id="B200RAND", dr=None):
    """Write a model file.

    spcz  atomic numbers per species; arch (D, h1, h2)
    nets  per species dict(W0[h1,D], b0[h1], W1[h2,h1], b1[h2], W2[h2], b2)
    rmin, rmax  per species arrays [D] of the input range table
    """
    D, h1, h2 = arch
    nspc = len(spcz)
    nw = nspc * ((D + 1) * h1 + (h1 + 1) * h2 + (h2 + 1))
    bar = "-" * 77

    def head(key, val):
        return f"|  {key:<21s}|  {val:<49s}|"

    out = [bar, "|                    neural network general information                     |", bar,
           head("model unique ID", model_id), head("number of species", str(nspc)),
           head("species types", " ".join(str(z) for z in spcz)),
           head("species names", " ".join(symbol(z) for z in spcz)),
           head("number of layers", "4"), head("architecture", f"{D} {h1} {h2} 1"),
           head("number of weights", str(nw)), head("reference", "random initialisation"), bar,
           "|                            training details                               |", bar,
           head("maise version", "maise.3.0.00"), bar,
           "|                          input component range                            |", bar,
           "        minimum                    maximum                     range"]
    for s in range(nspc):
        for n in range(D):
            lo, hi = float(rmin[s][n]), float(rmax[s][n])
            sc = float(dr[s][n]) if dr is not None else (1.0 / (hi - lo) if hi > lo else 1.0)
            out.append(f"  {lo: .16f}   {hi: .16f}   {sc: .16f}")
    out += [bar, "|                        neural network weights                             |", bar]
    for s in range(nspc):
        w = nets[s]
        vec = list(w["b0"]) + list(w["b1"]) + [float(w["b2"])]
        vec += list(np.asarray(w["W0"]).reshape(-1)) + list(np.asarray(w["W1"]).reshape(-1))
        vec += list(np.asarray(w["W2"]).reshape(-1))
        out += [f"  {v: .16f}" for v in vec]
    out.append(bar)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n" + basis_text)


def read_model(path):
    """Parse a model file in the layout write_model emits (the reference's,
    src/util.c:1233-1335 and src/nutl.c:502-633): dict(spcz, arch (D, h1, h2),
    nets, rmin, rmax, dr (the input scaling column) [nspc, D], basis_text)."""
    lines = open(path).read().split("\n")

    def field(key):
        for ln in lines:
            if ln.startswith("|") and key in ln:
                return ln.split("|")[2].strip()
        raise ValueError(f"{path}: no '{key}'")

    spcz = [int(v) for v in field("species types").split()]
    D, h1, h2 = (int(v) for v in field("architecture").split()[:3])
    nspc = len(spcz)
    k = next(i for i, ln in enumerate(lines) if "input component range" in ln) + 3
    rng = np.array([[float(v) for v in lines[k + r].split()[:3]] for r in range(nspc * D)]).reshape(nspc, D, 3)
    k = next(i for i, ln in enumerate(lines) if "neural network weights" in ln) + 2
    nper = h1 + h2 + 1 + h1 * D + h2 * h1 + h2
    V = np.array([float(lines[k + r]) for r in range(nspc * nper)])
    end = k + nspc * nper + 1
    nets = [nets_from_vector(V[s * nper:(s + 1) * nper], (D, h1, h2)) for s in range(nspc)]
    return dict(spcz=spcz, arch=(D, h1, h2), nets=nets, rmin=rng[:, :, 0], rmax=rng[:, :, 1], dr=rng[:, :, 2],
                basis_text="\n".join(lines[end:]))


def nets_from_vector(v, arch):
    """One species' network from its slice of the V2W-ordered parameter
    vector (src/nmlp.c:591-608): biases b0, b1, b2, then W0, W1, W2."""
    D, h1, h2 = arch
    v = np.asarray(v, float)
    o = 0
    b0 = v[o:o + h1]; o += h1
    b1 = v[o:o + h2]; o += h2
    b2 = float(v[o]); o += 1
    W0 = v[o:o + h1 * D].reshape(h1, D); o += h1 * D
    W1 = v[o:o + h2 * h1].reshape(h2, h1); o += h2 * h1
    W2 = v[o:o + h2].copy()
    return dict(W0=W0.copy(), b0=b0.copy(), W1=W1.copy(), b1=b1.copy(), W2=W2, b2=b2)


def vector_from_nets(nets):
    """The V2W-ordered parameter vector of all species' networks."""
    out = []
    for w in nets:
        out += list(np.asarray(w["b0"]).reshape(-1)) + list(np.asarray(w["b1"]).reshape(-1)) + [float(w["b2"])]
        out += list(np.asarray(w["W0"]).reshape(-1)) + list(np.asarray(w["W1"]).reshape(-1))
        out += list(np.asarray(w["W2"]).reshape(-1))
    return np.array(out)


def random_nets(nspc, arch, seed, binding=None, angular=0.3):
    """N(0, 1/fan_in) networks.  With binding = (ind2 offsets, ng2) the G2
    inputs get positive first-layer weights, the second layer is positive and
    the output weights negative: the atomic energy then falls monotonically
    and saturates with coordination (an embedding-like binding), so that
    together with the short-range repulsion every structure has minima to
    relax into.  G4 inputs keep random weights scaled by `angular` (larger
    values make the energy depend more on the bond angles, so that structures
    of one composition spread more in relaxed energy)."""
    D, h1, h2 = arch
    rng = np.random.default_rng(seed)
    nets = []
    for _ in range(nspc):
        W0 = rng.normal(0, 1 / np.sqrt(D), (h1, D))
        W1 = rng.normal(0, 1 / np.sqrt(h1), (h2, h1))
        W2 = rng.normal(0, 1 / np.sqrt(h2), h2)
        if binding is not None:
            offs, ng2 = binding
            W0 *= angular
            for o in offs:
                W0[:, o:o + ng2] = np.abs(rng.normal(0, 2.0 / np.sqrt(len(offs) * ng2), (h1, ng2)))
            W1 = np.abs(W1)
            W2 = -np.abs(W2)
        nets.append(dict(W0=W0, b0=rng.normal(0, 0.1, h1), W1=W1, b1=rng.normal(0, 0.1, h2), W2=W2,
                         b2=float(rng.normal(-3.0, 0.1))))
    return nets


# ---------------------------------------------------------------------------
# input ranges from a sample structure (numpy; only sets the input scaling)
# ---------------------------------------------------------------------------

def _images(X, LAT, ND, i, rc):
    L = np.asarray(LAT, float).reshape(3, 3)
    R = np.linalg.inv(L).T
    nq = [int(np.ceil(rc * np.linalg.norm(R[q]))) if q < ND else 0 for q in range(3)]
    shifts = np.array([[a, b, c] for a in range(-nq[0], nq[0] + 1) for b in range(-nq[1], nq[1] + 1)
                       for c in range(-nq[2], nq[2] + 1)], float) @ L
    d = (X[None, :, :] + shifts[:, None, :] - X[i][None, None, :]).reshape(-1, 3)
    j = np.tile(np.arange(len(X)), len(shifts))
    r = np.linalg.norm(d, axis=1)
    keep = (r < rc) & (r > 1e-12)
    return d[keep], r[keep], j[keep]


def sample_ranges(basis: Basis, X, LAT, atmn, ND, nspc, atoms_per_species=6, seed=0):
    """Per-species (min, max) of every descriptor component over a few atoms."""
    X = np.asarray(X, float).reshape(-1, 3)
    atmn = np.asarray(atmn)
    D = basis.ncmp(nspc)
    ng2, ng4 = basis.ng2, basis.ng4
    ind2 = {v: v * ng2 + (v * (v + 1) // 2) * ng4 for v in range(nspc)}
    ind4 = {}
    for b in range(nspc):
        base = ind2[b] + ng2
        ind4[(0, b)] = base
        if b > 0:
            ind4[(b, b)] = base + ng4
            for a in range(1, b):
                ind4[(a, b)] = base + (a + 1) * ng4
    rng = np.random.default_rng(seed)
    lo = np.full((nspc, D), np.inf)
    hi = np.full((nspc, D), -np.inf)
    fc = lambda r: np.where(r > basis.rc, 0.0, 0.5 * (np.cos(np.pi * r / basis.rc) + 1.0))
    for s in range(nspc):
        idx = np.flatnonzero(atmn == s)
        if len(idx) == 0:
            lo[s], hi[s] = 0.0, 1.0
            continue
        for i in rng.choice(idx, min(atoms_per_species, len(idx)), replace=False):
            d, r, j = _images(X, LAT, ND, i, basis.rc)
            rel = (atmn[j] - s) % nspc
            G = np.zeros(D)
            for v in range(nspc):
                m = rel == v
                G[ind2[v]:ind2[v] + ng2] = (fc(r[m])[:, None] * np.exp(-basis.eta2[None, :] * r[m, None] ** 2)).sum(0)
            jj, kk = np.triu_indices(len(r), 1)
            rjk = np.linalg.norm(d[jj] - d[kk], axis=1)
            ok = rjk < basis.rc
            jj, kk, rjk = jj[ok], kk[ok], rjk[ok]
            c = (d[jj] * d[kk]).sum(1) / (r[jj] * r[kk])
            A = 2 * fc(r[jj]) * fc(r[kk]) * fc(rjk)
            a, b = np.minimum(rel[jj], rel[kk]), np.maximum(rel[jj], rel[kk])
            r2 = r[jj] ** 2 + r[kk] ** 2 + rjk ** 2
            for f, (e, z, l) in enumerate(basis.g4):
                zeta, lam = basis.zetas[z], basis.lambdas[l]
                term = A * np.exp(-basis.eta4[e] * r2) * 2.0 ** (1 - zeta) * np.maximum(1 + lam * c, 0) ** zeta
                for (pa, pb), base in ind4.items():
                    G[base + f] = term[(a == pa) & (b == pb)].sum()
            lo[s] = np.minimum(lo[s], G)
            hi[s] = np.maximum(hi[s], G)
    span = np.maximum(hi - lo, 1e-3 * np.maximum(np.abs(hi), 1e-3))
    return lo - 0.25 * span, hi + 0.25 * span


def random_model(path, spcz, basis: Basis, sample, h=(10, 10), seed=1, model_id="B200RAND", binding=False,
                 angular=0.3):
    """Random-initialised model whose input ranges come from `sample` =
    (X, LAT, atmn, ND).  binding=True gives the sign structure of
    random_nets(binding=...) (used for relaxation workloads)."""
    nspc = len(spcz)
    D = basis.ncmp(nspc)
    X, LAT, atmn, ND = sample
    lo, hi = sample_ranges(basis, X, LAT, atmn, ND, nspc, seed=seed)
    offs = [v * basis.ng2 + (v * (v + 1) // 2) * basis.ng4 for v in range(nspc)]
    nets = random_nets(nspc, (D, h[0], h[1]), seed, binding=(offs, basis.ng2) if binding else None, angular=angular)
    write_model(path, spcz, (D, h[0], h[1]), nets, lo, hi, basis.text(), model_id=model_id)
    return path

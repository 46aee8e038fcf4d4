"""CPU restatement of the surrogate screen -- test infrastructure only.

Only tests/ and the bench's CPU leg import this module, as the checker of
the GPU kernels in maise_b200/csrc/cuda/mb_surrogate.cu; the product never
calls it.

* rdf_features follows RDF (src/cell.c:369-417): every atom pair i, j within
  rmax (all periodic images) with species(j) >= species(i) adds a Gaussian of
  width sigma, tapered by f(x) = cos(pi/2 * x / rmax) (Rmin = 0), to the bins
  k = o-Do .. o+Do around o = floor(r/dr), Do = floor(3 sigma/dr), x = k dr
  (cell.c:375-397); same-species histograms are halved (cell.c:399-401).  The
  pairs (m <= n) are laid out row-major over m, then n; bins are innermost.
  In place of the reference's optional unit-norm scaling (cell.c:402-415)
  each histogram is divided by the atom count, so that the features keep the
  coordination per atom that the relaxed energy depends on.
* mlp_* is the surrogate network: dense layers nin -> h1 -> h2 -> h3 -> 1 with
  SiLU after every hidden layer, squared-error loss averaged over the batch.
  Its back-propagation is the same chain rule DE_ANN_PARA (src/nmlp.c:292-354)
  applies to the potential's energy network, for a different activation.
* adam_step is Adam (Kingma and Ba, 2015, Algorithm 1); the reference trains
  with GSL minimisers (src/nmin.c) and has no Adam.
"""
from __future__ import annotations

import math

import numpy as np


def pair_index(nspc: int, m: int, n: int) -> int:
    """Row of the (m <= n) species pair in the feature layout."""
    return m * nspc - m * (m - 1) // 2 + (n - m)


def npairs(nspc: int) -> int:
    return nspc * (nspc + 1) // 2


def _image_range(L: np.ndarray, rmax: float):
    V = abs(float(np.dot(L[0], np.cross(L[1], L[2]))))
    n = []
    for a in range(3):
        b, c = L[(a + 1) % 3], L[(a + 2) % 3]
        h = V / float(np.linalg.norm(np.cross(b, c)))
        n.append(int(math.ceil(rmax / h + 0.5)))
    return n


def rdf_features(X, LAT, atmn, nspc: int, nbins: int = 128, rmax: float = 6.0, sigma: float = 0.05) -> np.ndarray:
    """Feature vector (npairs * nbins, float64) of one periodic structure."""
    X = np.asarray(X, float).reshape(-1, 3)
    L = np.asarray(LAT, float).reshape(3, 3)
    atmn = np.asarray(atmn, int)
    N = len(atmn)
    dr = rmax / nbins
    Do = int(3.0 * sigma / dr)
    DR = 0.5 / (sigma * sigma)
    Linv = np.linalg.inv(L)
    fr = X @ Linv
    n1, n2, n3 = _image_range(L, rmax)
    H = np.zeros((npairs(nspc), nbins))
    shifts = np.array([[a, b, c] for a in range(-n1, n1 + 1) for b in range(-n2, n2 + 1) for c in range(-n3, n3 + 1)],
                      float)
    for i in range(N):
        for j in range(N):
            if atmn[j] < atmn[i]:
                continue
            d = fr[j] - fr[i]
            d = d - np.round(d)
            v = (d[None, :] + shifts) @ L
            r = np.sqrt((v * v).sum(1))
            p = pair_index(nspc, atmn[i], atmn[j])
            for rr in r[(r < rmax) & (r > 0.0)]:
                o = int(rr / dr)
                for k in range(o - Do, o + Do + 1):
                    if 0 <= k < nbins:
                        x = k * dr
                        H[p, k] += math.cos(0.5 * math.pi * x / rmax) * math.exp(-(rr - x) * (rr - x) * DR)
    for m in range(nspc):
        H[pair_index(nspc, m, m)] *= 0.5
    return (H / N).reshape(-1)


# ---------------------------------------------------------------- network

def layer_shapes(nin: int, hidden):
    dims = [nin] + list(hidden) + [1]
    return [(dims[k + 1], dims[k]) for k in range(len(dims) - 1)]


def unflatten(params, nin: int, hidden):
    """[(W[out, in], b[out]) ...] views of the flat parameter vector (each
    layer's W row-major, then its b)."""
    out, o = [], 0
    for (no, ni) in layer_shapes(nin, hidden):
        W = params[o:o + no * ni].reshape(no, ni)
        o += no * ni
        b = params[o:o + no]
        o += no
        out.append((W, b))
    assert o == len(params)
    return out


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mlp_forward(params, X, nin: int, hidden):
    layers = unflatten(np.asarray(params, np.float64), nin, hidden)
    a = np.asarray(X, np.float64)
    for k, (W, b) in enumerate(layers):
        z = a @ W.T + b
        a = _silu(z) if k < len(layers) - 1 else z
    return a[:, 0]


def mlp_loss_grad(params, X, t, nin: int, hidden):
    """(loss, flat gradient) of mean((y - t)^2) over the batch."""
    params = np.asarray(params, np.float64)
    layers = unflatten(params, nin, hidden)
    acts, zs = [np.asarray(X, np.float64)], []
    for k, (W, b) in enumerate(layers):
        z = acts[-1] @ W.T + b
        zs.append(z)
        acts.append(_silu(z) if k < len(layers) - 1 else z)
    y = acts[-1][:, 0]
    B = len(y)
    loss = float(np.mean((y - t) ** 2))
    dz = (2.0 * (y - t) / B)[:, None]
    grads = []
    for k in range(len(layers) - 1, -1, -1):
        W, _ = layers[k]
        grads.append((dz.T @ acts[k], dz.sum(0)))
        if k:
            dz = (dz @ W) * _dsilu(zs[k - 1])
    flat = []
    for gW, gb in reversed(grads):
        flat += [gW.reshape(-1), gb]
    return loss, np.concatenate(flat)


def adam_step(params, grad, m, v, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns (params, m, v)."""
    m = b1 * m + (1.0 - b1) * grad
    v = b2 * v + (1.0 - b2) * grad * grad
    mh = m / (1.0 - b1 ** step)
    vh = v / (1.0 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def top_recall(pred, truth, keep_frac: float, top_frac: float = 0.10) -> float:
    """Fraction of the lowest top_frac of `truth` that the lowest keep_frac of
    `pred` keeps."""
    S = len(truth)
    ntop = max(1, int(round(top_frac * S)))
    nkeep = max(1, int(round(keep_frac * S)))
    top = set(np.argsort(truth, kind="stable")[:ntop].tolist())
    kept = set(np.argsort(pred, kind="stable")[:nkeep].tolist())
    return len(top & kept) / ntop

"""numpy restatement of MAISE's network-training objective and gradient
(TEST INFRASTRUCTURE ONLY -- the checker of maise_b200's GPU trainer).

Follows, for energy training with one output (EFS = 0, MIX = 0, O = 0):
  tot_err_gsl  src/nmin.c:93-170   RT = (sum_s w_s ((E_s - E(s))/N_s)^2 WE) / S
                                        + LREG (sum b^2 + sum W^2)
  ENE_ANN      src/nmlp.c:367-399  E(s) = sum over atoms of the network on
                                   x = (G - Rmin) DR, hidden tanh, output linear
  DE_ANN_PARA  src/nmlp.c:292-354  per structure c = 2 (E(s) - E_s) / N_s^2 WE w_s
                                   back-propagated to biases and weights
  dfunc_gsl    src/nmin.c:280-295  gradient / S + 2 LREG V
Parameters in V2W order (src/nmlp.c:591-608): per species b0[h1], b1[h2],
b2, W0[h1][D], W1[h2][h1], W2[h2].
"""
from __future__ import annotations

import numpy as np


def unpack(V, nspc, D, h1, h2):
    P = h1 + h2 + 1 + h1 * D + h2 * h1 + h2
    nets = []
    for s in range(nspc):
        v = V[s * P:(s + 1) * P]
        o = 0
        b0 = v[o:o + h1]; o += h1
        b1 = v[o:o + h2]; o += h2
        b2 = v[o]; o += 1
        W0 = v[o:o + h1 * D].reshape(h1, D); o += h1 * D
        W1 = v[o:o + h2 * h1].reshape(h2, h1); o += h2 * h1
        W2 = v[o:o + h2]
        nets.append((b0, b1, b2, W0, W1, W2))
    return nets, P


def objective(V, X, spc, nat, E_ref, weights, WE, LREG, nspc, h1, h2, grad=True):
    """(RT, gradient, predicted energies) for scaled inputs X[Na, D]."""
    V = np.asarray(V, float)
    Na, D = X.shape
    nets, P = unpack(V, nspc, D, h1, h2)
    S = len(nat)
    sat = np.repeat(np.arange(S), nat)
    Eat = np.zeros(Na)
    H1 = np.zeros((Na, h1))
    H2 = np.zeros((Na, h2))
    for s in range(nspc):
        m = spc == s
        b0, b1, b2, W0, W1, W2 = nets[s]
        H1[m] = np.tanh(X[m] @ W0.T + b0)
        H2[m] = np.tanh(H1[m] @ W1.T + b1)
        Eat[m] = H2[m] @ W2 + b2
    Es = np.bincount(sat, weights=Eat, minlength=S)
    w = np.ones(S) if weights is None else np.asarray(weights, float)
    n = np.asarray(nat, float)
    RT = WE * np.sum(w * ((E_ref - Es) / n) ** 2) / S + LREG * np.sum(V * V)
    if not grad:
        return RT, None, Es
    c = (2.0 * (Es - E_ref) / n ** 2 * WE * w)[sat]
    g = np.zeros_like(V)
    for s in range(nspc):
        m = spc == s
        b0, b1, b2, W0, W1, W2 = nets[s]
        cm = c[m]
        d1 = cm[:, None] * W2[None, :] * (1.0 - H2[m] ** 2)
        d0 = (d1 @ W1) * (1.0 - H1[m] ** 2)
        gs = np.concatenate([d0.sum(0), d1.sum(0), [cm.sum()], (d0.T @ X[m]).reshape(-1), (d1.T @ H1[m]).reshape(-1),
                             cm @ H2[m]])
        g[s * P:(s + 1) * P] = gs
    g = g / S + 2.0 * LREG * V
    return RT, g, Es

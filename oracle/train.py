"""numpy restatement of MAISE's network-training objective and gradient
(TEST INFRASTRUCTURE ONLY -- the checker of maise_b200's GPU trainer).

Follows, for training with one output (MIX = 0, O = 0):
  tot_err_gsl  src/nmin.c:93-170   RT = (sum_s w_s ((E_s - E(s))/N_s)^2 WE
                                         + WF sum_s w_s sum_i |F_i - f_i|^2) / S
                                        + LREG (sum b^2 + sum W^2)
  ENE_ANN      src/nmlp.c:367-399  E(s) = sum over atoms of the network on
                                   x = (G - Rmin) DR, hidden tanh, output linear
  DE_ANN_PARA  src/nmlp.c:292-354  per structure c = 2 (E(s) - E_s) / N_s^2 WE w_s
                                   back-propagated to biases and weights
  FRC_ANN_PARA src/nmlp.c:29-102   f_i = -sum_j sum_l Fn[i][j][l] g_j[l] over the
                                   marked atom's blocks (self block included)
  DF_ANN_PARA  src/nmlp.c:104-290  the force term's gradient, restated loop by
                                   loop per block (xn, xm as the reference names them)
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


def objective(V, X, spc, nat, E_ref, weights, WE, LREG, nspc, h1, h2, grad=True, forces=None):
    """(RT, gradient, predicted energies) for scaled inputs X[Na, D].

    forces (force training): dict with f_atom[NF], F_ref[NF, 3], blk_off[NF+1],
    blk_atom[NB], Fn[NB, D, 3] on the network's input scale and WF; the
    predicted forces are then returned in forces["f"]."""
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
    RF = 0.0
    if forces is not None:
        fr = _forces(nets, X, spc, H1, H2, sat, w, forces)
        RF = forces["WF"] * fr["RF"]
    RT = (WE * np.sum(w * ((E_ref - Es) / n) ** 2) + RF) / S + LREG * np.sum(V * V)
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
    if forces is not None:
        g += _force_gradient(nets, P, X, spc, H1, H2, fr, forces)
    g = g / S + 2.0 * LREG * V
    return RT, g, Es


def _forces(nets, X, spc, H1, H2, sat, w, fd):
    """FRC_ANN_PARA's forces on the marked atoms and sum_s w_s |F - f|^2."""
    NF = len(fd["f_atom"])
    f = np.zeros((NF, 3))
    for i in range(NF):
        for b in range(fd["blk_off"][i], fd["blk_off"][i + 1]):
            o = fd["blk_atom"][b]
            b0, b1, b2, W0, W1, W2 = nets[spc[o]]
            d1, d2 = 1.0 - H1[o] ** 2, 1.0 - H2[o] ** 2
            gx = ((W2 * d2) @ W1 * d1) @ W0  # dE_o / dx_o
            f[i] -= gx @ fd["Fn"][b]
    ws = w[sat[np.asarray(fd["f_atom"])]]
    r = f - np.asarray(fd["F_ref"])
    fd["f"] = f
    return {"f": f, "dfq": 2.0 * r * fd["WF"] * ws[:, None], "RF": float(np.sum(ws * np.sum(r * r, axis=1)))}


def _force_gradient(nets, P, X, spc, H1, H2, fr, fd):
    """DF_ANN_PARA (src/nmlp.c:171-288) for every block, in its loop structure:
    xn[n][q] = sum_l W0[n][l] Fn[l][q] dfq[q], xm[m][q] = sum_n W1[m][n] d1[n] xn[n][q],
    then the bias and weight terms of each layer with e, d = 1 - e^2 and
    c = 2 e (e^2 - 1) of the owner atom's activations."""
    nspc = len(nets)
    D = X.shape[1]
    h1, h2 = H1.shape[1], H2.shape[1]
    g = np.zeros(nspc * P)
    for i in range(len(fd["f_atom"])):
        dfq = fr["dfq"][i]
        for bk in range(fd["blk_off"][i], fd["blk_off"][i + 1]):
            o = fd["blk_atom"][bk]
            s = spc[o]
            b0, b1, b2, W0, W1, W2 = nets[s]
            Fn = fd["Fn"][bk]
            e0, e1, e2 = X[o], H1[o], H2[o]
            d1, d2 = 1.0 - e1 ** 2, 1.0 - e2 ** 2
            c1, c2 = 2.0 * e1 * (e1 ** 2 - 1.0), 2.0 * e2 * (e2 ** 2 - 1.0)
            xn = (W0 @ Fn) * dfq[None, :]            # [h1, 3]
            xm = (W1 * d1[None, :]) @ xn             # [h2, 3]
            Bp1 = np.zeros(h2)
            Bp0 = np.zeros(h1)
            Wp2 = np.zeros(h2)
            Wp1 = np.zeros((h2, h1))
            Wp0 = np.zeros((h1, D))
            for m in range(h2):
                for n in range(h1):
                    Bp1[m] -= W2[m] * c2[m] * W1[m, n] * d1[n] * xn[n].sum()
            for n in range(h1):
                for m in range(h2):
                    tn = W2[m] * d2[m] * W1[m, n] * c1[n]
                    tm = W2[m] * c2[m] * W1[m, n] * d1[n]
                    Bp0[n] -= (tn * xn[n] + tm * xm[m]).sum()
            for m in range(h2):
                Wp2[m] -= (d2[m] * W1[m, :] * d1 * xn.sum(axis=1)).sum()
            for m in range(h2):
                for n in range(h1):
                    Wp1[m, n] -= W2[m] * d2[m] * d1[n] * xn[n].sum() + W2[m] * c2[m] * e1[n] * xm[m].sum()
            for n in range(h1):
                dnl = Fn @ dfq * d1[n]               # [D]
                rnl = c1[n] * e0 * xn[n].sum()       # [D]
                for m in range(h2):
                    tmn = W2[m] * d2[m] * W1[m, n]
                    rmn = W2[m] * c2[m] * W1[m, n] * d1[n] * e0
                    Wp0[n] -= tmn * (dnl + rnl) + rmn * xm[m].sum()
            gs = np.concatenate([Bp0, Bp1, [0.0], Wp0.reshape(-1), Wp1.reshape(-1), Wp2])
            g[s * P:(s + 1) * P] += gs
    return g

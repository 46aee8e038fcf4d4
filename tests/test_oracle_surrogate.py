"""CPU checks of the surrogate oracle (oracle/surrogate.py) before it judges
the GPU kernels: finite-difference gradients, Adam's first step, and the
invariances and a known answer of the per-pair histogram."""
from __future__ import annotations

import math

import numpy as np

from oracle import surrogate as su


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, hidden = 12, (7, 5, 4)
    n = sum(o * i + o for o, i in su.layer_shapes(nin, hidden))
    p = rng.normal(0, 0.5, n)
    X = rng.normal(size=(9, nin))
    t = rng.normal(size=9)
    loss, g = su.mlp_loss_grad(p, X, t, nin, hidden)
    assert loss == np.mean((su.mlp_forward(p, X, nin, hidden) - t) ** 2)
    fd = np.zeros(n)
    for k in range(n):
        q = p.copy()
        q[k] += 1e-6
        a = np.mean((su.mlp_forward(q, X, nin, hidden) - t) ** 2)
        q[k] -= 2e-6
        b = np.mean((su.mlp_forward(q, X, nin, hidden) - t) ** 2)
        fd[k] = (a - b) / 2e-6
    np.testing.assert_allclose(g, fd, atol=1e-8)


def test_adam_first_step_moves_by_lr_times_sign():
    """With zero moments, bias correction makes the first step lr * g/(|g|+eps)."""
    g = np.array([0.3, -2.0, 1e-3, 0.0])
    p, m, v = su.adam_step(np.zeros(4), g, np.zeros(4), np.zeros(4), 1, lr=0.01)
    np.testing.assert_allclose(p, -0.01 * g / (np.abs(g) + 1e-8), rtol=1e-12)
    np.testing.assert_allclose(m, 0.1 * g)
    np.testing.assert_allclose(v, 0.001 * g * g)


def _cell(seed):
    from maise_b200 import workloads

    pop = workloads.ea_population(count=1, nmin=10, nmax=10, seed=seed, species=(29, 46, 47))
    return pop[0]


def test_histogram_is_invariant_to_translation_permutation_and_supercell():
    s = _cell(4)
    X, L, at = s["X"], s["LAT"], np.asarray(s["atmn"])
    f0 = su.rdf_features(X, L, at, 3)
    f1 = su.rdf_features(X + np.array([0.7, -1.3, 2.1]), L, at, 3)
    perm = np.random.default_rng(1).permutation(len(at))
    f2 = su.rdf_features(X[perm], L, at[perm], 3)
    X2 = np.concatenate([X, X + L[0]])
    f3 = su.rdf_features(X2, np.array([2 * L[0], L[1], L[2]]), np.concatenate([at, at]), 3)
    for f in (f1, f2, f3):
        np.testing.assert_allclose(f, f0, rtol=1e-10, atol=1e-13)
    assert f0.shape == (6 * 128,) and f0.sum() > 0


def test_histogram_dimer_known_answer():
    """Two atoms 2.5 A apart in a 20 A box: one Gaussian (halved from the two
    ordered pairs) over bins o-Do..o+Do, divided by N = 2."""
    X = np.array([[1.0, 1.0, 1.0], [3.5, 1.0, 1.0]])
    f = su.rdf_features(X, np.eye(3) * 20.0, [1, 1], 2, nbins=128, rmax=6.0, sigma=0.05)
    dr = 6.0 / 128
    o, Do = int(2.5 / dr), int(0.15 / dr)
    want = np.zeros(128)
    for k in range(o - Do, o + Do + 1):
        x = k * dr
        want[k] = math.cos(0.5 * math.pi * x / 6.0) * math.exp(-(2.5 - x) ** 2 * 0.5 / 0.05 ** 2) / 2
    H = f.reshape(3, 128)
    np.testing.assert_allclose(H[su.pair_index(2, 1, 1)], want, rtol=1e-12, atol=1e-15)
    assert not H[su.pair_index(2, 0, 0)].any() and not H[su.pair_index(2, 0, 1)].any()


def test_recall_helper():
    truth = np.arange(100.0)
    assert su.top_recall(truth, truth, 0.25) == 1.0
    assert su.top_recall(-truth, truth, 0.25) == 0.0

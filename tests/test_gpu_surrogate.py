"""GPU checks of the surrogate screen's kernels against the oracle
(oracle/surrogate.py): histogram features, loss and gradient of every
parameter, Adam steps, prediction with the fitted standardisation.
Tolerances: features 1e-5 relative (FP32 output of FP64 sums), gradient 1e-4
of its largest component (FP32 network), Adam 1e-5 relative."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import surrogate as su

pytestmark = pytest.mark.gpu


def _pop(count, seed, species=(29, 46, 47), nmin=16, nmax=48):
    from maise_b200 import workloads

    return workloads.ea_population(count=count, nmin=nmin, nmax=nmax, seed=seed, species=species)


def test_histogram_features_match_oracle():
    from maise_b200.surrogate import Surrogate

    pop = _pop(6, 1) + _pop(2, 2, nmin=4, nmax=6)
    # a skewed thin cell that needs several images per direction
    pop.append(dict(X=np.array([[0.1, 0.2, 0.3], [1.4, 1.1, 0.9]]), LAT=np.array([[2.6, 0, 0], [1.9, 2.2, 0],
                                                                                  [0.4, 0.9, 2.5]]),
                    atmn=np.array([0, 2])))
    sur = Surrogate(3)
    F = sur.features(pop)
    for k, s in enumerate(pop):
        want = su.rdf_features(s["X"], s["LAT"], s["atmn"], 3)
        np.testing.assert_allclose(F[k], want, rtol=1e-5, atol=1e-6)
    sur.close()


def test_loss_gradient_matches_oracle():
    from maise_b200.surrogate import Surrogate

    sur = Surrogate(2, nbins=40, hidden=(48, 24, 16), seed=3)
    rng = np.random.default_rng(5)
    B = 300  # more rows than one 64-row tile, a ragged last tile
    x = rng.normal(size=(B, sur.nin)).astype(np.float32)
    t = rng.normal(size=B).astype(np.float32)
    p = sur.params
    loss, g = sur.loss_grad(x, t)
    want_loss, want_g = su.mlp_loss_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64), sur.nin,
                                         sur.hidden)
    assert loss == pytest.approx(want_loss, rel=1e-5)
    scale = np.abs(want_g).max()
    np.testing.assert_allclose(g, want_g, atol=1e-4 * scale)
    sur.close()


def test_default_network_gradient_matches_oracle():
    from maise_b200.surrogate import Surrogate

    sur = Surrogate(3, seed=7)  # 768 -> 128 -> 64 -> 64 -> 1
    assert sur.nin == 768 and sur.nparams == 768 * 128 + 128 + 128 * 64 + 64 + 64 * 64 + 64 + 64 + 1
    rng = np.random.default_rng(6)
    x = rng.normal(size=(256, sur.nin)).astype(np.float32)
    t = rng.normal(size=256).astype(np.float32)
    loss, g = sur.loss_grad(x, t)
    want_loss, want_g = su.mlp_loss_grad(sur.params.astype(np.float64), x.astype(np.float64), t.astype(np.float64),
                                         sur.nin, sur.hidden)
    assert loss == pytest.approx(want_loss, rel=1e-5)
    np.testing.assert_allclose(g, want_g, atol=1e-4 * np.abs(want_g).max())
    sur.close()


def test_adam_steps_match_oracle():
    from maise_b200.surrogate import Surrogate

    sur = Surrogate(1, nbins=16, hidden=(8, 8, 4), seed=2)
    rng = np.random.default_rng(7)
    m = np.zeros(sur.nparams)
    v = np.zeros(sur.nparams)
    for step in (1, 2, 3):
        before = sur.params.astype(np.float64)
        g = rng.normal(size=sur.nparams).astype(np.float32)
        sur.adam_step(g, 1e-2)
        want, m, v = su.adam_step(before, g.astype(np.float64), m, v, step, 1e-2)
        # the update itself to 1e-4; storing the parameters in FP32 rounds
        # each by up to half an ulp (6e-8 relative)
        np.testing.assert_allclose(sur.params - before, want - before, rtol=1e-4,
                                   atol=1e-7 * (1.0 + np.abs(before)).max())
    sur.close()


def test_fit_lowers_loss_and_prediction_matches_oracle_forward():
    from maise_b200.surrogate import Surrogate

    rng = np.random.default_rng(8)
    sur = Surrogate(2, nbins=32, seed=4)
    S = 700
    feat = rng.uniform(0, 1, (S, sur.nin)).astype(np.float32)
    w = rng.normal(size=sur.nin)
    y = feat @ w / sur.nin + 0.1 * np.sin(feat[:, 0] * 6)  # a smooth target
    loss = sur.fit(feat, y, epochs=30, batch=128, lr=2e-3, seed=3)
    assert loss[-1] < 0.2 * loss[0]
    mean, istd, tm, ts = sur.norm()
    np.testing.assert_allclose(mean, feat.astype(np.float64).mean(0), rtol=1e-5, atol=1e-6)
    pred = sur.predict(feat[:50])
    xs = (feat[:50].astype(np.float64) - mean) * istd
    want = su.mlp_forward(sur.params.astype(np.float64), xs, sur.nin, sur.hidden) * ts + tm
    np.testing.assert_allclose(pred, want, rtol=1e-4, atol=1e-4 * ts)
    sur.close()


def test_screen_equals_features_then_predict():
    from maise_b200.surrogate import Surrogate

    pop = _pop(40, 9)
    sur = Surrogate(3, seed=5)
    F = sur.features(pop)
    sur.fit(F, np.linspace(-3, -2, len(pop)), epochs=3, batch=16)
    np.testing.assert_allclose(sur.screen(pop), sur.predict(F), rtol=1e-6, atol=1e-7)
    sur.close()

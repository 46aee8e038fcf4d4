"""The training oracle (oracle/train.py, a restatement of tot_err_gsl /
dfunc_gsl / DE_ANN_PARA) against central finite differences of its own
objective: the gradient the GPU trainer is checked against is itself
checked here."""
from __future__ import annotations

import numpy as np

from oracle.train import objective


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nspc, D, h1, h2 = 2, 7, 4, 3
    nat = np.array([3, 5, 2, 4])
    spc = rng.integers(0, nspc, nat.sum())
    X = rng.normal(size=(nat.sum(), D))
    P = h1 + h2 + 1 + h1 * D + h2 * h1 + h2
    V = rng.normal(0, 0.5, nspc * P)
    E = rng.normal(-3.0, 1.0, len(nat)) * nat
    w = rng.uniform(0.5, 1.5, len(nat))
    RT, g, _ = objective(V, X, spc, nat, E, w, 1.3, 1e-3, nspc, h1, h2)
    h = 1e-6
    fd = np.zeros_like(V)
    for k in range(len(V)):
        Vp, Vm = V.copy(), V.copy()
        Vp[k] += h
        Vm[k] -= h
        fd[k] = (objective(Vp, X, spc, nat, E, w, 1.3, 1e-3, nspc, h1, h2, grad=False)[0]
                 - objective(Vm, X, spc, nat, E, w, 1.3, 1e-3, nspc, h1, h2, grad=False)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-8 * np.abs(g).max())


def test_model_file_round_trip(tmp_path):
    from maise_b200 import models, workloads

    w = workloads.random_alloy(n=2, a=3.8, seed=1)
    p = str(tmp_path / "model")
    models.random_model(p, w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=3)
    m = models.read_model(p)
    assert m["arch"] == (282, 10, 10) and m["spcz"] == [29, 46, 47]
    V = models.vector_from_nets(m["nets"])
    assert len(V) == 3 * (10 + 10 + 1 + 2820 + 100 + 10)
    nets = [models.nets_from_vector(V[s * 2951:(s + 1) * 2951], m["arch"]) for s in range(3)]
    models.write_model(str(tmp_path / "again"), m["spcz"], m["arch"], nets, m["rmin"], m["rmax"], m["basis_text"],
                       dr=m["dr"])
    assert open(p).read() == open(tmp_path / "again").read()

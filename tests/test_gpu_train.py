"""GPU training of the per-species networks (mb_train_*): the objective,
its gradient and the predicted energies against the numpy restatement of
tot_err_gsl / dfunc_gsl / DE_ANN_PARA (oracle/train.py, itself checked by
finite differences), and a fit whose written model, loaded by the
evaluation path, reproduces the energies the trainer predicted."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.train import objective

pytestmark = pytest.mark.gpu

SPC = (29, 46, 47)


@pytest.fixture(scope="module")
def data(tmp_path_factory):
    import maise_b200
    from maise_b200 import models, workloads

    structs = workloads.ea_population(count=40, nmin=8, nmax=24, seed=41, species=SPC)
    big = max(structs, key=lambda s: len(s["atmn"]))
    d = tmp_path_factory.mktemp("train")
    sample = (big["X"], big["LAT"], big["atmn"], 3)
    teacher = models.random_model(str(d / "teacher"), list(SPC), models.Basis(), sample, seed=7, binding=True)
    student = models.random_model(str(d / "student"), list(SPC), models.Basis(), sample, seed=8)
    pot = maise_b200.Potential(teacher)
    E = np.array([pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300)["H"] for s in structs])
    pot.close()
    return structs, E, student, d


def test_objective_and_gradient_match_oracle(data):
    from maise_b200.train import Trainer

    structs, E, student, _ = data
    w = np.linspace(0.5, 1.5, len(structs))
    tr = Trainer(student, structs, E, weights=w, WE=1.7, LREG=1e-4)
    V = tr.initial() + np.random.default_rng(1).normal(0, 0.01, tr.nparams)
    RT, g, Ep = tr.eval(V)
    t = tr.template
    spc = np.concatenate([np.asarray(s["atmn"]) for s in structs])
    X = (tr.G - t["rmin"][spc]) * t["dr"][spc]
    nat = np.array([len(s["atmn"]) for s in structs])
    RTo, go, Eo = objective(V, X, spc, nat, E, w, 1.7, 1e-4, 3, *t["arch"][1:])
    assert RT == pytest.approx(RTo, rel=1e-12)
    np.testing.assert_allclose(Ep, Eo, rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(g, go, rtol=0, atol=1e-12 * np.abs(go).max())
    tr.close()


def test_fit_lowers_the_objective_and_the_model_file_reproduces_it(data):
    import maise_b200
    from maise_b200.train import Trainer

    structs, E, student, d = data
    tr = Trainer(student, structs, E)
    V0 = tr.initial()
    RT0, _, _ = tr.eval(V0, grad=False)
    V, RT, it = tr.fit(V0, mitr=200)
    assert RT < 0.05 * RT0, (RT0, RT, it)
    _, _, Ep = tr.eval(V, grad=False)
    path = tr.save(str(d / "trained"), V)
    tr.close()
    pot = maise_b200.Potential(path)
    Eg = np.array([pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300)["H"] for s in structs])
    pot.close()
    np.testing.assert_allclose(Eg, Ep, rtol=1e-10)

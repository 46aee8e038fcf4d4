"""GPU training of the per-species networks (mb_train_*): the objective,
its gradient, the predicted energies and forces against the numpy
restatement of tot_err_gsl / dfunc_gsl / DE_ANN_PARA / DF_ANN_PARA
(oracle/train.py, itself checked by finite differences and against the
reference's own functions), force training from the golden descriptor set
and from descriptor files the parse path writes, and a fit whose written
model, loaded by the evaluation path, reproduces the energies the trainer
predicted."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.train import objective

pytestmark = pytest.mark.gpu

SPC = (29, 46, 47)


@pytest.fixture(scope="module")
def mb_parse():
    import maise_b200

    return maise_b200


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


def golden_force_set(g, structs):
    """Marked atoms, reference forces and derivative blocks of the golden parse
    set restricted to `structs` (rows renumbered to those structures)."""
    off = g["offsets"]
    base = {s: sum(off[t + 1] - off[t] for t in structs[:k]) for k, s in enumerate(structs)}
    f_atom, F, owners, Fn, counts = [], [], [], [], []
    for k in range(len(g["mk_atom"])):
        s = int(g["mk_struct"][k])
        if s not in base:
            continue
        atom = int(g["mk_atom"][k])
        own = np.concatenate([g["mk_dni"][k], [atom]]).astype(np.int64)
        f_atom.append(base[s] + atom)
        F.append(g["mk_F"][k])
        owners.append(base[s] + own)
        Fn.append(g["mk_fn"][k])
        counts.append(len(own))
    return (np.array(f_atom), np.array(F), np.concatenate([[0], np.cumsum(counts)]), np.concatenate(owners),
            np.concatenate(Fn))


def test_force_training_matches_oracle(parse_golden, parse_model_dir):
    """Energy + force objective, gradient and predicted forces on the golden
    descriptor set (136 Cu-Ag structures, 30 marked atoms with the reference's
    own blocks and forces)."""
    from maise_b200.train import Trainer

    g = parse_golden
    structs = list(range(len(g["names"])))
    nat = np.diff(g["offsets"])
    w = np.linspace(0.6, 1.4, len(structs))
    tr = Trainer(parse_model_dir + "/model", energies=g["E"], weights=w, WE=1.1, LREG=1e-5,
                 descriptors=(g["G"], g["atmn"], nat))
    f_atom, F, boff, bown, Fn = golden_force_set(g, structs)
    tr.set_forces(f_atom, F, boff, bown, Fn, WF=0.6)
    V = tr.initial()
    RT, grad, Ep = tr.eval(V)
    fp, RF = tr.eval_forces(V)
    t = tr.template
    spc = np.asarray(g["atmn"])
    X = (g["G"] - t["rmin"][spc]) * t["dr"][spc]
    fd = dict(f_atom=f_atom, F_ref=F, blk_off=boff, blk_atom=bown, Fn=Fn * t["dr"][spc[bown]][:, :, None], WF=0.6)
    RTo, go, Eo = objective(V, X, spc, nat, g["E"], w, 1.1, 1e-5, 2, *t["arch"][1:], forces=fd)
    assert RT == pytest.approx(RTo, rel=1e-11)
    np.testing.assert_allclose(Ep, Eo, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(fp, fd["f"], rtol=1e-11, atol=1e-12 * np.abs(fd["f"]).max())
    np.testing.assert_allclose(grad, go, rtol=0, atol=1e-11 * np.abs(go).max())
    assert RF > 0.0
    tr.close()


def test_force_training_from_descriptor_files(mb_parse, parse_golden, parse_model_dir, tmp_path):
    """Descriptor files written by the parse path (mb_parse_efile, EFS 1) and
    read by Trainer.from_efiles give the objective of the same data passed
    directly; a fit lowers both the energy and the force error."""
    from maise_b200.train import Trainer

    g = parse_golden
    pot = mb_parse.Potential(parse_model_dir + "/model")
    structs = sorted(set(int(s) for s in g["mk_struct"]))[:8]
    off = g["offsets"]
    for k, s in enumerate(structs):
        a, b = off[s], off[s + 1]
        N = b - a
        marked = np.zeros(N, bool)
        F = np.zeros((N, 3))
        for m in range(len(g["mk_atom"])):
            if int(g["mk_struct"][m]) == s:
                marked[int(g["mk_atom"][m])] = True
                F[int(g["mk_atom"][m])] = g["mk_F"][m]
        pot.parse_efile(str(tmp_path), k, g["x"][a:b], g["lat"][s], g["atmn"][a:b], EFS=1, ND=3, NM=400,
                        E=float(g["E"][s]), marked=marked, frc_ref=F)
    pot.close()
    tr = Trainer.from_efiles(parse_model_dir + "/model", str(tmp_path), range(len(structs)), WE=1.0, WF=0.5)
    nat = np.array([off[s + 1] - off[s] for s in structs])
    rows = np.concatenate([np.arange(off[s], off[s + 1]) for s in structs])
    direct = Trainer(parse_model_dir + "/model", energies=g["E"][structs], WE=1.0,
                     descriptors=(g["G"][rows], g["atmn"][rows], nat))
    direct.set_forces(*golden_force_set(g, structs), WF=0.5)
    V = tr.initial()
    RT1, g1, _ = tr.eval(V)
    RT2, g2, _ = direct.eval(V)
    assert RT1 == pytest.approx(RT2, rel=1e-9)
    np.testing.assert_allclose(g1, g2, rtol=0, atol=1e-9 * np.abs(g2).max())
    _, RF0 = tr.eval_forces(V)
    V1, RT, it = tr.fit(V, mitr=60)
    _, RF1 = tr.eval_forces(V1)
    assert RT < 0.5 * RT1 and RF1 < RF0, (RT1, RT, RF0, RF1, it)
    tr.close()
    direct.close()

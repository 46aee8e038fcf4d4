"""The training oracle (oracle/train.py, a restatement of tot_err_gsl /
dfunc_gsl / DE_ANN_PARA / FRC_ANN_PARA / DF_ANN_PARA) against central finite
differences of its own objective and against the reference's own training
functions on golden descriptor files: the gradient the GPU trainer is
checked against is itself checked here."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import RefOracle, ref_available, reference_dir
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


def _force_set(rng, nspc, D, h1, h2, nat):
    """A random training set with force data: X[Na, D], species, and per
    structure one or two marked atoms whose blocks are owned by a random
    subset of the structure's other atoms and the atom itself."""
    Na = int(np.sum(nat))
    off = np.concatenate([[0], np.cumsum(nat)])
    spc = rng.integers(0, nspc, Na)
    X = rng.normal(size=(Na, D))
    f_atom, owners, counts = [], [], []
    for s, n in enumerate(nat):
        for atom in rng.choice(n, size=min(2, n), replace=False):
            others = [j for j in range(n) if j != atom]
            own = sorted(rng.choice(others, size=rng.integers(1, len(others) + 1), replace=False).tolist())
            f_atom.append(off[s] + atom)
            owners.extend(off[s] + np.array(own + [atom]))
            counts.append(len(own) + 1)
    NB = int(np.sum(counts))
    return spc, X, dict(f_atom=np.array(f_atom), F_ref=rng.normal(size=(len(f_atom), 3)),
                        blk_off=np.concatenate([[0], np.cumsum(counts)]), blk_atom=np.array(owners),
                        Fn=rng.normal(size=(NB, D, 3)), WF=0.7)


def test_oracle_force_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    nspc, D, h1, h2 = 2, 6, 4, 3
    nat = np.array([3, 4, 2])
    spc, X, fd = _force_set(rng, nspc, D, h1, h2, nat)
    P = h1 + h2 + 1 + h1 * D + h2 * h1 + h2
    V = rng.normal(0, 0.5, nspc * P)
    E = rng.normal(-3.0, 1.0, len(nat)) * nat
    w = rng.uniform(0.5, 1.5, len(nat))
    args = (X, spc, nat, E, w, 1.3, 1e-3, nspc, h1, h2)
    RT, g, _ = objective(V, *args, forces=fd)
    h = 1e-6
    num = np.zeros_like(V)
    for k in range(len(V)):
        Vp, Vm = V.copy(), V.copy()
        Vp[k] += h
        Vm[k] -= h
        num[k] = (objective(Vp, *args, grad=False, forces=fd)[0] - objective(Vm, *args, grad=False, forces=fd)[0]) / (2 * h)
    np.testing.assert_allclose(g, num, rtol=1e-6, atol=1e-8 * np.abs(g).max())
    # the force term is there: without it the objective changes
    assert objective(V, *args, grad=False)[0] < RT


@pytest.mark.skipif(reference_dir() is None or not ref_available(), reason="reference sources or build absent")
def test_oracle_force_terms_match_the_reference(parse_golden):
    """The reference's own LNK_IN + ADJT_LNK + FRC_ANN_PARA + DE_ANN_PARA +
    DF_ANN_PARA on golden descriptor files with marked atoms, against the
    oracle on the same files read by the product's reader."""
    from maise_b200.efile import read_efile

    directory = os.path.join(reference_dir(), "test", "parse", "ref")
    rng = np.random.default_rng(11)
    nspc, D, h1, h2 = 2, 82, 6, 5
    P = h1 + h2 + 1 + h1 * D + h2 * h1 + h2
    V = rng.normal(0, 0.3, nspc * P)
    names = parse_golden["names"]
    structs = sorted(set(int(s) for s in parse_golden["mk_struct"]))[:5]
    for s in structs:
        idx = int(str(names[s])[1:])
        f = read_efile(directory, idx)
        assert f["EFS"] == 1 and f["D"] == D
        rmin = np.zeros((nspc, D))
        dr = 1.0 / (np.abs(parse_golden["G"]).max(axis=0) + 1.0)[None, :].repeat(nspc, 0)
        X = (f["G"] - rmin[f["atmn"]]) * dr[f["atmn"]]
        counts = [len(o) for _, o, _ in f["blocks"]]
        fd = dict(f_atom=np.array([a for a, _, _ in f["blocks"]]), F_ref=f["F"],
                  blk_off=np.concatenate([[0], np.cumsum(counts)]), blk_atom=np.concatenate([o for _, o, _ in f["blocks"]]),
                  Fn=np.concatenate([fn * dr[f["atmn"][o]][:, :, None] for _, o, fn in f["blocks"]]), WF=0.8)
        w = 0.9
        RT, g, Es = objective(V, X, f["atmn"], np.array([f["N"]]), np.array([f["E"]]), np.array([w]), 1.2, 0.0, nspc,
                              h1, h2, forces=fd)
        E, fr, gE, gF = RefOracle.train_terms(directory, idx, V, nspc, D, h1, h2, rmin, dr, WE=1.2, WF=0.8, w=w)
        assert Es[0] == pytest.approx(E, rel=1e-12)
        np.testing.assert_allclose(fd["f"], fr[fd["f_atom"]], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(g, gE + gF, rtol=1e-9, atol=1e-11 * np.abs(g).max())
        assert np.abs(gF).max() > 1e-3 * np.abs(gE).max()  # the force term is not negligible here

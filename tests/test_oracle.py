"""The CPU oracle (C restatement) pinned against the reference: its golden
descriptor and derivative vectors (test/parse/ref), the interface
known-answer test, relax fixtures, and live runs of the reference sources
compiled under oracle/_ref when present."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, parse_structures, write_model_dir
from oracle import Oracle, RefOracle, ref_available

# printed precision of the e-files is 16 decimals; our sums differ in order only
G_RTOL, G_ATOL = 1e-12, 1e-13


def test_oracle_descriptors_match_golden_parse_files(parse_golden, parse_model_dir):
    o = Oracle(parse_model_dir + "/model")
    assert o.D == 82 and o.ng2 == 8 and o.ng4 == 22
    worst = 0.0
    for s, LAT, X, atmn, Gref in parse_structures(parse_golden):
        G = o.descriptors(X, LAT, atmn, 3, NM=400)
        err = np.abs(G - Gref) / (G_ATOL + G_RTOL * np.abs(Gref))
        worst = max(worst, err.max())
    assert worst <= 1.0, worst


def test_oracle_derivative_blocks_match_golden(parse_golden, parse_model_dir):
    o = Oracle(parse_model_dir + "/model")
    off = parse_golden["offsets"]
    n = 0
    for k in range(len(parse_golden["mk_atom"])):
        s = int(parse_golden["mk_struct"][k])
        atom = int(parse_golden["mk_atom"][k])
        a, b = off[s], off[s + 1]
        dni, Fn, _ = o.fn(parse_golden["x"][a:b], parse_golden["lat"][s], parse_golden["atmn"][a:b], 3, atom, NM=400)
        assert (dni == parse_golden["mk_dni"][k]).all()
        ref = parse_golden["mk_fn"][k]
        np.testing.assert_allclose(Fn, ref, rtol=1e-11, atol=1e-13)
        n += 1
    assert n >= 20


def test_oracle_interface_known_answer(tmp_path):
    g = load_golden("kat_interface.npz")
    d = write_model_dir(tmp_path, g["model"])
    o = Oracle(d + "/model")
    r = o.efs(g["X"], g["LAT"], g["atmn"], 0, NM=int(g["NM"]))
    assert r["H"] == pytest.approx(float(g["outcar_H"]), abs=5e-9)
    np.testing.assert_allclose(np.abs(r["F"]).max(), float(g["outcar_F"]), atol=5e-7)
    np.testing.assert_allclose(r["EA"], float(g["outcar_EA"]), atol=5e-13)
    # full-precision pins from the compiled reference
    assert r["H"] == pytest.approx(float(g["ref_H"]), rel=1e-13)
    np.testing.assert_allclose(r["F"], g["ref_F"], atol=1e-12)
    np.testing.assert_allclose(r["U"], g["ref_U"], rtol=1e-12, atol=1e-12)


def test_oracle_virial_known_answer_per_volume(tmp_path):
    """OUTCAR prints U/V with the particle volume of NP_VOL (src/nutl.c:846-898)."""
    g = load_golden("kat_interface.npz")
    d = write_model_dir(tmp_path, g["model"])
    o = Oracle(d + "/model")
    r = o.efs(g["X"], g["LAT"], g["atmn"], 0, NM=int(g["NM"]))
    X = g["X"]
    m = 63.546
    M = m * len(X)
    c = X.sum(0) * m / M
    I = np.zeros((3, 3))
    for x in X - c:
        I += m * (np.dot(x, x) * np.eye(3) - np.outer(x, x))
    vol = 4.0 * np.pi / 3.0 * (2.5 / M) ** 1.5 * np.sqrt(np.prod(np.linalg.eigvalsh(I)))
    assert r["U"][0] / vol == pytest.approx(float(g["outcar_UV"]), abs=5e-9)
    assert r["U"][1] / vol == pytest.approx(float(g["outcar_UV"]), abs=5e-9)


@pytest.mark.parametrize("case", range(5))
def test_oracle_matches_reference_vectors(tmp_path, case):
    c = load_golden("ref_efs.npz")["cases"][case]
    d = write_model_dir(tmp_path, c["model"])
    o = Oracle(d + "/model")
    r = o.efs(c["X"], c["LAT"], c["atmn"], c["ND"], urep=c["urep"], p_gpa=c["p"], NM=400)
    assert r["H"] == pytest.approx(c["H"], rel=1e-13, abs=1e-12)
    np.testing.assert_allclose(r["EA"], c["EA"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(r["F"], c["F"], atol=1e-11)
    np.testing.assert_allclose(r["U"], c["U"], rtol=1e-12, atol=1e-10)
    G = o.descriptors(c["X"], c["LAT"], c["atmn"], c["ND"], NM=400)
    np.testing.assert_allclose(G, c["G"], rtol=1e-13, atol=1e-14)


def test_oracle_forces_are_energy_gradient(tmp_path):
    """CELL_TEST-style central differences (src/cmod.c:981-1027)."""
    c = load_golden("ref_efs.npz")["cases"][2]
    d = write_model_dir(tmp_path, c["model"])
    o = Oracle(d + "/model")
    X = np.array(c["X"], float)
    r = o.efs(X, c["LAT"], c["atmn"], 3, NM=400)
    h = 1e-5
    for i, q in [(0, 0), (5, 1), (17, 2), (31, 0)]:
        Xp, Xm = X.copy(), X.copy()
        Xp[i, q] += h
        Xm[i, q] -= h
        Ep = o.efs(Xp, c["LAT"], c["atmn"], 3, forces=False, NM=400)["E"]
        Em = o.efs(Xm, c["LAT"], c["atmn"], 3, forces=False, NM=400)["E"]
        assert -(Ep - Em) / (2 * h) == pytest.approx(r["F"][i, q], abs=1e-6)


def test_oracle_virial_is_strain_derivative(tmp_path):
    """U_ab = -dE/d(eps_ab) under homogeneous strain of cell and atoms."""
    c = load_golden("ref_efs.npz")["cases"][1]
    d = write_model_dir(tmp_path, c["model"])
    o = Oracle(d + "/model")
    X, L = np.array(c["X"], float), np.array(c["LAT"], float)
    r = o.efs(X, L, c["atmn"], 3, NM=400)
    h = 1e-6
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]
    for k, (a, b) in enumerate(pairs):
        e = np.zeros((3, 3))
        e[a, b] = e[b, a] = h if a != b else h
        if a != b:
            e[a, b] = e[b, a] = h / 2
        Es = []
        for sgn in (1, -1):
            T = np.eye(3) + sgn * e
            Es.append(o.efs(X @ T, L @ T, c["atmn"], 3, forces=False, NM=400)["E"])
        dE = (Es[0] - Es[1]) / (2 * h)
        assert -dE == pytest.approx(r["U"][k], rel=1e-5, abs=1e-5)


needs_ref = pytest.mark.skipif(not ref_available(), reason="reference sources were not compiled here")


@needs_ref
def test_restatement_equals_compiled_reference_on_random_cells(tmp_path):
    from maise_b200 import models, workloads

    rng = np.random.default_rng(3)
    for k in range(3):
        X, L, at = workloads.random_cell(12 + 6 * k, rng, 3)
        d = tmp_path / f"m{k}"
        d.mkdir()
        models.random_model(str(d / "model"), [29, 46, 47], models.Basis(), (X, L, at, 3), seed=k)
        o = Oracle(str(d / "model"))
        r = RefOracle(str(d), 1)
        a = o.efs(X, L, at, 3, urep=100.0, p_gpa=1.5, NM=400)
        b = r.efs(X, L, at, 3, urep=100.0, p_gpa=1.5, NM=400)
        assert a["H"] == pytest.approx(b["H"], rel=1e-13)
        np.testing.assert_allclose(a["F"], b["F"], atol=1e-11)
        np.testing.assert_allclose(a["U"], b["U"], rtol=1e-12, atol=1e-10)
        np.testing.assert_array_equal(a["X"], b["X"])


@needs_ref
def test_reference_relax_over_project_bfgs_reproduces_gsl_fixtures():
    g = load_golden("relax.npz")
    assert float(g["cu3pd_ref_H"]) == pytest.approx(float(g["cu3pd_gsl_H"]), abs=1e-8)
    assert float(g["cu3pd_ref_lat"][0, 0]) == pytest.approx(float(g["cu3pd_gsl_a"]), abs=2e-4)
    assert float(g["cu4_ref_H"]) == pytest.approx(float(g["cu4_gsl_H"]), abs=1e-9)

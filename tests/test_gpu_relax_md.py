"""GPU relaxation and NVT molecular dynamics against the reference's fixtures
and the compiled reference (oracle/_ref) through the C-ABI."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, write_model_dir
from oracle import RefOracle, ref_available

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref was not built")


@pytest.fixture(scope="module")
def mb():
    import maise_b200

    return maise_b200


@pytest.mark.parametrize("key", ["cu3pd", "cu4"])
def test_relax_reproduces_reference_fixtures(mb, tmp_path, key):
    """test/relax (Cu3Pd) and examples/03-rlx (Cu4): full-cell BFGS, ETOL 1e-6."""
    g = load_golden("relax.npz")
    d = write_model_dir(tmp_path, g[key + "_model"])
    pot = mb.Potential(d + "/model")
    r = pot.relax(g[key + "_x"], g[key + "_lat"], g[key + "_atmn"], ND=3, NM=300, rlxt=3, mitr=100, etol=1e-6)
    # GSL-produced values printed in the reference's files
    assert r["H"] == pytest.approx(float(g[key + "_gsl_H"]), abs=2e-8)
    # the compiled reference relaxed by the same BFGS restatement
    assert r["H"] == pytest.approx(float(g[key + "_ref_H"]), abs=1e-9)
    np.testing.assert_allclose(r["LAT"], g[key + "_ref_lat"], atol=1e-5)
    if key == "cu3pd":
        assert r["LAT"][0, 0] == pytest.approx(float(g["cu3pd_gsl_a"]), abs=2e-4)
        assert r["iters"] <= 10


@needs_ref
def test_relax_random_cell_matches_reference_relax(mb, tmp_path):
    from maise_b200 import models, workloads

    rng = np.random.default_rng(21)
    X, L, at = workloads.random_cell(10, rng, 2)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), [12, 20], models.Basis(), (X, L, at, 3), seed=4)
    pot = mb.Potential(str(d / "model"))
    # This relax is still far from a minimum after many steps, and past about
    # 30 BFGS iterations its path is chaotic: the reference itself moves by
    # 1e-6 .. 1e-3 eV when the start is shifted by 1e-12 A.  Over the first
    # 20 iterations that spread is 2e-9 eV, so the paths are compared there.
    r = pot.relax(X, L, at, ND=3, NM=300, rlxt=3, mitr=20, etol=1e-7, urep=100.0)
    ref = RefOracle(str(d), 1).relax(X, L, at, 3, rlxt=3, mitr=20, etol=1e-7, urep=100.0, NM=300)
    assert r["H"] == pytest.approx(ref["H"], abs=1e-6)
    np.testing.assert_allclose(r["LAT"], ref["LAT"], atol=1e-6)
    longer = pot.relax(X, L, at, ND=3, NM=300, rlxt=3, mitr=60, etol=1e-7, urep=100.0)
    assert longer["H"] < r["H"] < pot.energy(X, L, at, ND=3, NM=300, urep=100.0)["H"]


@needs_ref
@pytest.mark.parametrize("species", [(29,), (29, 46, 47)])
def test_nvt_trajectory_matches_reference(mb, tmp_path, species):
    from maise_b200 import atomic_mass, maxwell, models, workloads

    w = workloads.random_alloy(n=3, a=3.7, seed=5, species=species, jitter=0.05)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=6)
    V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=99)
    steps = 20
    ref = RefOracle(str(d), 1).nvt(w["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, steps, V=V, NM=300)
    pot = mb.Potential(str(d / "model"))
    g = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 600.0, dt=1.0, tau=25.0, nsteps=steps, NM=300)
    np.testing.assert_allclose(g["H"], ref["H"], rtol=1e-11, atol=1e-10)
    np.testing.assert_allclose(g["K"], ref["K"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(g["X"], ref["X"], atol=1e-9)
    np.testing.assert_allclose(g["V"], ref["V"], atol=1e-11)
    assert g["xi"] == pytest.approx(ref["xi"], rel=1e-9, abs=1e-14)


@needs_ref
def test_nvt_full_size_matches_reference(mb, tmp_path):
    """4000-atom Cu-Pd-Ag at 600 K: the first NVT steps equal the reference's
    CELL_FRC + NVT update (the integrator is first order in v, as in
    src/cmod.c:440-450, so H + K is not a conserved quantity to test)."""
    import os

    from maise_b200 import atomic_mass, maxwell, models, workloads

    w = workloads.random_alloy(n=10, a=3.8, seed=0)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=1)
    V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=3)
    ref = RefOracle(str(d), os.cpu_count() or 1).nvt(w["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, 3, V=V,
                                                     NM=100)
    pot = mb.Potential(str(d / "model"))
    g = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 600.0, dt=1.0, tau=25.0, nsteps=3, NM=100)
    np.testing.assert_allclose(g["H"], ref["H"], rtol=1e-11)
    np.testing.assert_allclose(g["K"], ref["K"], rtol=1e-11)
    np.testing.assert_allclose(g["X"], ref["X"], atol=1e-10)
    np.testing.assert_allclose(g["V"], ref["V"], atol=1e-12)


def test_md_results_independent_of_chunking(mb, tmp_path):
    """Two runs of 7 then 8 steps equal one run of 15 (state carried through x, v, xi)."""
    from maise_b200 import atomic_mass, maxwell, models, workloads

    w = workloads.fcc_supercell(n=2, seed=8)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=2)
    pot = mb.Potential(str(d / "model"))
    V = maxwell([atomic_mass(29)] * 32, 900.0, seed=4)
    a = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 900.0, nsteps=15, NM=200)
    b1 = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 900.0, nsteps=7, NM=200)
    b2 = pot.md_nvt(b1["X"], w["LAT"], w["atmn"], b1["V"], 900.0, nsteps=8, NM=200, xi=b1["xi"])
    np.testing.assert_allclose(b2["X"], a["X"], atol=1e-12)
    np.testing.assert_allclose(b2["H"], a["H"][7:], rtol=1e-13)


@pytest.mark.parametrize("size", [2, 5])
def test_md_graph_replay_equals_plain_launches(mb, tmp_path, size, monkeypatch):
    """The NVT loop replayed as captured CUDA graphs (chunks of 10 steps, a
    shorter last chunk, a second call reusing the graph) gives the trajectory
    of plain launches; 32 atoms take the all-pairs list, 500 the cell list.
    Both handles run one fixed kernel variant, so that their launch counts
    compare (each handle's autotuner could otherwise pick another family)."""
    from maise_b200 import atomic_mass, maxwell, models, workloads

    monkeypatch.setenv("MAISE_B200_SHAPE", "6")

    w = workloads.random_alloy(n=size, a=3.8, seed=9, species=(29, 46), jitter=0.05)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=2)
    N = len(w["atmn"])
    V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=3)
    runs = []
    for graphs in (False, True):
        pot = mb.Potential(str(d / "model"))
        pot.graphs(graphs)
        a = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 600.0, nsteps=23, NM=200)
        b = pot.md_nvt(a["X"], w["LAT"], w["atmn"], a["V"], 600.0, nsteps=20, NM=200, xi=a["xi"])
        runs.append((a, b, pot.launches))
        pot.close()
    (a0, b0, n0), (a1, b1, n1) = runs
    for r0, r1 in ((a0, a1), (b0, b1)):
        np.testing.assert_allclose(r1["X"], r0["X"], atol=1e-9)
        np.testing.assert_allclose(r1["V"], r0["V"], atol=1e-9)
        np.testing.assert_allclose(r1["H"], r0["H"], rtol=1e-11, atol=1e-9 * N)
        assert r1["xi"] == pytest.approx(r0["xi"], rel=1e-9, abs=1e-12)
    assert n1 == n0  # the replays count the launches they contain


def test_relax_with_replayed_passes_equals_plain_launches(mb, tmp_path):
    """A cell relaxation whose evaluations replay the captured pass graphs
    (energy and energy+force passes alternate; the cell is re-pointed at each
    call) follows the plain-launch path."""
    from maise_b200 import models, workloads

    rng = np.random.default_rng(21)
    X, L, at = workloads.random_cell(10, rng, 2)
    d = tmp_path / "m"
    d.mkdir()
    models.random_model(str(d / "model"), [12, 20], models.Basis(), (X, L, at, 3), seed=4)
    res = []
    for graphs in (False, True):
        pot = mb.Potential(str(d / "model"))
        pot.graphs(graphs)
        res.append(pot.relax(X, L, at, ND=3, NM=300, rlxt=3, mitr=20, etol=1e-7, urep=100.0))
        pot.close()
    assert res[1]["H"] == pytest.approx(res[0]["H"], abs=1e-8)
    np.testing.assert_allclose(res[1]["LAT"], res[0]["LAT"], atol=1e-8)

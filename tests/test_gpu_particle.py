"""The large 0D particle (Au fcc sphere of ~20000 atoms, a = 4.08 A, 5%
vacancies, 0.05 A jitter, 15 A of vacuum padding; one-element 51-10-10-1
model) through the one-structure FP64 path at full size: E/F/S against the
compiled reference (oracle/_ref), the properties of an isolated cluster, and
NVT at 300 K.  ND = 0 with more than 64 atoms takes the cell-list neighbour
build without periodic images."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import RefOracle, ref_available

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref was not built")

NM = 100
E_RTOL = 1e-10
F_ATOL = 1e-9


@pytest.fixture(scope="module")
def particle(tmp_path_factory):
    from maise_b200 import models, workloads

    w = workloads.fcc_particle(seed=0)
    d = tmp_path_factory.mktemp("au")
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 0), seed=1)
    return w, str(d)


@pytest.fixture(scope="module")
def pot(particle):
    import maise_b200

    p = maise_b200.Potential(particle[1] + "/model")
    yield p
    p.close()


@needs_ref
def test_efs_matches_reference_at_full_size(particle, pot):
    w, d = particle
    assert len(w["atmn"]) > 19000
    ref = RefOracle(d, os.cpu_count() or 1).efs(w["X"], w["LAT"], w["atmn"], 0, NM=NM)
    r = pot.efs(w["X"], w["LAT"], w["atmn"], ND=0, NM=NM)
    assert r["H"] == pytest.approx(ref["H"], rel=E_RTOL)
    assert r["E"] == pytest.approx(ref["E"], rel=E_RTOL)
    np.testing.assert_allclose(r["EA"], ref["EA"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(r["F"], ref["F"], atol=F_ATOL)
    np.testing.assert_allclose(r["U"], ref["U"], rtol=E_RTOL, atol=1e-8)
    np.testing.assert_array_equal(r["X"], ref["X"])


def test_isolated_cluster_invariants(particle, pot):
    """No periodic images: forces and torques sum to zero, the virial is
    sum_i x_i (x) F_i (order xx, yy, zz, xy, yz, zx), and a rigid rotation
    about the box centre leaves the energy unchanged and rotates the forces."""
    w, _ = particle
    X = np.asarray(w["X"], float)
    r = pot.efs(X, w["LAT"], w["atmn"], ND=0, NM=NM)
    F = r["F"]
    c = X.mean(0)
    scale = np.abs(F).max()
    assert np.abs(F.sum(0)).max() < 1e-10 * len(X) * scale
    assert np.abs(np.cross(X - c, F).sum(0)).max() < 1e-9 * len(X) * scale
    W = np.einsum("ia,ib->ab", X - c, F)
    xf = np.array([W[0, 0], W[1, 1], W[2, 2], W[0, 1], W[1, 2], W[2, 0]])
    np.testing.assert_allclose(r["U"], xf, rtol=1e-9, atol=1e-7)

    th = 0.37
    Rz = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
    Rx = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(0.81), -np.sin(0.81)], [0.0, np.sin(0.81), np.cos(0.81)]])
    Rm = Rx @ Rz
    box = np.diag(w["LAT"]) / 2.0
    Xr = box + (X - box) @ Rm.T
    rr = pot.efs(Xr, w["LAT"], w["atmn"], ND=0, NM=NM)
    assert rr["E"] == pytest.approx(r["E"], rel=E_RTOL)
    np.testing.assert_allclose(rr["F"], F @ Rm.T, atol=F_ATOL)


def test_forces_are_energy_gradients(particle, pot):
    """Central differences of the energy on sampled atoms, from the per-atom
    energies (the change is local, so the difference is taken atom by atom
    and does not lose digits to the 20000-term total)."""
    w, _ = particle
    X = np.asarray(w["X"], float)
    r = pot.efs(X, w["LAT"], w["atmn"], ND=0, NM=NM)
    h = 1e-4
    surface = int(np.argmax(np.linalg.norm(X - X.mean(0), axis=1)))
    for i, q in [(0, 0), (len(X) // 2, 1), (surface, 2)]:
        Xp, Xm = X.copy(), X.copy()
        Xp[i, q] += h
        Xm[i, q] -= h
        Ep = pot.energy(Xp, w["LAT"], w["atmn"], ND=0, NM=NM)["EA"]
        Em = pot.energy(Xm, w["LAT"], w["atmn"], ND=0, NM=NM)["EA"]
        assert -np.sum(Ep - Em) / (2 * h) == pytest.approx(r["F"][i, q], abs=1e-6)


@needs_ref
def test_nvt_first_steps_match_reference(particle, pot):
    """Two NVT steps at 300 K from the reference's Maxwell velocities equal the
    reference's CELL_FRC + NVT update."""
    from maise_b200 import atomic_mass, maxwell

    w, d = particle
    V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 300.0, seed=5)
    ref = RefOracle(d, os.cpu_count() or 1).nvt(w["X"], w["LAT"], w["atmn"], 0, 300.0, 1.0, 25.0, 2, V=V, NM=NM)
    g = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 300.0, dt=1.0, tau=25.0, nsteps=2, ND=0, NM=NM)
    np.testing.assert_allclose(g["H"], ref["H"], rtol=1e-11)
    np.testing.assert_allclose(g["K"], ref["K"], rtol=1e-11)
    np.testing.assert_allclose(g["X"], ref["X"], atol=1e-10)
    np.testing.assert_allclose(g["V"], ref["V"], atol=1e-12)


def test_nvt_500_steps(particle, pot):
    """The configured run: 500 NVT steps at 300 K.  Total momentum starts at
    zero (Maxwell removes it) and stays zero, since the forces of an isolated
    cluster sum to zero and the thermostat scales every velocity alike; the
    run is the same in one call or in two calls that carry xi (to rounding:
    500 steps of a chaotic trajectory amplify last-bit differences)."""
    from maise_b200 import atomic_mass, maxwell

    w, _ = particle
    m = np.array([atomic_mass(w["spcz"][s]) for s in w["atmn"]])
    V = maxwell(m, 300.0, seed=5)
    a = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 300.0, nsteps=500, ND=0, NM=NM)
    assert np.isfinite(a["X"]).all() and np.isfinite(a["H"]).all()
    p0 = np.abs((m[:, None] * V).sum(0)).max()
    p = np.abs((m[:, None] * a["V"]).sum(0)).max()
    assert p < 1e-9 * np.abs(m[:, None] * a["V"]).sum() + p0
    assert 0.1 < a["K"][-1] / a["K"][0] < 10.0
    b = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 300.0, nsteps=250, ND=0, NM=NM)
    b = pot.md_nvt(b["X"], w["LAT"], w["atmn"], b["V"], 300.0, nsteps=250, ND=0, NM=NM, xi=b["xi"])
    np.testing.assert_allclose(b["X"], a["X"], atol=1e-9)
    np.testing.assert_allclose(b["V"], a["V"], atol=1e-11)
    np.testing.assert_allclose(b["H"], a["H"][250:], rtol=1e-12)

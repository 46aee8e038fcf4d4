"""The persistent population relax (mb_relax_batch: FP32 descriptors and MLP,
FP64 reductions and BFGS) against the FP64 one-structure path.  The bar is
1e-5 eV/atom for energies and minima that the FP64 path accepts as minima."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EV_ATOM = 1e-5
FMAX = 0.01
UREP = 100.0


@pytest.fixture(scope="module")
def mgca(tmp_path_factory):
    import maise_b200
    from maise_b200 import models, workloads

    pop = workloads.ea_population(count=40, seed=3)
    big = max(pop, key=lambda s: len(s["atmn"]))
    d = tmp_path_factory.mktemp("mgca")
    models.random_model(str(d / "model"), [12, 20], models.Basis(), (big["X"], big["LAT"], big["atmn"], 3), seed=5,
                        binding=True)
    return maise_b200.Potential(str(d / "model")), pop


def _nat(pop):
    return np.array([len(s["atmn"]) for s in pop])


@pytest.fixture(params=[("12", "1"), ("4", "1"), ("12", "2"), ("12", "4")],
                ids=["12warps", "4warps", "12warps-cluster2", "12warps-cluster4"])
def width(request, monkeypatch):
    """Warps per CTA and CTAs per structure (a thread-block cluster sharing
    the structure's evaluations) of the batched kernel.  The library reads
    MAISE_B200_BATCH_WARPS and MAISE_B200_BATCH_CLUSTER at every launch; by
    default it uses 12 warps, with clusters of 4 for populations of at most
    two structures per SM."""
    monkeypatch.setenv("MAISE_B200_BATCH_WARPS", request.param[0])
    monkeypatch.setenv("MAISE_B200_BATCH_CLUSTER", request.param[1])
    return request.param


def test_fp32_energy_of_start_structures_matches_fp64(mgca, width):
    """With no iterations the batched path reports each structure's enthalpy
    from its FP32 evaluation: within 1e-5 eV/atom of the FP64 path, for
    every CTA width and cluster size."""
    pot, pop = mgca
    r = pot.relax_batch(pop, urep=UREP, rlxt=3, mitr=0, fmax=FMAX)
    for k, s in enumerate(pop):
        h64 = pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=UREP)["H"]
        assert abs(r["H"][k] - h64) / len(s["atmn"]) < EV_ATOM
        np.testing.assert_allclose(r["X"][k], s["X"], atol=1e-12)


@pytest.mark.parametrize("rlxt", [2, 3])
def test_batched_minima_are_fp64_minima(mgca, rlxt, width):
    pot, pop = mgca
    r = pot.relax_batch(pop, urep=UREP, rlxt=rlxt, mitr=1000, fmax=FMAX)
    conv = np.flatnonzero(r["status"] == 0)
    assert len(conv) >= 0.6 * len(pop)
    nat = _nat(pop)
    for k in conv:
        e = pot.efs(r["X"][k], r["LAT"][k], pop[k]["atmn"], ND=3, NM=300, urep=UREP)
        assert abs(r["H"][k] - e["H"]) / nat[k] < EV_ATOM
        assert np.abs(e["F"]).max() < FMAX + 2e-3
        assert r["H"][k] < pot.energy(pop[k]["X"], pop[k]["LAT"], pop[k]["atmn"], ND=3, NM=300, urep=UREP)["H"]
        if rlxt == 2:
            np.testing.assert_allclose(r["LAT"][k], pop[k]["LAT"], atol=1e-12)


@pytest.mark.parametrize("sigma", ["0.1", "0.5"])
def test_line_search_constant(mgca, sigma, monkeypatch):
    """The batched line search's strong Wolfe curvature constant (0.5 by
    default; 0.1 is the reference's): either one reaches minima the FP64
    path accepts, and the looser one takes fewer evaluations per iteration."""
    pot, pop = mgca
    nat = _nat(pop)
    monkeypatch.setenv("MAISE_B200_BATCH_SIGMA", "0.1")
    ref = pot.relax_batch(pop, urep=UREP, rlxt=3, mitr=1000, fmax=FMAX)
    monkeypatch.setenv("MAISE_B200_BATCH_SIGMA", sigma)
    r = pot.relax_batch(pop, urep=UREP, rlxt=3, mitr=1000, fmax=FMAX)
    conv = np.flatnonzero(r["status"] == 0)
    assert len(conv) >= 0.6 * len(pop)
    for k in conv:
        e = pot.efs(r["X"][k], r["LAT"][k], pop[k]["atmn"], ND=3, NM=300, urep=UREP)
        assert abs(r["H"][k] - e["H"]) / nat[k] < EV_ATOM
        assert np.abs(e["F"]).max() < FMAX + 2e-3
    if sigma == "0.5":
        per_iter = r["evals"] / r["iters"].sum()
        assert per_iter < 0.8 * ref["evals"] / ref["iters"].sum()


def test_batched_and_plain_reach_the_same_minimum(mgca):
    """Started inside one basin (a plain FP64 minimum shaken by 0.02 A), the
    batched and the plain relax end in the same minimum.  Both stop anywhere
    in the region where max |F| < 0.01 eV/A, whose energies spread by
    sum F^2 / 2k (a few 1e-4 eV/atom along soft modes: 2.2e-4 has been
    seen on a 54-atom cell), so the agreement asked for is that of one basin;
    the FP32 evaluation itself is held to 1e-5 eV/atom at identical
    structures by the tests above and by test_gpu_batch_forces.py."""
    pot, pop = mgca
    rng = np.random.default_rng(4)
    starts, plain = [], []
    for s in pop[:10]:
        a = pot.relax_fmax(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=UREP, rlxt=3, mitr=1000, fmax=FMAX)
        if not a["converged"]:
            continue
        x = a["X"] + rng.normal(0.0, 0.02, a["X"].shape)
        starts.append(dict(X=x, LAT=a["LAT"], atmn=s["atmn"]))
        plain.append(pot.relax_fmax(x, a["LAT"], s["atmn"], ND=3, NM=300, urep=UREP, rlxt=3, mitr=1000, fmax=FMAX))
    assert len(starts) >= 5
    b = pot.relax_batch(starts, urep=UREP, rlxt=3, mitr=1000, fmax=FMAX)
    for k, s in enumerate(starts):
        assert b["status"][k] == 0 and plain[k]["converged"]
        assert abs(b["H"][k] - plain[k]["H"]) / len(s["atmn"]) < 5e-4


def test_results_do_not_depend_on_population_order(mgca):
    """Each structure's relax is independent of where it sits in the queue.
    FP32 shared-memory atomics make the path reproducible to rounding only,
    and an unconverged BFGS path amplifies rounding, so a few iterations are
    compared."""
    pot, pop = mgca
    sub = pop[:12]
    nat = _nat(sub)
    a = pot.relax_batch(sub, urep=UREP, rlxt=3, mitr=0, fmax=FMAX)
    b = pot.relax_batch(sub[::-1], urep=UREP, rlxt=3, mitr=0, fmax=FMAX)
    np.testing.assert_allclose(a["H"] / nat, (b["H"] / nat[::-1])[::-1], atol=1e-6)
    # a line-search decision that falls inside the FP32 rounding floor can go
    # either way, so a few iterations agree to the early-path scale only
    a = pot.relax_batch(sub, urep=UREP, rlxt=3, mitr=4, fmax=FMAX)
    b = pot.relax_batch(sub[::-1], urep=UREP, rlxt=3, mitr=4, fmax=FMAX)
    np.testing.assert_allclose(a["H"] / nat, (b["H"] / nat[::-1])[::-1], atol=2e-4)


def test_oversized_structure_is_rejected(mgca):
    import maise_b200
    from maise_b200 import workloads

    pot, _ = mgca
    w = workloads.random_alloy(n=3, a=4.4, seed=1, species=(12, 20))  # 108 atoms
    with pytest.raises(maise_b200.MaiseError) as e:
        pot.relax_batch([w], urep=UREP, rlxt=3, mitr=5, fmax=FMAX)
    assert e.value.code == 1

"""GPU neighbour sets against the reference's LIST (src/cell.c:82-185),
exactly: for every atom the multiset of (neighbour atom, integer image) built
by each of the two GPU paths -- the all-pairs search (k_nlist_brute) and the
cell list (k_cell_* + k_nlist_cell) -- equals the one LIST builds in the
compiled reference sources.  Integer comparison only.  Cases: pairs planted
one ulp either side of r^2 = Rc^2 (inside the cell, across a periodic
boundary, and in a cluster), skewed cells whose thinnest direction holds the
minimum of 3 bins, small EA cells, the 4000-atom alloy and the 20000-atom
particle (no periodic directions)."""
from __future__ import annotations

import numpy as np
import pytest

import neighbour_cases as nc
from oracle import RefOracle, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference oracle not built")]

NM = 100


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    import maise_b200
    from maise_b200 import models, workloads

    d = tmp_path_factory.mktemp("nbr_model")
    w = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=0)
    models.random_model(str(d / "model"), [29], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=1)
    pot = maise_b200.Potential(str(d / "model"))
    yield pot, RefOracle(str(d))
    pot.close()


def _check(setup, w, paths):
    pot, ref = setup
    nn, nj, nic, Xw = ref.nlist(w["X"], w["LAT"], w["atmn"], w["ND"], NM=NM)
    want = nc.multiset(nn, nj, nic)
    for path in paths:
        gnn, gnj, gsh, gX = pot.neighbours(w["X"], w["LAT"], w["atmn"], ND=w["ND"], NM=NM, path=path)
        assert np.array_equal(gX, Xw), path
        got = nc.multiset(gnn, gnj, gsh)
        bad = [i for i in range(len(want)) if got[i] != want[i]]
        assert not bad, (path, bad[:5], len(bad))
    return want


@pytest.mark.parametrize("periodic", [True, False])
def test_planted_boundary_pairs(setup, periodic):
    w = nc.planted_pairs(setup[0].rc, periodic=periodic)
    ms = _check(setup, w, (1, 2))
    for i, j, img, inside in w["planted"]:
        assert ((j,) + tuple(img) in ms[i]) == inside


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_skewed_cells_both_paths(setup, seed):
    _check(setup, nc.skewed_cell(300, setup[0].rc, seed), (1, 2))


def test_small_ea_cells(setup):
    from maise_b200 import workloads

    for s in workloads.ea_population(count=8, nmin=8, nmax=64, seed=3, species=(29,)):
        _check(setup, dict(s, atmn=np.zeros(len(s["atmn"]), np.int32)), (0, 1))


def test_alloy_4000_both_paths(setup):
    from maise_b200 import workloads

    w = workloads.random_alloy(n=10, a=3.8, seed=0, jitter=0.05)
    _check(setup, dict(w, atmn=np.zeros(len(w["atmn"]), np.int32)), (0, 1))


def test_particle_20000_both_paths(setup):
    from maise_b200 import workloads

    w = workloads.fcc_particle()
    _check(setup, w, (0, 1))

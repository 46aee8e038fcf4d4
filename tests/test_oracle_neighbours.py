"""Neighbour sets of the C restatement against the reference's LIST
(src/cell.c:82-185), compiled from the reference sources: exact equality of
each atom's multiset of (neighbour atom, integer image), including pairs
planted one ulp either side of r^2 = Rc^2."""
from __future__ import annotations

import numpy as np
import pytest

import neighbour_cases as nc
from oracle import Oracle, RefOracle, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference oracle not built")


@pytest.fixture(scope="module")
def model_dir(tmp_path_factory):
    from maise_b200 import models, workloads

    d = tmp_path_factory.mktemp("nbr_model")
    w = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=0)
    models.random_model(str(d / "model"), [29], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=1)
    return str(d)


def _compare(model_dir, w, NM=200):
    o, ref = Oracle(model_dir + "/model"), RefOracle(model_dir)
    nn, nj, nic, Xw = ref.nlist(w["X"], w["LAT"], w["atmn"], w["ND"], NM=NM)
    onn, onj, onic, _, oX = o.nlist(w["X"], w["LAT"], w["atmn"], w["ND"], NM=NM)
    assert np.array_equal(oX, Xw)
    assert nc.multiset(onn, onj, onic) == nc.multiset(nn, nj, nic)
    return nc.multiset(nn, nj, nic)


@pytest.mark.parametrize("periodic", [True, False])
def test_planted_boundary_pairs(model_dir, periodic):
    rc = Oracle(model_dir + "/model").rc
    w = nc.planted_pairs(rc, periodic=periodic)
    ms = _compare(model_dir, w)
    for i, j, img, inside in w["planted"]:
        assert ((j,) + tuple(img) in ms[i]) == inside, (i, j, img, inside)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_skewed_cells(model_dir, seed):
    rc = Oracle(model_dir + "/model").rc
    _compare(model_dir, nc.skewed_cell(300, rc, seed))


def test_small_ea_cells(model_dir):
    from maise_b200 import workloads

    for s in workloads.ea_population(count=6, nmin=8, nmax=40, seed=3, species=(29,)):
        s = dict(s, atmn=np.zeros(len(s["atmn"]), np.int32))
        _compare(model_dir, s)

"""The evolutionary-search hand-off without a GPU: member files written by
the library (mb_evos_write) are read back by the reference's own READ_CELL
and Read_OSZI (compiled from the reference sources), as RELX_TR does
(src/emod.c:710-718); RANK_TR's ordering and fitness (src/emod.c:304-393)
against a restatement."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import RefOracle, ref_available


@pytest.fixture(scope="module")
def ref(tmp_path_factory):
    if not ref_available():
        pytest.skip("reference oracle not built")
    from maise_b200 import models, workloads

    d = tmp_path_factory.mktemp("evos_model")
    pop = workloads.ea_population(count=1, nmin=24, nmax=24, seed=1, species=(29, 46, 47))
    s = pop[0]
    models.random_model(str(d / "model"), [29, 46, 47], models.Basis(), (s["X"], s["LAT"], s["atmn"], 3), seed=2)
    r = RefOracle(str(d), 1)
    r.efs(s["X"], s["LAT"], s["atmn"], 3, NM=200)  # loads the model and sizes the reference cell
    return r


def test_member_files_read_back_by_the_reference(ref, tmp_path):
    from maise_b200 import evos, workloads

    rng = np.random.default_rng(0)
    pop = workloads.ea_population(count=4, nmin=8, nmax=24, seed=5, species=(29, 46, 47))
    for m, s in enumerate(pop):
        lat = s["LAT"] * (1.0 + 0.01 * rng.normal(size=(3, 3)))
        x = s["X"] + 0.05 * rng.normal(size=s["X"].shape)
        H = float(rng.normal(-3.0, 1.0) * len(s["atmn"]))
        evos.write_member(str(tmp_path), 7, 10 + m, [29, 46, 47], s["atmn"], s["LAT"], s["X"], lat, x, H,
                          frc=rng.normal(size=x.shape), str6=rng.normal(size=6), iters=42)
        mdir = tmp_path / "G007" / f"M{10 + m:03d}"
        for name in ("POSCAR.0", "CONTCAR.0", "OSZICAR.0", "OUTCAR.0"):
            assert (mdir / name).exists(), name
        got = ref.read_cell(str(mdir / "CONTCAR.0"))
        np.testing.assert_array_equal(got["atmn"], s["atmn"])
        np.testing.assert_allclose(got["LAT"], lat, atol=1e-13)
        np.testing.assert_allclose(got["X"], x, atol=1e-12)
        start = ref.read_cell(str(mdir / "POSCAR.0"))
        np.testing.assert_allclose(start["X"], s["X"], atol=1e-12)
        assert ref.read_oszi(str(mdir / "OSZICAR.0")) == pytest.approx(H, abs=5e-9)
        assert f"{H:14.8f}".strip() in (mdir / "OUTCAR.0").read_text()


def test_species_must_be_grouped(tmp_path):
    import maise_b200
    from maise_b200 import evos

    lat = np.eye(3) * 5.0
    x = np.random.default_rng(1).uniform(0, 5, (3, 3))
    with pytest.raises(maise_b200.MaiseError):
        evos.write_member(str(tmp_path), 0, 0, [12, 20], [1, 0, 1], lat, x, lat, x, -1.0)


def _rank_restated(H, nat, per_atom):
    """RANK_TR: e = enthalpy (per atom on request), ascending order, fitness
    (1 - tanh(2 (e - e_min) / (e_max - e_min) - 1)) / 2."""
    e = np.asarray(H, float) / (np.asarray(nat, float) if per_atom else 1.0)
    order = np.argsort(e, kind="stable")
    fit = 0.5 * (1.0 - np.tanh(2.0 * (e - e.min()) / (e.max() - e.min()) - 1.0))
    return order, fit


@pytest.mark.parametrize("per_atom", [False, True])
def test_rank_matches_rank_tr(per_atom):
    from maise_b200 import evos

    rng = np.random.default_rng(3)
    nat = rng.integers(8, 64, 40)
    H = rng.normal(-3.5, 0.2, 40) * nat
    H[5] = H[9]  # a tie keeps member order
    order, fit = evos.rank(H, nat, per_atom=per_atom)
    want_order, want_fit = _rank_restated(H, nat, per_atom)
    np.testing.assert_array_equal(order, want_order)
    np.testing.assert_allclose(fit, want_fit, rtol=1e-15, atol=1e-15)
    if not per_atom:
        # total enthalpy favours large cells; per atom does not
        assert nat[order[0]] >= np.median(nat)


def test_rank_rejects_a_degenerate_population():
    import maise_b200
    from maise_b200 import evos

    with pytest.raises(maise_b200.MaiseError):
        evos.rank(np.full(5, -10.0))

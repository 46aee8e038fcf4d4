"""The batched drop-in for RELX_INT (mb_evos_relax): one generation of
offspring relaxed in one launch, each member's files written where the
reference's RELX_TR reads them, and read back by the reference's READ_CELL
and Read_OSZI (src/emod.c:710-718): the enthalpies and relaxed structures
are the ones the relax returned, and RANK_TR's order follows from them."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import RefOracle, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference oracle not built")]

UREP = 100.0


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    import maise_b200
    from maise_b200 import models, workloads

    pop = workloads.ea_population(count=24, seed=13)
    big = max(pop, key=lambda s: len(s["atmn"]))
    d = tmp_path_factory.mktemp("evos_mgca")
    models.random_model(str(d / "model"), [12, 20], models.Basis(), (big["X"], big["LAT"], big["atmn"], 3), seed=5,
                        binding=True)
    ref = RefOracle(str(d), 1)
    ref.efs(big["X"], big["LAT"], big["atmn"], 3, NM=300)  # loads the model into the reference harness
    pot = maise_b200.Potential(str(d / "model"))
    yield pot, ref, pop
    pot.close()


def test_generation_files_round_trip_through_relx_tr(setup, tmp_path):
    from maise_b200 import evos

    pot, ref, pop = setup
    r = evos.relax_generation(pot, str(tmp_path / "EVOS"), 3, pop, first_member=len(pop), urep=UREP, mitr=300)
    assert list(r["members"]) == list(range(len(pop), 2 * len(pop)))
    for k, p in enumerate(r["members"]):
        mdir = tmp_path / "EVOS" / "G003" / f"M{p:03d}"
        got = ref.read_cell(str(mdir / "CONTCAR.0"))
        np.testing.assert_allclose(got["LAT"], r["LAT"][k], atol=1e-12)
        np.testing.assert_allclose(got["X"], r["X"][k], atol=1e-11)
        np.testing.assert_array_equal(got["atmn"], pop[k]["atmn"])
        assert ref.read_oszi(str(mdir / "OSZICAR.0")) == pytest.approx(r["H"][k], abs=5e-9)
        start = ref.read_cell(str(mdir / "POSCAR.0"))
        np.testing.assert_allclose(start["X"], pop[k]["X"], atol=1e-11)
        # the written enthalpy is the FP64 enthalpy of the written structure to the batched path's bar
        h64 = pot.energy(got["X"], got["LAT"], got["atmn"], ND=3, NM=300, urep=UREP)["H"]
        assert abs(h64 - r["H"][k]) / len(got["atmn"]) < 1e-5
    order, fit = evos.rank(r["H"], [len(s["atmn"]) for s in pop], per_atom=True)
    e = r["H"] / np.array([len(s["atmn"]) for s in pop])
    assert np.all(np.diff(e[order]) >= 0)
    assert fit[order[0]] == pytest.approx(0.5 * (1.0 - np.tanh(-1.0)))


def test_screened_generation_writes_only_the_kept_members(setup, tmp_path):
    from maise_b200 import evos
    from maise_b200.surrogate import Surrogate

    pot, ref, pop = setup
    sur = Surrogate(2)
    y = np.array([pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=UREP)["H"] / len(s["atmn"])
                  for s in pop])
    sur.fit(sur.features(pop), y, epochs=5, batch=8)
    r = evos.relax_generation(pot, str(tmp_path / "EVOS"), 0, pop, first_member=0, urep=UREP, mitr=200,
                              surrogate=sur, keep=0.25)
    sur.close()
    assert len(r["members"]) == len(pop) // 4
    written = sorted(p.name for p in (tmp_path / "EVOS" / "G000").iterdir())
    assert written == [f"M{p:03d}" for p in range(len(pop) // 4)]

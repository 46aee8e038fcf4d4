"""The leg-table descriptor pass (k_legs + k_efs_leg) against the general
fused kernel (k_efs, MAISE_B200_LEGS=0) and the oracle, in every mode:
descriptors, energy, energy+forces+virial and the descriptor VJP.  The two
paths sum the same terms in different orders, so they agree to rounding;
both are held to the plain-path bar against the oracle (1e-10 relative
energy, 1e-9 eV/A forces)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import Oracle

pytestmark = pytest.mark.gpu


def _pots(monkeypatch, path, force_legs=True):
    """(leg path, general path): the first handle is held to the leg kernel
    (a fixed leg shape; the autotuner may otherwise prefer k_efs for small
    structures), the second cannot use it."""
    import maise_b200

    monkeypatch.setenv("MAISE_B200_LEGS", "1")
    if force_legs:
        monkeypatch.setenv("MAISE_B200_SHAPE", "2")
    a = maise_b200.Potential(path)
    monkeypatch.delenv("MAISE_B200_SHAPE", raising=False)
    monkeypatch.setenv("MAISE_B200_LEGS", "0")
    b = maise_b200.Potential(path)
    monkeypatch.delenv("MAISE_B200_LEGS")
    return a, b


def _cases():
    from maise_b200 import workloads

    alloy = workloads.random_alloy(n=4, a=3.8, seed=5, jitter=0.1)               # 256 atoms, cell list
    small = workloads.random_alloy(n=2, a=3.7, seed=6, jitter=0.1)               # 32 atoms, all-pairs, images
    pop = workloads.ea_population(count=3, nmin=20, nmax=40, seed=8, species=(29, 46, 47))
    part = workloads.fcc_particle(n_target=600, seed=2, species=(29, 46, 47))
    part["atmn"] = (np.arange(len(part["atmn"])) % 3).astype(np.int32)
    return [("alloy", alloy), ("small", small), ("skewed", pop[0]), ("cluster", part)]


@pytest.mark.parametrize("name", ["alloy", "small", "skewed", "cluster"])
def test_leg_path_matches_general_path_and_oracle(tmp_path, monkeypatch, name):
    from maise_b200 import models

    w = dict(_cases())[name]
    ND = int(w["ND"])
    path = str(tmp_path / "model")
    models.random_model(path, [29, 46, 47], models.Basis(), (w["X"], w["LAT"], w["atmn"], max(ND, 1)), seed=4)
    legs, plain = _pots(monkeypatch, path)
    args = (w["X"], w["LAT"], w["atmn"])
    a = legs.efs(*args, ND=ND, NM=300, urep=100.0, p_gpa=2.0)
    b = plain.efs(*args, ND=ND, NM=300, urep=100.0, p_gpa=2.0)
    o = Oracle(path).efs(*args, ND, urep=100.0, p_gpa=2.0, NM=300)
    assert a["H"] == pytest.approx(b["H"], rel=1e-13)
    assert a["H"] == pytest.approx(o["H"], rel=1e-10)
    np.testing.assert_allclose(a["F"], b["F"], atol=1e-11)
    np.testing.assert_allclose(a["F"], o["F"], atol=1e-9)
    np.testing.assert_allclose(a["U"], o["U"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(a["EA"], b["EA"], rtol=1e-12, atol=1e-12)
    e = legs.energy(*args, ND=ND, NM=300, urep=100.0, p_gpa=2.0)
    assert e["H"] == pytest.approx(a["H"], rel=1e-14)
    G1, G2 = legs.descriptors(*args, ND=ND, NM=300), plain.descriptors(*args, ND=ND, NM=300)
    np.testing.assert_allclose(G1, G2, rtol=1e-12, atol=1e-14)
    g = np.random.default_rng(3).normal(size=G1.shape)
    F1, U1 = legs.descriptor_vjp(*args, g, ND=ND, NM=300)
    F2, U2 = plain.descriptor_vjp(*args, g, ND=ND, NM=300)
    np.testing.assert_allclose(F1, F2, atol=1e-10)
    np.testing.assert_allclose(U1, U2, rtol=1e-11, atol=1e-10)
    legs.close()
    plain.close()


def test_leg_path_every_shape(tmp_path, monkeypatch):
    """Every kernel shape of the leg path (warps per atom x atoms per block,
    each with both reverse-pass layouts) gives the same forces; the
    autotuner only chooses among them."""
    import maise_b200
    from maise_b200 import models, workloads

    w = workloads.random_alloy(n=4, a=3.8, seed=9, jitter=0.1)
    path = str(tmp_path / "model")
    models.random_model(path, [29, 46, 47], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=2)
    want = Oracle(path).efs(w["X"], w["LAT"], w["atmn"], 3, NM=300)
    for shape in range(8):
        monkeypatch.setenv("MAISE_B200_SHAPE", str(shape))
        pot = maise_b200.Potential(path)
        r = pot.efs(w["X"], w["LAT"], w["atmn"], ND=3, NM=300)
        pot.close()
        assert r["H"] == pytest.approx(want["H"], rel=1e-10), shape
        np.testing.assert_allclose(r["F"], want["F"], atol=1e-9, err_msg=str(shape))


def test_tune_table_records_the_chosen_shapes(tmp_path, monkeypatch):
    """The autotuner keeps one decision per (mode, kernel family, size
    bucket, capacity) and the table reports it with the shape's dimensions."""
    from maise_b200 import models

    w = dict(_cases())["alloy"]
    path = str(tmp_path / "model")
    models.random_model(path, [29, 46, 47], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=4)
    legs, plain = _pots(monkeypatch, path, force_legs=False)
    for pot, can_use_legs in ((legs, True), (plain, False)):
        pot.efs(w["X"], w["LAT"], w["atmn"], ND=3, NM=300)
        pot.energy(w["X"], w["LAT"], w["atmn"], ND=3, NM=300)
        tt = pot.tune_table()
        modes = {e["mode"] for e in tt}
        assert {"efs", "energy"} <= modes
        for e in tt:
            # with leg tables available the tuner picks the faster kernel family
            assert e["legs"] in ((True, False) if can_use_legs else (False,))
            assert e["size_bucket"] == 8  # 256 atoms
            assert e["wpa"] in (1, 2, 4, 8) and e["apb"] in (1, 2, 4)
        n = len(tt)
        pot.efs(w["X"], w["LAT"], w["atmn"], ND=3, NM=300)  # same key: no new decision
        assert len(pot.tune_table()) == n

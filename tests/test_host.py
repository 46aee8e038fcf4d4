"""CPU-side checks of the product: the C-ABI library loads and exports every
declared entry point, the reference-struct ABI offsets, the Maxwell
initialiser, model writing/parsing and the workload generators."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden
from oracle import Oracle, RefOracle, ref_available

LIB = os.path.join(ROOT, "maise_b200", "libmaise_b200.so")


def _declared_functions():
    names = []
    for h in ("maise_b200.h", "maise_call.h", "maise_surrogate.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                            text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "return")))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from maise_b200 import _build

        _build.build()
    from maise_b200 import load_library

    return load_library()


def test_library_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert "CALL_MAISE" in declared and "mb_efs" in declared and len(declared) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    missing = [n for n in declared if n not in exported]
    assert not missing, missing
    for n in declared:
        assert hasattr(lib, n)


@pytest.mark.skipif(not ref_available(), reason="reference sources were not compiled here")
def test_struct_abi_offsets_match_reference_headers():
    text = open(os.path.join(ROOT, "include", "maise_call.h")).read()
    val = {k: int(v) for k, v in re.findall(r"#define (MB_\w+) (\d+)", text)}
    s = RefOracle(".", 1).sizes()
    assert [val["MB_SIZEOF_ANN"], val["MB_SIZEOF_PRS"], val["MB_SIZEOF_LNK"], val["MB_SIZEOF_CELL"]] == s[:4]
    assert val["MB_OFFSET_ANN_UREP"] == s[4]
    assert val["MB_OFFSET_LNK_B"] == s[5]
    assert val["MB_OFFSET_CELL_P"] == s[6]
    assert val["MB_OFFSET_CELL_E"] == s[7]
    assert val["MB_OFFSET_CELL_H"] == s[8]


def test_no_gpu_path_fails_loudly(lib, tmp_path):
    from maise_b200 import MaiseError, Potential
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present")
    g = load_golden("kat_interface.npz")
    (tmp_path / "model").write_text(str(g["model"]))
    with pytest.raises(MaiseError) as e:
        Potential(str(tmp_path / "model"))
    assert e.value.code == 6
    from maise_b200.surrogate import Surrogate

    with pytest.raises(MaiseError) as e:
        Surrogate(3)
    assert e.value.code == 6


@pytest.mark.skipif(not ref_available(), reason="reference sources were not compiled here")
def test_maxwell_velocities_equal_reference(lib, tmp_path):
    from maise_b200 import atomic_mass, maxwell, models, workloads

    w = workloads.random_alloy(n=2, seed=4, species=(29, 46, 47))
    models.random_model(str(tmp_path / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3))
    ref = RefOracle(str(tmp_path), 1).maxwell(w["X"], w["LAT"], w["atmn"], 3, 600.0, seed=12345, NM=300)
    amu = [atomic_mass(w["spcz"][s]) for s in w["atmn"]]
    v = maxwell(amu, 600.0, seed=12345)
    np.testing.assert_array_equal(v, ref)


def test_park_miller_stream_known_answer(lib):
    """rngs.c self-test: 10000 draws from seed 1 end in state 399268537 (src/util.c:1922-1945)."""
    m, a = 2147483647, 48271
    x = 1
    for _ in range(10000):
        x = (a * x) % m
    assert x == 399268537
    from maise_b200 import maxwell

    v1 = maxwell([63.546] * 4, 300.0, seed=1)
    v2 = maxwell([63.546] * 4, 300.0, seed=1)
    np.testing.assert_array_equal(v1, v2)
    # zero total momentum and the target temperature (src/cmod.c:266-278)
    np.testing.assert_allclose(v1.sum(0), 0.0, atol=1e-15)
    K = 0.5 * (63.546 * 103.6427 * (v1 ** 2).sum())
    assert K * 11604.0 / 1.5 / 4 == pytest.approx(300.0, rel=1e-12)


def test_generated_model_parses_and_round_trips(tmp_path):
    from maise_b200 import models, workloads

    w = workloads.random_alloy(n=2, seed=1, species=(29, 46, 47))
    models.random_model(str(tmp_path / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3))
    o = Oracle(str(tmp_path / "model"))
    assert o.nspc == 3 and o.D == 282 and o.ng2 == 8 and o.ng4 == 43
    assert o.rc == pytest.approx(6.0, abs=1e-9)
    assert o.spcz == [29, 46, 47]


def test_workload_generators():
    from maise_b200 import workloads

    w1 = workloads.fcc_supercell()
    assert len(w1["atmn"]) == 32 and w1["ND"] == 3
    w2 = workloads.random_alloy()
    assert len(w2["atmn"]) == 4000 and np.bincount(w2["atmn"]).tolist() == [1334, 1333, 1333]
    assert (np.diff(w2["atmn"]) >= 0).all()
    pop = workloads.ea_population(count=6, seed=2)
    for s in pop:
        N = len(s["atmn"])
        assert 8 <= N <= 64
        vol = abs(np.linalg.det(s["LAT"]))
        assert 0.84 * 20 * N <= vol <= 1.16 * 20 * N
        assert (np.diff(s["atmn"]) >= 0).all()
    w4 = workloads.fcc_particle(n_target=2000, seed=1)
    assert 1800 <= len(w4["atmn"]) <= 2200 and w4["ND"] == 0
    assert (w4["X"] > 14.0).all() and (w4["X"] < w4["LAT"][0, 0] - 14.0).all()


def test_vectorised_cell_placement_keeps_the_random_stream():
    """Batched candidate scoring consumes the generator exactly as one
    candidate at a time, so a seed's population does not change."""
    import numpy as np

    from maise_b200 import workloads

    L0 = np.diag([6.0, 6.5, 7.0])
    rng_a, rng_b = np.random.default_rng(7), np.random.default_rng(7)
    pa, pb = [], []
    for _ in range(12):
        pa.append(workloads._place(rng_a, L0, np.array(pa).reshape(-1, 3), 2.0, batch=64))
        pb.append(workloads._place(rng_b, L0, np.array(pb).reshape(-1, 3), 2.0, batch=1))
    np.testing.assert_array_equal(np.array(pa), np.array(pb))
    assert rng_a.uniform() == rng_b.uniform()


def test_chunked_population_does_not_depend_on_workers():
    import numpy as np

    from maise_b200 import workloads

    a = workloads.ea_population_chunked(70, seed=4, chunk=32, workers=1, nmin=8, nmax=12)
    b = workloads.ea_population_chunked(70, seed=4, chunk=32, workers=2, nmin=8, nmax=12)
    assert len(a) == len(b) == 70
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x["X"], y["X"])
        np.testing.assert_array_equal(x["atmn"], y["atmn"])


def test_keep_fraction_calibration_on_held_out_pairs():
    from maise_b200.surrogate import calibrate_keep, recall

    rng = np.random.default_rng(4)
    truth = rng.normal(size=2000)
    # a perfect screen needs no more than the best tenth, plus the margin
    assert calibrate_keep(truth, truth, margin=0.02) == 0.12
    # a noisy screen needs a wider keep, and the chosen keep reaches the target
    pred = truth + rng.normal(scale=0.3, size=truth.size)
    q = calibrate_keep(pred, truth, target=0.99, margin=0.0)
    assert 0.12 < q < 1.0
    assert recall(pred, truth, q) >= 0.99
    assert recall(pred, truth, q - 0.01) < 0.99
    # an anti-correlated screen finds nothing short of relaxing everything
    assert calibrate_keep(-truth, truth) == 1.0
    with pytest.raises(ValueError):
        calibrate_keep([], [])

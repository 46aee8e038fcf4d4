"""Duplicate detection of the evolutionary search on the GPU against the
reference: the per-species-pair RDF (mb_rdf / k_rdf_ref) equals RDF of the
compiled reference sources (src/cell.c:369-417, run after LIST with the cutoff
Rmax) bin by bin, the all-pairs overlap matrix (mb_rdf_overlap) equals CxC
(src/cell.c:419-430) of the reference's vectors, and the duplicate rule
(mb_evos_duplicates) equals RANK_TR's (src/emod.c:351-368) with COMP_CL
(src/eutl.c:394-413) restated."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import RefOracle, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference oracle not built")]

SPC = (29, 46, 47)


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    from maise_b200 import models, workloads

    pop = workloads.ea_population(count=10, nmin=8, nmax=40, seed=21, species=SPC)
    big = max(pop, key=lambda s: len(s["atmn"]))
    d = tmp_path_factory.mktemp("rdf_model")
    models.random_model(str(d / "model"), list(SPC), models.Basis(), (big["X"], big["LAT"], big["atmn"], 3), seed=2)
    ref = RefOracle(str(d), 1)
    ref.efs(big["X"], big["LAT"], big["atmn"], 3, NM=300)
    return ref, pop


@pytest.mark.parametrize("normalise", [True, False])
def test_rdf_equals_reference(setup, normalise):
    from maise_b200 import evos

    ref, pop = setup
    got = evos.rdf(pop, 3, normalise=normalise)
    for k, s in enumerate(pop):
        want = ref.rdf(s["X"], s["LAT"], s["atmn"], 3, 3, normalise=normalise, NM=300)
        scale = 1.0 if normalise else max(1.0, float(np.abs(want).max()))
        np.testing.assert_allclose(got[k], want, rtol=0, atol=1e-12 * scale)


def test_overlaps_equal_cxc_of_reference_vectors(setup):
    from maise_b200 import evos

    ref, pop = setup
    R = np.stack([ref.rdf(s["X"], s["LAT"], s["atmn"], 3, 3, NM=300) for s in pop])
    cxc = evos.overlaps(evos.rdf(pop, 3))
    want = R.reshape(len(pop), -1) @ R.reshape(len(pop), -1).T
    np.testing.assert_allclose(cxc, want, atol=1e-12)
    np.testing.assert_allclose(np.diag(cxc), 1.0, atol=1e-12)
    # a structure and its rigidly shifted copy are the same structure
    s = pop[0]
    shifted = dict(s, X=s["X"] + np.array([0.3, -0.2, 0.1]))
    c2 = evos.overlaps(evos.rdf([s, shifted], 3))
    assert c2[0, 1] == pytest.approx(1.0, abs=1e-10)


def comp_cl(cxc, Hp, Hk, Vp, Vk):
    """COMP_CL (src/eutl.c:394-413)."""
    v = 0.5 * (Vp - Vk) / (Vp + Vk)
    return 0.8 * cxc + 0.1 * np.exp(-0.5 * (Hp - Hk) ** 2 / 0.05 ** 2) + 0.1 * np.exp(-0.5 * v * v / 0.01 ** 2)


def test_duplicate_rule_equals_rank_tr(setup):
    from maise_b200 import evos

    ref, pop = setup
    members = pop + [dict(pop[2], X=pop[2]["X"] + 0.001), dict(pop[5])]  # two near-copies
    H = np.array([-3.0 * len(s["atmn"]) for s in members]) + np.linspace(0, 0.5, len(members))
    H[-2], H[-1] = H[2] + 0.01, H[5] + 0.02
    vol = np.array([abs(np.linalg.det(np.asarray(s["LAT"]))) for s in members])
    order = np.argsort(H, kind="stable")
    members, H, vol = [members[k] for k in order], H[order], vol[order]
    cxc = evos.overlaps(evos.rdf(members, 3))
    fit0 = np.linspace(1.0, 0.1, len(members))
    got = evos.duplicates(cxc, H, vol, fit0, 0.95)
    want = fit0.copy()
    for p in range(len(members) - 1, 0, -1):
        for k in range(p - 1, -1, -1):
            t = comp_cl(cxc[p, k], H[p], H[k], vol[p], vol[k])
            if t > 0.95:
                want[p] *= 0.001 + (1.0 - t) ** 2
                break
    np.testing.assert_allclose(got, want, rtol=1e-14)
    assert (got < fit0 * 0.5).sum() >= 2  # both copies found

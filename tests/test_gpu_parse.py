"""The parse path on the GPU: the descriptor tangent (mb_descriptor_jvp) is
the adjoint of the VJP and reproduces the reference's derivative blocks Fn
of the golden parse set (test/parse/ref, read by tests/golden/make_golden.py)
and the oracle's strain blocks Sn; descriptor files written by
mb_parse_efile are read back by the reference's own LNK_IN
(src/nprs.c:308-377) with the golden descriptors and blocks."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, write_model_dir
from oracle import Oracle, RefOracle, ref_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import maise_b200

    return maise_b200


def test_tangent_is_the_adjoint_of_the_vjp(mb, tmp_path):
    c = load_golden("ref_efs.npz")["cases"][2]
    d = write_model_dir(tmp_path, c["model"])
    pot = mb.Potential(d + "/model")
    rng = np.random.default_rng(5)
    N = len(c["atmn"])
    g = rng.normal(size=(N, pot.D))
    dx = rng.normal(size=(N, 3))
    e6 = rng.normal(size=6)
    eps = np.zeros((3, 3))
    for k, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]):
        eps[a, b] = e6[k]
    dG = pot.descriptor_jvp(c["X"], c["LAT"], c["atmn"], dx=dx, eps=eps, ND=3, NM=400)
    F, U = pot.descriptor_vjp(c["X"], c["LAT"], c["atmn"], g, ND=3, NM=400)
    lhs = float((g * dG).sum())
    rhs = -float((F * dx).sum()) - float(U @ e6)
    assert lhs == pytest.approx(rhs, rel=1e-10, abs=1e-10)


def golden_total(dni, Fn, atom, owner):
    """dG_owner/dx_atom from the reference's blocks: the reference keeps the
    part of an atom's own descriptors that comes through its periodic images
    in a separate block listed under its own index, beside the self block
    (slot dnn); the tangent gives their sum."""
    tot = sum(Fn[slot] for slot, o in enumerate(dni) if o == owner)
    if owner == atom:
        tot = tot + Fn[len(dni)]
    return tot


def test_tangent_gives_the_golden_derivative_blocks(mb, parse_golden, parse_model_dir):
    pot = mb.Potential(parse_model_dir + "/model")
    off = parse_golden["offsets"]
    for k in range(len(parse_golden["mk_atom"])):
        s, atom = int(parse_golden["mk_struct"][k]), int(parse_golden["mk_atom"][k])
        a, b = off[s], off[s + 1]
        X, at, L = parse_golden["x"][a:b], parse_golden["atmn"][a:b], parse_golden["lat"][s]
        cols = []
        for q in range(3):
            dx = np.zeros((len(at), 3))
            dx[atom, q] = 1.0
            cols.append(pot.descriptor_jvp(X, L, at, dx=dx, ND=3, NM=400))
        blk = np.stack(cols, axis=-1)  # [owner, n, q]
        dni, Fn = parse_golden["mk_dni"][k], parse_golden["mk_fn"][k]
        for o in set(dni.tolist()) | {atom}:
            np.testing.assert_allclose(blk[o], golden_total(dni, Fn, atom, o), atol=1e-10)
        # no atom outside the reference's list depends on this atom
        others = np.setdiff1d(np.arange(len(at)), np.concatenate([dni, [atom]]))
        assert np.abs(blk[others]).max(initial=0.0) == 0.0


def test_strain_tangent_matches_oracle_blocks(mb, tmp_path):
    c = load_golden("ref_efs.npz")["cases"][1]
    d = write_model_dir(tmp_path, c["model"])
    pot, o = mb.Potential(d + "/model"), Oracle(d + "/model")
    cols = []
    for a, b in [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]:
        eps = np.zeros((3, 3))
        eps[a, b] = 1.0
        cols.append(pot.descriptor_jvp(c["X"], c["LAT"], c["atmn"], eps=eps, ND=int(c["ND"]), NM=400))
    Sn = np.stack(cols, axis=-1)
    for atom in (0, len(c["atmn"]) // 2):
        _, _, Sno = o.fn(c["X"], c["LAT"], c["atmn"], int(c["ND"]), atom, NM=400)
        np.testing.assert_allclose(Sn[atom], Sno, atol=1e-10 * max(1.0, np.abs(Sno).max()))


@pytest.mark.skipif(not ref_available(), reason="reference oracle not built")
def test_descriptor_files_read_back_by_lnk_in(mb, parse_golden, parse_model_dir, tmp_path):
    pot = mb.Potential(parse_model_dir + "/model")
    off = parse_golden["offsets"]
    marked_by_struct = {}
    for k in range(len(parse_golden["mk_atom"])):
        marked_by_struct.setdefault(int(parse_golden["mk_struct"][k]), []).append(k)
    structs = sorted(marked_by_struct)[:6] + [0, 1]
    for idx, s in enumerate(structs):
        a, b = off[s], off[s + 1]
        X, at, L = parse_golden["x"][a:b], parse_golden["atmn"][a:b], parse_golden["lat"][s]
        N = len(at)
        EFS = 1 if idx < 6 else 3
        marked = np.zeros(N, bool)
        for k in marked_by_struct.get(s, []):
            marked[int(parse_golden["mk_atom"][k])] = True
        F = np.random.default_rng(idx).normal(size=(N, 3))
        pot.parse_efile(str(tmp_path), idx, X, L, at, EFS=EFS, ND=3, NM=400, E=-2.5 * N, p=1.25, DE=0.5,
                        marked=marked, frc_ref=F, str_ref=np.arange(6.0), data_path=f"./DATA/{s}/")
        r = RefOracle.read_efile(str(tmp_path), idx)
        assert (r["EFS"], r["D"], r["N"], r["NF"]) == (EFS, 82, N, int(marked.sum()))
        assert (r["E"], r["DE"]) == pytest.approx((-2.5 * N, 0.5), abs=1e-6)
        head = open(tmp_path / f"e{idx:06d}").readline().split()
        assert float(head[6]) == pytest.approx(1.25)  # LNK_IN reads the pressure but Build_LNK resets it
        np.testing.assert_array_equal(r["atmn"], at)
        np.testing.assert_allclose(r["Cn"], parse_golden["G"][a:b], rtol=1e-12, atol=1e-13)
        for k in marked_by_struct.get(s, []):
            atom = int(parse_golden["mk_atom"][k])
            dni, Fr, Fn = r["blocks"][atom]
            np.testing.assert_allclose(Fr, F[atom], atol=1e-6)
            gdni, gFn = parse_golden["mk_dni"][k], parse_golden["mk_fn"][k]
            assert sorted(dni) == sorted(set(gdni.tolist()) - {atom})
            np.testing.assert_allclose(Fn[len(dni)], golden_total(gdni, gFn, atom, atom), atol=1e-10)
            for slot, o in enumerate(dni):
                np.testing.assert_allclose(Fn[slot], golden_total(gdni, gFn, atom, o), atol=1e-10)
        if EFS == 3:
            np.testing.assert_allclose(r["S"], np.arange(6.0))
            assert r["Sn"].shape == (N, 82, 6)

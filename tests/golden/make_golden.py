"""Generate the golden fixtures under tests/golden/ from the reference.

Run in a container where the reference sources are mounted (default
/root/reference, override with MAISE_REFERENCE) and oracle/_ref has been
built (`make -C oracle ref`):

    python tests/golden/make_golden.py

Outputs (committed; nothing at test time reads the reference tree):

  parse_cuag.npz    136 Cu-Ag structures of test/parse: geometry, the
                    reference's descriptor vectors (e-files, 82 inputs) and
                    the derivative blocks of the marked atoms; plus the basis.
  kat_interface.npz the interface known-answer test (interface/c): model
                    text, 4-atom cluster, printed OUTCAR values and the
                    compiled reference's full-precision outputs.
  relax.npz         test/relax (Cu3Pd) and examples/03-rlx (Cu4) inputs with
                    the GSL-produced results printed in their reference files,
                    and the compiled reference's relax over the project BFGS.
  ref_efs.npz       compiled-reference energies/forces/virials of small
                    seeded structures for generated models (1, 2, 3 species;
                    crystal and cluster), with the model texts.

The reference runs single-threaded: CELL_UREP's force loop shares the
pair radius R between OpenMP threads (src/cmod.c:95-98 omit it from
private), so with more than one thread its repulsive forces race.
"""
from __future__ import annotations

import glob
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from maise_b200 import models, workloads  # noqa: E402
from oracle import RefOracle  # noqa: E402

REF = os.environ.get("MAISE_REFERENCE", "/root/reference")
SYMB = {"Cu": 29, "Ag": 47, "Pd": 46, "Au": 79, "Mg": 12, "Ca": 20, "Li": 3}


def read_poscar(path, species_order):
    """POSCAR -> (LAT rows, X Cartesian, atmn) with READ_CELL's arithmetic
    (src/util.c:820-989): lattice times scale, Direct -> Cartesian by
    x_q = sum_j f_j L_jq accumulated from 0."""
    with open(path) as f:
        lines = f.read().splitlines()
    scale = float(lines[1].split()[0])
    L = [[float(v) * scale for v in lines[2 + i].split()[:3]] for i in range(3)]
    names = lines[5].split()
    counts = [int(v) for v in lines[6].split()]
    k = 7
    if lines[k].strip()[0] in "Ss":
        k += 1
    direct = lines[k].strip()[0] in "Dd"
    k += 1
    X, atmn = [], []
    for name, cnt in zip(names, counts):
        for _ in range(cnt):
            v = [float(t) for t in lines[k].split()[:3]]
            k += 1
            if direct:
                c = []
                for q in range(3):
                    s = 0.0
                    for j in range(3):
                        s += v[j] * L[j][q]
                    c.append(s)
                v = c
            X.append(v)
            atmn.append(species_order.index(SYMB[name]))
    return np.array(L), np.array(X), np.array(atmn, np.int32)


def read_efile(path, D):
    """Parse an e-file written by LNK_OUT (src/nprs.c:380-442)."""
    with open(path) as f:
        toks = f.read().split("\n")
    head = toks[0].split()
    efs, d, N, NF, _dnn = int(head[0]), int(head[1]), int(head[2]), int(head[3]), int(head[4])
    assert d == D
    li = 1
    marked = []
    if efs in (1, 3):
        marked = [int(v) for v in toks[li].split()]
        li += 1
    li += 1  # path
    G = np.zeros((N, D))
    atmn = np.zeros(N, np.int32)
    for i in range(N):
        atmn[i] = int(toks[li]); li += 1
        for n in range(D):
            G[i, n] = float(toks[li]); li += 1
    blocks = []
    if efs in (1, 3):
        for _ in range(NF):
            hdr = toks[li].split(); li += 1
            atom, dnn = int(hdr[0]), int(hdr[1])
            F = np.array([float(v) for v in hdr[2:5]])
            Fn = np.zeros((dnn + 1, D, 3))
            for n in range(D):
                Fn[dnn, n] = [float(v) for v in toks[li].split()]; li += 1
            dni = []
            for j in range(dnn):
                dni.append(int(toks[li])); li += 1
                for n in range(D):
                    Fn[j, n] = [float(v) for v in toks[li].split()]; li += 1
            blocks.append((atom, np.array(dni, np.int32), Fn, F))
    return G, atmn, marked, blocks, float(head[5])


def make_parse():
    base = os.path.join(REF, "test", "parse")
    species = [29, 47]
    index = {}
    with open(os.path.join(base, "ref", "index.dat")) as f:
        for line in f:
            name, path = line.split()
            index[name] = path
    out = dict(basis=open(os.path.join(base, "basis")).read(), spcz=np.array(species))
    names = sorted(k for k in index if os.path.exists(os.path.join(base, "ref", k)))
    lats, xs, ats, gs, offs = [], [], [], [], [0]
    mk_atom, mk_struct, mk_dni, mk_fn, mk_F, E = [], [], [], [], [], []
    for s, name in enumerate(names):
        rel = index[name].replace("./", "")
        L, X, at = read_poscar(os.path.join(base, rel, "POSCAR.0"), species)
        G, gat, marked, blocks, e = read_efile(os.path.join(base, "ref", name), 82)
        E.append(e)
        assert (gat == at).all(), name
        lats.append(L); xs.append(X); ats.append(at); gs.append(G); offs.append(offs[-1] + len(at))
        for atom, dni, Fn, F in blocks:
            mk_struct.append(s); mk_atom.append(atom); mk_dni.append(dni); mk_fn.append(Fn); mk_F.append(F)
    out.update(names=np.array(names), lat=np.array(lats), x=np.concatenate(xs), atmn=np.concatenate(ats),
               G=np.concatenate(gs), offsets=np.array(offs), mk_struct=np.array(mk_struct),
               mk_atom=np.array(mk_atom), mk_dni=np.array(mk_dni, dtype=object), mk_fn=np.array(mk_fn, dtype=object),
               mk_F=np.array(mk_F), E=np.array(E))
    np.savez_compressed(os.path.join(HERE, "parse_cuag.npz"), **out)
    print("parse:", len(names), "structures,", len(mk_atom), "marked atoms")


def make_kat():
    base = os.path.join(REF, "interface", "c")
    model = open(os.path.join(base, "bin", "model")).read()
    X = np.array([[2.0, 0, 0], [-2.0, 0, 0], [0, 2.0, 0], [0, -2.0, 0]])
    LAT = np.eye(3) * 20.0
    at = np.zeros(4, np.int32)
    r = RefOracle(os.path.join(base, "bin"), 1)
    res = r.efs(X, LAT, at, 0, NM=500)
    np.savez_compressed(os.path.join(HERE, "kat_interface.npz"), model=model, X=X, LAT=LAT, atmn=at, NM=500,
                        outcar_H=-6.35967864, outcar_F=1.141127, outcar_UV=-0.06891844,
                        outcar_EA=-1.589919661072, ref_H=res["H"], ref_F=res["F"], ref_U=res["U"], ref_EA=res["EA"])
    print("kat: H", res["H"])


def make_relax():
    out = {}
    for key, d, species in (("cu3pd", os.path.join(REF, "test", "relax"), [29, 46]),
                            ("cu4", os.path.join(REF, "examples", "03-rlx"), [29])):
        L, X, at = read_poscar(os.path.join(d, "POSCAR"), species)
        out[key + "_model"] = open(os.path.join(d, "model")).read()
        out[key + "_lat"], out[key + "_x"], out[key + "_atmn"] = L, X, at
        r = RefOracle(d, 1)
        res = r.relax(X, L, at, 3, rlxt=3, mitr=100, etol=1e-6, NM=300)
        out[key + "_ref_H"], out[key + "_ref_lat"], out[key + "_ref_x"] = res["H"], res["LAT"], res["X"]
        out[key + "_ref_calls"] = np.array([res["n_energy"], res["n_force"], res["iters"]])
        print(key, "relax H", res["H"], "calls", res["n_energy"], res["n_force"], res["iters"])
    # values printed by the reference's GSL runs
    out["cu3pd_gsl_H0"], out["cu3pd_gsl_H"], out["cu3pd_gsl_a"] = -17.25531076, -18.08137782, 3.72890112684628
    out["cu4_gsl_H0"], out["cu4_gsl_H"] = -12.9467487748680767, -16.3965601100172194
    np.savez_compressed(os.path.join(HERE, "relax.npz"), **out)


def make_ref_efs():
    cases = []
    rng = np.random.default_rng(7)
    w1 = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=11)
    w2 = workloads.random_alloy(n=2, a=3.8, seed=12, species=(29, 47), jitter=0.08)
    w3 = workloads.random_alloy(n=2, a=3.8, seed=13, species=(29, 46, 47), jitter=0.08)
    X4, L4, a4 = workloads.random_cell(9, rng, 2)
    w4 = dict(X=X4, LAT=L4, atmn=a4, ND=3, spcz=[12, 20])
    cl = workloads.fcc_particle(n_target=60, a=3.61, jitter=0.05, pad=10.0, seed=14, species=(29,))
    for name, w, urep, p in (("cu32", w1, 0.0, 0.0), ("cuag32", w2, 0.0, 2.0), ("cupdag32", w3, 0.0, 0.0),
                             ("mgca9", w4, 100.0, 1.0), ("cu_cluster", cl, 0.0, 0.0)):
        with tempfile.TemporaryDirectory() as td:
            models.random_model(os.path.join(td, "model"), w["spcz"], models.Basis(),
                                (w["X"], w["LAT"], w["atmn"], w["ND"]), seed=3)
            text = open(os.path.join(td, "model")).read()
            r = RefOracle(td, 1)
            res = r.efs(w["X"], w["LAT"], w["atmn"], w["ND"], urep=urep, p_gpa=p, NM=400)
            G = r.descriptors(w["X"], w["LAT"], w["atmn"], w["ND"], NM=400)
        cases.append(dict(name=name, model=text, X=w["X"], LAT=w["LAT"], atmn=w["atmn"], ND=w["ND"], urep=urep,
                          p=p, H=res["H"], E=res["E"], F=res["F"], U=res["U"], EA=res["EA"], G=G))
        print(name, "N", len(w["atmn"]), "H", res["H"])
    np.savez_compressed(os.path.join(HERE, "ref_efs.npz"), cases=np.array(cases, dtype=object))


if __name__ == "__main__":
    parts = {"parse": make_parse, "kat": make_kat, "relax": make_relax, "ref_efs": make_ref_efs}
    for name in sys.argv[1:] or list(parts):
        parts[name]()

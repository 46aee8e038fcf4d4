"""Training of a MAISE model's per-species networks on the GPU (ctypes view of
include/maise_train.h).

The reference trains by minimising tot_err_gsl with GSL's BFGS (MLP_MIN,
src/nmin.c:314-445) over the energies and, with EFS 1 or 3, the forces of
marked atoms in its parsed descriptor files (PARS_DAT, src/nprs.c:983-1366).
Here the descriptors come from the GPU (Potential.descriptors on a model
file that fixes the basis and the input range table) or from descriptor
files (Trainer.from_efiles), the force blocks from the descriptor tangent
(Potential.descriptor_jvp) or the same files, and the objective, its
gradient and the minimisation run in libmaise_b200 (mb_train_*); the
trained parameters are written back to a model file in the reference's
format, with the template's basis and ranges.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import MaiseError, Potential, load_library, models

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _lib():
    lib = load_library()
    if getattr(lib, "_train_ready", False):
        return lib
    c_i, c_d, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    lib.mb_train_open.argtypes = [c_i, c_i, _I, _I, c_i, c_i, c_i, c_i, _D, _D, _D, _D, _D, c_d, c_d,
                                  ctypes.POINTER(vp)]
    lib.mb_train_close.argtypes = [vp]
    lib.mb_train_info.argtypes = [vp, _I]
    lib.mb_train_eval.argtypes = [vp, _D, _D, _D, _D]
    lib.mb_train_fit.argtypes = [vp, _D, c_i, c_d, _D, _I]
    lib.mb_train_set_forces.argtypes = [vp, c_i, _I, _D, _I, _I, _D, c_i, _D, c_d]
    lib.mb_train_eval_forces.argtypes = [vp, _D, _D, _D]
    lib._train_ready = True
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


class Trainer:
    """Training of the networks of `model_path` (its basis, range table and
    architecture) on `structures` (list of dict(X, LAT, atmn, ND)) with
    reference energies `energies` (eV per structure), or on given
    descriptors: descriptors=(G[Na, D], atmn[Na], nat[S]).  Force training
    is added by set_forces or forces_from_structures."""

    def __init__(self, model_path, structures=None, energies=None, weights=None, WE=1.0, LREG=0.0, device=0, NM=300,
                 descriptors=None):
        self.lib = _lib()
        self.template = models.read_model(model_path)
        self.model_path, self.device, self.NM = model_path, device, NM
        self.structures = structures
        D, h1, h2 = self.template["arch"]
        nspc = len(self.template["spcz"])
        if descriptors is None:
            pot = Potential(model_path, device=device)
            G = np.concatenate([pot.descriptors(s["X"], s["LAT"], s["atmn"], ND=int(s.get("ND", 3)), NM=NM)
                                for s in structures])
            pot.close()
            nat = np.array([len(s["atmn"]) for s in structures], np.int32)
            atmn = np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures])
        else:
            G, atmn, nat = descriptors
            nat = np.asarray(nat, np.int32)
        atmn = np.ascontiguousarray(np.asarray(atmn, np.int32))
        rmin = np.ascontiguousarray(self.template["rmin"], float)
        dr = np.ascontiguousarray(self.template["dr"], float)
        E = np.ascontiguousarray(np.asarray(energies, float))
        W = None if weights is None else np.ascontiguousarray(np.asarray(weights, float))
        self.G = np.ascontiguousarray(np.asarray(G, float))
        self.atmn, self.nat = atmn, nat
        self.offsets = np.concatenate([[0], np.cumsum(nat)]).astype(np.int64)
        self.h = ctypes.c_void_p()
        self._check(self.lib.mb_train_open(device, len(nat), nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I), nspc, D,
                                           h1, h2, _dp(self.G), _dp(rmin), _dp(dr), _dp(E), _dp(W), WE, LREG,
                                           ctypes.byref(self.h)))
        n = ctypes.c_int()
        self._check(self.lib.mb_train_info(self.h, ctypes.byref(n)))
        self.nparams = n.value
        self.S = len(nat)
        self.NF = 0

    @classmethod
    def from_efiles(cls, model_path, directory, indices, WE=1.0, WF=1.0, LREG=0.0, WENE=None, device=0):
        """Training set read from descriptor files (the reference's LNK_IN
        layout): energies, descriptors and, for EFS 1 and 3, the marked atoms'
        forces and blocks (scaled to the input range for EFS 1 only, as
        ADJT_LNK does, src/nmod.c:244-259).  Structure weights from the
        energy spread DE as the reference sets them (src/nmod.c:233-239):
        1 when DE < |WENE| (or WENE is None), else |WENE| / DE."""
        from .efile import read_efile

        files = [read_efile(directory, i) for i in indices]
        G = np.concatenate([f["G"] for f in files])
        atmn = np.concatenate([f["atmn"] for f in files])
        nat = [f["N"] for f in files]
        E = [f["E"] for f in files]
        w = [1.0 if WENE is None or f["DE"] < abs(WENE) else abs(WENE) / f["DE"] for f in files]
        tr = cls(model_path, None, E, weights=w, WE=WE, LREG=LREG, device=device, descriptors=(G, atmn, nat))
        f_atom, F, owners, Fn, counts = [], [], [], [], []
        efs = {f["EFS"] for f in files if f["blocks"]}
        for k, f in enumerate(files):
            for (atom, own, fn), fr in zip(f["blocks"], f["F"]):
                f_atom.append(tr.offsets[k] + atom)
                F.append(fr)
                owners.append(tr.offsets[k] + own)
                Fn.append(fn)
                counts.append(len(own))
        if f_atom:
            if len(efs) != 1:
                raise ValueError("descriptor files mix EFS 1 and 3")
            tr.set_forces(np.array(f_atom), np.array(F), np.concatenate([[0], np.cumsum(counts)]),
                          np.concatenate(owners), np.concatenate(Fn), WF=WF, scale_blocks=efs == {1})
        return tr

    def _check(self, rc):
        if rc:
            raise MaiseError(rc, self.lib.mb_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_train_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initial(self):
        """The template model's parameters (V2W order)."""
        return models.vector_from_nets(self.template["nets"])

    def eval(self, V, grad=True):
        """(RT, gradient or None, predicted energies[S])."""
        V = np.ascontiguousarray(np.asarray(V, float))
        RT = ctypes.c_double()
        g = np.zeros(self.nparams) if grad else None
        E = np.zeros(self.S)
        self._check(self.lib.mb_train_eval(self.h, _dp(V), ctypes.byref(RT), _dp(g), _dp(E)))
        return RT.value, g, E

    def set_forces(self, f_atom, F_ref, blk_off, blk_atom, Fn, WF=1.0, scale_blocks=True):
        """Force training data: marked atoms f_atom[NF] (rows of the training
        set's atoms), reference forces F_ref[NF, 3], and for marked atom i
        the blocks blk_off[i] .. blk_off[i+1]-1, block b being dG_o/dx_i
        (Fn[b], D x 3) of owner atom o = blk_atom[b], self block included."""
        f_atom = np.ascontiguousarray(np.asarray(f_atom, np.int32))
        F_ref = np.ascontiguousarray(np.asarray(F_ref, float).reshape(-1))
        blk_off = np.ascontiguousarray(np.asarray(blk_off, np.int32))
        blk_atom = np.ascontiguousarray(np.asarray(blk_atom, np.int32))
        Fn = np.ascontiguousarray(np.asarray(Fn, float).reshape(-1))
        dr = np.ascontiguousarray(self.template["dr"], float)
        self._check(self.lib.mb_train_set_forces(self.h, len(f_atom), f_atom.ctypes.data_as(_I), _dp(F_ref),
                                                 blk_off.ctypes.data_as(_I), blk_atom.ctypes.data_as(_I), _dp(Fn),
                                                 1 if scale_blocks else 0, _dp(dr), WF))
        self.NF = len(f_atom)

    def forces_from_structures(self, marked, F_ref, WF=1.0):
        """Force training on the constructor's structures: marked[s] the
        marked atoms of structure s, F_ref[s] their reference forces [.., 3].
        Blocks from the descriptor tangent, owners as the parse path lists
        them (the atom's neighbour atoms in ascending order, then itself)."""
        pot = Potential(self.model_path, device=self.device)
        f_atom, F, owners, Fn, counts = [], [], [], [], []
        try:
            for k, s in enumerate(self.structures):
                ND = int(s.get("ND", 3))
                nn, nj, _, _ = pot.neighbours(s["X"], s["LAT"], s["atmn"], ND=ND, NM=self.NM)
                N = len(s["atmn"])
                for atom, fr in zip(marked[k], F_ref[k]):
                    own = np.array(sorted(set(nj[atom, :nn[atom]].tolist()) - {int(atom)}) + [int(atom)], np.int32)
                    cols = []
                    for q in range(3):
                        dx = np.zeros((N, 3))
                        dx[atom, q] = 1.0
                        cols.append(pot.descriptor_jvp(s["X"], s["LAT"], s["atmn"], dx=dx, ND=ND, NM=self.NM))
                    blk = np.stack(cols, axis=-1)  # [owner, D, 3]
                    f_atom.append(self.offsets[k] + atom)
                    F.append(fr)
                    owners.append(self.offsets[k] + own)
                    Fn.append(blk[own])
                    counts.append(len(own))
        finally:
            pot.close()
        self.set_forces(np.array(f_atom), np.array(F), np.concatenate([[0], np.cumsum(counts)]),
                        np.concatenate(owners), np.concatenate(Fn), WF=WF, scale_blocks=True)

    def eval_forces(self, V):
        """(predicted forces of the marked atoms [NF, 3], sum_s w_s |F - f|^2)."""
        V = np.ascontiguousarray(np.asarray(V, float))
        f = np.zeros(3 * self.NF)
        RF = ctypes.c_double()
        self._check(self.lib.mb_train_eval_forces(self.h, _dp(V), _dp(f), ctypes.byref(RF)))
        return f.reshape(self.NF, 3), RF.value

    def fit(self, V, mitr=200, gtol=1e-12):
        """BFGS from V: (V, RT, iterations)."""
        V = np.ascontiguousarray(np.asarray(V, float)).copy()
        RT, it = ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.mb_train_fit(self.h, _dp(V), mitr, gtol, ctypes.byref(RT), ctypes.byref(it)))
        return V, RT.value, it.value

    def save(self, path, V):
        """Write a model file: the template with the networks of V."""
        t = self.template
        D, h1, h2 = t["arch"]
        nper = len(V) // len(t["spcz"])
        nets = [models.nets_from_vector(V[s * nper:(s + 1) * nper], (D, h1, h2)) for s in range(len(t["spcz"]))]
        models.write_model(path, t["spcz"], t["arch"], nets, t["rmin"], t["rmax"], t["basis_text"],
                           model_id="B200TRAINED", dr=t["dr"])
        return path

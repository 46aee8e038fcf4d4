"""Training of a MAISE model's per-species networks on the GPU (ctypes view of
include/maise_train.h).

The reference trains by minimising tot_err_gsl with GSL's BFGS (MLP_MIN,
src/nmin.c:314-445) over energies of parsed structures (the descriptors of
PARS_DAT, src/nprs.c:983-1366).  Here the descriptors come from the GPU
(Potential.descriptors on a model file that fixes the basis and the input
range table), and the objective, its gradient and the minimisation run in
libmaise_b200 (mb_train_*); the trained parameters are written back to a
model file in the reference's format, with the template's basis and ranges.
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
    lib._train_ready = True
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


class Trainer:
    """Energy training of the networks of `model_path` (its basis, range
    table and architecture) on `structures` (list of dict(X, LAT, atmn, ND))
    with reference energies `energies` (eV per structure)."""

    def __init__(self, model_path, structures, energies, weights=None, WE=1.0, LREG=0.0, device=0, NM=300):
        self.lib = _lib()
        self.template = models.read_model(model_path)
        D, h1, h2 = self.template["arch"]
        nspc = len(self.template["spcz"])
        pot = Potential(model_path, device=device)
        G = np.concatenate([pot.descriptors(s["X"], s["LAT"], s["atmn"], ND=int(s.get("ND", 3)), NM=NM)
                            for s in structures])
        pot.close()
        nat = np.array([len(s["atmn"]) for s in structures], np.int32)
        atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures]))
        rmin = np.ascontiguousarray(self.template["rmin"], float)
        dr = np.ascontiguousarray(self.template["dr"], float)
        E = np.ascontiguousarray(np.asarray(energies, float))
        W = None if weights is None else np.ascontiguousarray(np.asarray(weights, float))
        self.G = np.ascontiguousarray(G)
        self.h = ctypes.c_void_p()
        self._check(self.lib.mb_train_open(device, len(nat), nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I), nspc, D,
                                           h1, h2, _dp(self.G), _dp(rmin), _dp(dr), _dp(E), _dp(W), WE, LREG,
                                           ctypes.byref(self.h)))
        n = ctypes.c_int()
        self._check(self.lib.mb_train_info(self.h, ctypes.byref(n)))
        self.nparams = n.value
        self.S = len(nat)

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

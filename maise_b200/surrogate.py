"""Surrogate screen for EA offspring (ctypes view of include/maise_surrogate.h).

The reference relaxes every offspring of a generation (RELX_INT / RELX_TR,
src/emod.c:521-757) and then ranks them by enthalpy (RANK_TR,
src/emod.c:304-393).  Here a small FP32 MLP on per-species-pair radial
histograms (the analogue of RDF, src/cell.c:369-417) predicts each
offspring's relaxed enthalpy per atom from its unrelaxed structure; only the
best-ranked fraction is relaxed, by the full method, whose enthalpies then
rank the survivors as before.  Features, forward, backward and Adam run in
the library's own kernels; this module only moves arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import MaiseError, load_library

_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

NBINS = 128
RMAX = 6.0
SIGMA = 0.05
HIDDEN = (128, 64, 64)


def _lib():
    lib = load_library()
    if getattr(lib, "_sur_ready", False):
        return lib
    c_i, c_d, vp, c_u = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_uint
    lib.mb_sur_open.argtypes = [c_i, c_i, c_i, c_d, c_d, c_i, c_i, c_i, c_u, ctypes.POINTER(vp)]
    lib.mb_sur_close.argtypes = [vp]
    lib.mb_sur_close.restype = None
    lib.mb_sur_info.argtypes = [vp, _I, ctypes.POINTER(ctypes.c_long)]
    lib.mb_sur_features.argtypes = [vp, c_i, _I, _I, _D, _D, _F]
    lib.mb_sur_fit.argtypes = [vp, c_i, _F, _D, c_i, c_i, c_d, c_u, _F]
    lib.mb_sur_predict.argtypes = [vp, c_i, _F, _D]
    lib.mb_sur_screen.argtypes = [vp, c_i, _I, _I, _D, _D, _D]
    lib.mb_sur_loss_grad.argtypes = [vp, c_i, _F, _F, _D, _F]
    lib.mb_sur_adam_step.argtypes = [vp, _F, c_d]
    lib.mb_sur_get_params.argtypes = [vp, _F]
    lib.mb_sur_set_params.argtypes = [vp, _F]
    lib.mb_sur_get_norm.argtypes = [vp, _F, _F, _D, _D]
    lib._sur_ready = True
    return lib


def _f32(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def pack(structures):
    """(nat, atmn, lat, x) arrays of a list of dict(X, LAT, atmn)."""
    nat = np.array([len(s["atmn"]) for s in structures], np.int32)
    atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures]))
    lat = np.ascontiguousarray(np.stack([np.asarray(s["LAT"], float).reshape(9) for s in structures]))
    x = np.ascontiguousarray(np.concatenate([np.asarray(s["X"], float).reshape(-1) for s in structures]))
    return nat, atmn, lat, x


class Surrogate:
    """Relaxed-enthalpy-per-atom predictor nin -> h1 -> h2 -> h3 -> 1 (SiLU, FP32)."""

    def __init__(self, nspc: int, nbins: int = NBINS, rmax: float = RMAX, sigma: float = SIGMA, hidden=HIDDEN,
                 seed: int = 1, device: int = 0):
        self.lib = _lib()
        self.h = ctypes.c_void_p()
        self.nspc, self.nbins, self.rmax, self.sigma, self.hidden = nspc, nbins, rmax, sigma, tuple(hidden)
        self._check(self.lib.mb_sur_open(device, nspc, nbins, rmax, sigma, hidden[0], hidden[1], hidden[2], seed,
                                         ctypes.byref(self.h)))
        nin, npar = ctypes.c_int(), ctypes.c_long()
        self._check(self.lib.mb_sur_info(self.h, ctypes.byref(nin), ctypes.byref(npar)))
        self.nin, self.nparams = nin.value, npar.value

    def _check(self, rc):
        if rc:
            raise MaiseError(rc, self.lib.mb_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_sur_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def features(self, structures) -> np.ndarray:
        nat, atmn, lat, x = pack(structures)
        out = np.zeros((len(nat), self.nin), np.float32)
        self._check(self.lib.mb_sur_features(self.h, len(nat), nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I),
                                             lat.ctypes.data_as(_D), x.ctypes.data_as(_D), out.ctypes.data_as(_F)))
        return out

    def fit(self, feat, y, epochs=100, batch=256, lr=1e-3, seed=1) -> np.ndarray:
        feat = _f32(feat)
        S = feat.size // self.nin
        y = np.ascontiguousarray(np.asarray(y, float).reshape(-1))
        loss = np.zeros(max(epochs, 1), np.float32)
        self._check(self.lib.mb_sur_fit(self.h, S, feat.ctypes.data_as(_F), y.ctypes.data_as(_D), epochs, batch, lr,
                                        seed, loss.ctypes.data_as(_F)))
        return loss[:epochs]

    def predict(self, feat) -> np.ndarray:
        feat = _f32(feat)
        S = feat.size // self.nin
        out = np.zeros(S)
        self._check(self.lib.mb_sur_predict(self.h, S, feat.ctypes.data_as(_F), out.ctypes.data_as(_D)))
        return out

    def screen(self, structures) -> np.ndarray:
        """Predicted relaxed enthalpy per atom, features kept on the GPU."""
        nat, atmn, lat, x = pack(structures)
        out = np.zeros(len(nat))
        self._check(self.lib.mb_sur_screen(self.h, len(nat), nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I),
                                           lat.ctypes.data_as(_D), x.ctypes.data_as(_D), out.ctypes.data_as(_D)))
        return out

    def loss_grad(self, x, t):
        x = _f32(x)
        t = _f32(t)
        B = t.size
        loss = ctypes.c_double()
        g = np.zeros(self.nparams, np.float32)
        self._check(self.lib.mb_sur_loss_grad(self.h, B, x.ctypes.data_as(_F), t.ctypes.data_as(_F),
                                              ctypes.byref(loss), g.ctypes.data_as(_F)))
        return loss.value, g

    def adam_step(self, grad, lr):
        g = _f32(grad, self.nparams)
        self._check(self.lib.mb_sur_adam_step(self.h, g.ctypes.data_as(_F), lr))

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, np.float32)
        self._check(self.lib.mb_sur_get_params(self.h, p.ctypes.data_as(_F)))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p, self.nparams)
        self._check(self.lib.mb_sur_set_params(self.h, p.ctypes.data_as(_F)))

    def norm(self):
        mean = np.zeros(self.nin, np.float32)
        istd = np.zeros(self.nin, np.float32)
        tm, ts = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mb_sur_get_norm(self.h, mean.ctypes.data_as(_F), istd.ctypes.data_as(_F),
                                             ctypes.byref(tm), ctypes.byref(ts)))
        return mean, istd, tm.value, ts.value


def keep_best(pred, keep_frac: float) -> np.ndarray:
    """Indices of the lowest keep_frac of the predictions (stable order)."""
    n = max(1, int(round(keep_frac * len(pred))))
    return np.sort(np.argsort(pred, kind="stable")[:n])


def recall(pred, truth, keep_frac: float, top_frac: float = 0.10) -> float:
    """Fraction of the lowest top_frac of `truth` (the relaxed enthalpies that
    judge the screen) found among the lowest keep_frac of `pred`."""
    truth = np.asarray(truth)
    ntop = max(1, int(round(top_frac * len(truth))))
    top = set(np.argsort(truth, kind="stable")[:ntop].tolist())
    return len(top & set(keep_best(pred, keep_frac).tolist())) / ntop


def calibrate_keep(pred, truth, target: float = 0.99, top_frac: float = 0.10, margin: float = 0.02,
                   step: float = 0.01) -> float:
    """Keep fraction for a generation, chosen on held-out training pairs
    (predictions `pred` of structures whose relaxed enthalpies `truth` are
    known but were not fitted): the smallest fraction on a `step` grid from
    `top_frac` up whose recall of the held-out best `top_frac` reaches
    `target`, plus `margin`; 1.0 (relax everything) when no fraction below
    1 does."""
    pred, truth = np.asarray(pred), np.asarray(truth)
    if len(pred) != len(truth) or len(pred) == 0:
        raise ValueError("calibrate_keep: pred and truth must be non-empty and of one length")
    k = 0
    while True:
        q = round(top_frac + k * step, 6)
        if q >= 1.0:
            return 1.0
        if recall(pred, truth, q, top_frac) >= target:
            return min(1.0, round(q + margin, 6))
        k += 1

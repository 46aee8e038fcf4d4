"""One generation of MAISE's evolutionary search around the batched relax.

The reference's EA loop (src/emod.c) breeds offspring (EVLV_TR), relaxes
members N..2N-1 one after the other (RELX_INT, src/emod.c:521-548), reads the
results back from EVOS/Gnnn/Mppp (RELX_TR, src/emod.c:552-757) and ranks the
2N members by enthalpy (RANK_TR, src/emod.c:304-393).  ``relax_generation``
is the drop-in for RELX_INT: one persistent launch relaxes every offspring
and the library writes each member's POSCAR.0, CONTCAR.0, OSZICAR.0 and
OUTCAR.0 where RELX_TR reads them.  With a trained surrogate
(maise_b200.surrogate) the offspring are screened first and only the best
predicted fraction is relaxed; the others are not written, as RELX_TR then
has no files for them (the caller drops them from the tribe).  ``rank``
is RANK_TR's ordering and fitness, by total enthalpy as the reference does,
or per atom for populations whose members differ in size.

These are bindings of libmaise_b200's C-ABI (mb_evos_relax, mb_evos_write,
mb_evos_rank); the files are written by the library.
"""
from __future__ import annotations

import os

import numpy as np

from . import _D, _I, _dp, load_library

__all__ = ["relax_generation", "write_member", "rank", "rdf", "overlaps", "duplicates"]


def _check(lib, rc):
    from . import MaiseError

    if rc:
        raise MaiseError(rc, lib.mb_last_error().decode())


def relax_generation(pot, evos_dir, gen, offspring, first_member, p_gpa=0.0, urep=100.0, rlxt=3, mitr=1000,
                     fmax=0.01, surrogate=None, keep=1.0):
    """Relax `offspring` (list of dict(X, LAT, atmn)) as members
    first_member, first_member+1, ... of generation `gen` and write their
    EVOS files.  Returns dict(members, H, iters, status, X, LAT): with a
    surrogate, only the kept offspring (best `keep` fraction by predicted
    enthalpy per atom) are relaxed and numbered, in screening order."""
    lib = load_library()
    idx = np.arange(len(offspring))
    if surrogate is not None and keep < 1.0:
        from .surrogate import keep_best

        idx = np.sort(keep_best(surrogate.screen(offspring), keep))
    chosen = [offspring[k] for k in idx]
    nat = np.array([len(s["atmn"]) for s in chosen], np.int32)
    atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in chosen]))
    X = np.ascontiguousarray(np.concatenate([np.asarray(s["X"], float).reshape(-1, 3) for s in chosen]))
    LAT = np.ascontiguousarray(np.stack([np.asarray(s["LAT"], float).reshape(3, 3) for s in chosen]))
    S = len(chosen)
    H = np.zeros(S)
    iters = np.zeros(S, np.int32)
    status = np.zeros(S, np.int32)
    _check(lib, lib.mb_evos_relax(pot.h, os.fsencode(evos_dir), gen, first_member, S, nat.ctypes.data_as(_I),
                                  atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), p_gpa, urep, rlxt, mitr, fmax, _dp(H),
                                  iters.ctypes.data_as(_I), status.ctypes.data_as(_I)))
    offs = np.concatenate([[0], np.cumsum(nat)])
    return dict(members=first_member + np.arange(S), offspring=idx, H=H, iters=iters, status=status,
                X=[X[offs[k]:offs[k + 1]] for k in range(S)], LAT=LAT)


def write_member(evos_dir, gen, member, spcz, atmn, lat0, x0, lat, x, H, E=None, p_gpa=0.0, frc=None, str6=None,
                 iters=0):
    """Write one member's EVOS files (no GPU needed)."""
    lib = load_library()
    atmn = np.ascontiguousarray(np.asarray(atmn, np.int32))
    spcz = np.ascontiguousarray(np.asarray(spcz, np.int32))
    f64 = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a, float).reshape(-1))  # noqa: E731
    _check(lib, lib.mb_evos_write(os.fsencode(evos_dir), gen, member, len(atmn), len(spcz), spcz.ctypes.data_as(_I),
                                  atmn.ctypes.data_as(_I), _dp(f64(lat0)), _dp(f64(x0)), _dp(f64(lat)), _dp(f64(x)),
                                  H, H if E is None else E, p_gpa, _dp(f64(frc)), _dp(f64(str6)), iters))


def rank(H, nat=None, per_atom=False):
    """RANK_TR's order (best first) and fitness of members with enthalpies H."""
    lib = load_library()
    H = np.ascontiguousarray(np.asarray(H, float))
    M = len(H)
    nat_a = np.ascontiguousarray(np.asarray(nat if nat is not None else np.ones(M), np.int32))
    order = np.zeros(M, np.int32)
    fit = np.zeros(M)
    _check(lib, lib.mb_evos_rank(M, _dp(H), nat_a.ctypes.data_as(_I), int(per_atom), order.ctypes.data_as(_I),
                                 _dp(fit)))
    return order, fit


def rdf(structures, nspc, nbins=3000, rmin=5.8, rmax=6.0, sigma=0.008, normalise=True, ND=3, device=0):
    """RANK_TR's per-species-pair RDF of every structure, on the GPU:
    [S, nspc (nspc + 1) / 2, nbins] (the reference's defaults)."""
    lib = load_library()
    nat = np.array([len(s["atmn"]) for s in structures], np.int32)
    atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures]))
    X = np.ascontiguousarray(np.concatenate([np.asarray(s["X"], float).reshape(-1, 3) for s in structures]))
    LAT = np.ascontiguousarray(np.stack([np.asarray(s["LAT"], float).reshape(3, 3) for s in structures]))
    npair = nspc * (nspc + 1) // 2
    out = np.zeros((len(nat), npair, nbins))
    _check(lib, lib.mb_rdf(device, len(nat), nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), ND,
                           nspc, nbins, rmin, rmax, sigma, int(normalise), _dp(out)))
    return out


def overlaps(R, device=0):
    """CxC of every pair of members: [S, S] from RDFs R[S, ...]."""
    lib = load_library()
    R = np.ascontiguousarray(np.asarray(R, float).reshape(len(R), -1))
    out = np.zeros((len(R), len(R)))
    _check(lib, lib.mb_rdf_overlap(device, len(R), R.shape[1], _dp(R), _dp(out)))
    return out


def duplicates(cxc, H, vol, fit, cut):
    """RANK_TR's duplicate down-weighting of `fit` (members in rank order)."""
    lib = load_library()
    cxc = np.ascontiguousarray(np.asarray(cxc, float))
    H = np.ascontiguousarray(np.asarray(H, float))
    vol = np.ascontiguousarray(np.asarray(vol, float))
    fit = np.ascontiguousarray(np.asarray(fit, float)).copy()
    _check(lib, lib.mb_evos_duplicates(len(H), _dp(cxc), _dp(H), _dp(vol), cut, _dp(fit)))
    return fit

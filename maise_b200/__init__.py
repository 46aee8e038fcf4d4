"""maise_b200 -- B200 (sm_100a) implementation of MAISE's neural-network
interatomic potential path, driven through the C-ABI of libmaise_b200.so.

The compute lives entirely in the shared library (C host + CUDA kernels);
this module is a thin ctypes view of it with the reference's argument
meanings (positions in Angstrom, lattice vectors as rows, species indices in
model order, virial in eV with order xx,yy,zz,xy,yz,zx).  There is no CPU
fallback: if the library or a GPU is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["Potential", "MaiseError", "library_path", "load_library", "maxwell", "atomic_mass"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmaise_b200.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)

MB_ERRORS = {1: "argument", 2: "model", 3: "neighbours", 4: "cuda", 5: "capacity", 6: "no gpu", 7: "state"}


class MaiseError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{MB_ERRORS.get(code, code)}] {message}")
        self.code = code


def library_path() -> str:
    return _LIB_PATH


def load_library():
    """Load libmaise_b200.so (built by maise_b200._build); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise FileNotFoundError(f"{_LIB_PATH} is missing; run `python -m maise_b200._build` (needs nvcc)")
    lib = ctypes.CDLL(_LIB_PATH)
    c_i, c_d, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    lib.mb_last_error.restype = ctypes.c_char_p
    lib.mb_open.argtypes = [ctypes.c_char_p, c_i, ctypes.POINTER(vp)]
    lib.mb_close.argtypes = [vp]
    lib.mb_model_info.argtypes = [vp, _I, _I, _I, _D]
    lib.mb_reserve.argtypes = [vp, c_i, c_i]
    lib.mb_efs.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, _D, _D, _D, _D, _D, _D]
    lib.mb_energy.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, _D, _D, _D]
    lib.mb_descriptors.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, _D]
    lib.mb_descriptor_vjp.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, _D, _D, _D]
    lib.mb_neighbours.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, c_i, c_i, _I, _I, _I, _D]
    lib.mb_descriptor_jvp.argtypes = [vp, c_i, c_i, c_i, c_i, _I, _D, _D, _D, _D, _D]
    lib.mb_parse_efile.argtypes = [vp, ctypes.c_char_p, c_i, c_i, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, c_d, _I,
                                   _D, _D, ctypes.c_char_p]
    lib.mb_relax.argtypes = [vp, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, c_i, c_i, c_d, _D, _L]
    lib.mb_md_nvt.argtypes = [vp, c_i, c_i, c_i, _I, _D, _D, _D, c_d, c_d, c_d, c_i, c_d, _D, _D, _D]
    lib.mb_maxwell.argtypes = [c_i, _D, c_d, ctypes.c_long, _D]
    lib.mb_relax_fmax.argtypes = [vp, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, c_i, c_i, c_d, _D, _L, _I]
    lib.mb_relax_batch.argtypes = [vp, c_i, _I, _I, _D, _D, c_d, c_d, c_i, c_i, c_d, _D, _I, _I]
    lib.mb_efs_batch.argtypes = [vp, c_i, _I, _I, _D, _D, c_d, c_d, _D, _D, _D]
    lib.mb_evos_write.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _I, _D, _D, _D, _D, c_d, c_d, c_d, _D, _D,
                                  c_i]
    lib.mb_evos_relax.argtypes = [vp, ctypes.c_char_p, c_i, c_i, c_i, _I, _I, _D, _D, c_d, c_d, c_i, c_i, c_d, _D, _I,
                                  _I]
    lib.mb_evos_rank.argtypes = [c_i, _D, _I, c_i, _I, _D]
    lib.mb_evos_duplicates.argtypes = [c_i, _D, _D, _D, c_d, _D]
    lib.mb_rdf.argtypes = [c_i, c_i, _I, _I, _D, _D, c_i, c_i, c_i, c_d, c_d, c_d, c_i, _D]
    lib.mb_rdf_overlap.argtypes = [c_i, c_i, c_i, _D, _D]
    lib.mb_batch_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), _D]
    lib.mb_tune_read.argtypes = [vp, ctypes.c_int, _I, _I, _I, _I, _I, _I, _I, _I]
    lib.mb_atomic_mass.restype = c_d
    lib.mb_atomic_mass.argtypes = [c_i]
    lib.mb_stream.restype = vp
    lib.mb_stream.argtypes = [vp]
    lib.mb_launch_count.restype = ctypes.c_long
    lib.mb_launch_count.argtypes = [vp]
    lib.mb_graphs.argtypes = [vp, c_i]
    lib.mb_profile.argtypes = [vp, c_i, c_i]
    lib.mb_profile_read.argtypes = [vp, _D, _I, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
    lib.mb_fp64_peak.argtypes = [c_i, _D]
    lib.mb_fp32_peak.argtypes = [c_i, _D]
    lib.mb_batch_work.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                  ctypes.POINTER(ctypes.c_longlong)]
    lib.mb_md_profile.argtypes = [vp, c_i, c_i, ctypes.c_size_t]
    lib.mb_md_profile_read.argtypes = [vp, _D, _I]
    lib.CALL_MAISE.restype = c_d
    lib.CALL_MAISE.argtypes = [vp, vp, vp, vp, vp, c_i, c_i, c_i, c_i, c_i, c_i, _I, _D, _D, _D, _D]
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _f64(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(-1) if n is None else a.reshape(n)


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


def maxwell(amu, T, seed=1):
    """Maxwell velocities (A/fs) drawn as src/cmod.c:224-280 does; no GPU needed."""
    lib = load_library()
    amu = _f64(amu)
    V = np.zeros(3 * len(amu))
    rc = lib.mb_maxwell(len(amu), _dp(amu), T, seed, _dp(V))
    if rc:
        raise MaiseError(rc, lib.mb_last_error().decode())
    return V.reshape(-1, 3)


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput of the device (TFLOP/s)."""
    lib = load_library()
    t = ctypes.c_double()
    rc = lib.mb_fp64_peak(device, ctypes.byref(t))
    if rc:
        raise MaiseError(rc, "fp64 peak probe failed")
    return t.value


def fp32_peak_tflops(device: int = 0) -> float:
    """Measured FP32 FMA throughput of the device (TFLOP/s)."""
    lib = load_library()
    t = ctypes.c_double()
    rc = lib.mb_fp32_peak(device, ctypes.byref(t))
    if rc:
        raise MaiseError(rc, "fp32 peak probe failed")
    return t.value


def atomic_mass(z: int) -> float:
    return float(load_library().mb_atomic_mass(z))


class Potential:
    """A MAISE neural-network model resident on one CUDA device.

    Mirrors the reference's per-structure operations: ``efs`` (CELL_FRC /
    CALL_MAISE), ``energy`` (CELL_ENE), ``descriptors`` (PRS_BP energy part),
    ``relax`` (CELL_RELX/CELL_MIN) and ``md_nvt`` (the NVT branch of
    Dynamics).  ``ND`` is the number of periodic directions (0 or 3).
    """

    def __init__(self, model_path: str, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        self._check(self.lib.mb_open(os.fsencode(model_path), device, ctypes.byref(h)))
        self.h = h
        nspc, D, rc = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        spcz = (ctypes.c_int * 8)()
        self._check(self.lib.mb_model_info(self.h, ctypes.byref(nspc), spcz, ctypes.byref(D), ctypes.byref(rc)))
        self.nspc, self.D, self.rc = nspc.value, D.value, rc.value
        self.spcz = list(spcz)[: self.nspc]

    def _check(self, rc: int) -> None:
        if rc:
            raise MaiseError(rc, self.lib.mb_last_error().decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mb_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        return int(self.lib.mb_stream(self.h) or 0)

    @property
    def launches(self) -> int:
        return int(self.lib.mb_launch_count(self.h))

    def profile(self, enable=True, capacity=4096) -> None:
        """Bracket each fused-kernel launch with CUDA events; reset counters."""
        self._check(self.lib.mb_profile(self.h, int(enable), capacity))

    def profile_read(self):
        """dict(ms_total, launches, pairs, triplets) since profile(True)."""
        ms, n = ctypes.c_double(), ctypes.c_int()
        pr, tr = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        self._check(self.lib.mb_profile_read(self.h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(pr),
                                             ctypes.byref(tr)))
        return dict(ms_total=ms.value, launches=n.value, pairs=pr.value, triplets=tr.value)

    def md_profile(self, enable=True, capacity=100000, flush_bytes=0) -> None:
        """Per-step CUDA-event timing of md_nvt, with an optional L2 flush between steps."""
        self._check(self.lib.mb_md_profile(self.h, int(enable), capacity, flush_bytes))

    def md_profile_read(self):
        ms, n = ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.mb_md_profile_read(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return dict(ms_total=ms.value, steps=n.value)

    def tune_table(self):
        """The autotuner's choices: list of dict(mode, legs, size_bucket,
        capacity, wpa, apb, layout), modes 'descriptors', 'energy', 'efs',
        'vjp'; layout is the leg kernel's reverse pass ('runs' or 'rounds')."""
        cap = 32
        cols = [np.zeros(cap, np.int32) for _ in range(7)]
        cnt = ctypes.c_int()
        self._check(self.lib.mb_tune_read(self.h, cap, ctypes.byref(cnt), *(c.ctypes.data_as(_I) for c in cols)))
        n = cnt.value
        names = ("descriptors", "energy", "efs", "vjp")
        return [dict(mode=names[int(cols[0][k])], legs=bool(cols[1][k]), size_bucket=int(cols[2][k]),
                     capacity=int(cols[3][k]), wpa=int(cols[4][k]), apb=int(cols[5][k]),
                     layout="rounds" if cols[6][k] else "runs") for k in range(n)]

    def graphs(self, enable: bool) -> None:
        """MD chunks as CUDA graphs (default) or plain launches."""
        self._check(self.lib.mb_graphs(self.h, 1 if enable else 0))

    def reserve(self, max_atoms: int, max_neighbours: int) -> None:
        self._check(self.lib.mb_reserve(self.h, max_atoms, max_neighbours))

    def efs(self, X, LAT, atmn, ND=3, NM=512, XT=1, p_gpa=0.0, urep=0.0):
        """dict(H, E, F[N,3], U[6], EA[N], X[N,3] wrapped) -- CELL_FRC semantics."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        H, E = ctypes.c_double(), ctypes.c_double()
        F = np.zeros(3 * N)
        U = np.zeros(6)
        EA = np.zeros(N)
        Xw = np.zeros(3 * N)
        self._check(self.lib.mb_efs(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), p_gpa, urep,
                                    ctypes.byref(H), ctypes.byref(E), _dp(F), _dp(U), _dp(EA), _dp(Xw)))
        return dict(H=H.value, E=E.value, F=F.reshape(N, 3), U=U, EA=EA, X=Xw.reshape(N, 3))

    def energy(self, X, LAT, atmn, ND=3, NM=512, XT=1, p_gpa=0.0, urep=0.0):
        """dict(H, E, EA) -- CELL_ENE semantics."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        H, E = ctypes.c_double(), ctypes.c_double()
        EA = np.zeros(N)
        self._check(self.lib.mb_energy(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), p_gpa,
                                       urep, ctypes.byref(H), ctypes.byref(E), _dp(EA)))
        return dict(H=H.value, E=E.value, EA=EA)

    def descriptors(self, X, LAT, atmn, ND=3, NM=512, XT=1):
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        G = np.zeros(N * self.D)
        self._check(self.lib.mb_descriptors(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X),
                                            _dp(G)))
        return G.reshape(N, self.D)

    def descriptor_vjp(self, X, LAT, atmn, g, ND=3, NM=512, XT=1):
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        g = _f64(g, N * self.D)
        F = np.zeros(3 * N)
        U = np.zeros(6)
        self._check(self.lib.mb_descriptor_vjp(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X),
                                               _dp(g), _dp(F), _dp(U)))
        return F.reshape(N, 3), U

    def neighbours(self, X, LAT, atmn, ND=3, NM=512, XT=1, path=0, cap=None):
        """The neighbour list of the E/F/S passes (LIST's set):
        (nn[N], nj[N,cap], shift[N,cap,3] integer images, X[N,3] wrapped).
        path 0 as the passes choose, 1 all-pairs search, 2 cell list."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        cap = cap or NM
        nn = np.zeros(N, np.int32)
        nj = np.zeros(N * cap, np.int32)
        sh = np.zeros(N * cap * 3, np.int32)
        Xw = np.zeros(3 * N)
        self._check(self.lib.mb_neighbours(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), path,
                                           cap, nn.ctypes.data_as(_I), nj.ctypes.data_as(_I),
                                           sh.ctypes.data_as(_I), _dp(Xw)))
        return nn, nj.reshape(N, cap), sh.reshape(N, cap, 3), Xw.reshape(N, 3)

    def descriptor_jvp(self, X, LAT, atmn, dx=None, eps=None, ND=3, NM=512, XT=1):
        """Tangent of the descriptors, [N, D], for atom displacements dx[N, 3]
        and/or the deformation eps[3, 3] of every neighbour displacement."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        dxa = None if dx is None else _f64(dx, 3 * N)
        ea = None if eps is None else _f64(eps, 9)
        dG = np.zeros(N * self.D)
        self._check(self.lib.mb_descriptor_jvp(self.h, N, NM, ND, XT, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X),
                                               _dp(dxa), _dp(ea), _dp(dG)))
        return dG.reshape(N, self.D)

    def parse_efile(self, directory, index, X, LAT, atmn, EFS=1, ND=3, NM=512, XT=1, E=0.0, p=0.0, DE=0.0,
                    marked=None, frc_ref=None, str_ref=None, data_path="./"):
        """Write <directory>/e%06d in the reference's parse layout (LNK_OUT)."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N)
        LAT = _f64(LAT, 9)
        mk = None if marked is None else _i32(np.asarray(marked, bool).astype(np.int32))
        fr = None if frc_ref is None else _f64(frc_ref, 3 * N)
        sr = None if str_ref is None else _f64(str_ref, 6)
        self._check(self.lib.mb_parse_efile(self.h, os.fsencode(directory), index, EFS, N, NM, ND, XT,
                                            atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), E, p, DE,
                                            None if mk is None else mk.ctypes.data_as(_I), _dp(fr), _dp(sr),
                                            os.fsencode(data_path)))
        return os.path.join(directory, f"e{index:06d}")

    def relax(self, X, LAT, atmn, ND=3, NM=512, p_gpa=0.0, urep=0.0, rlxt=3, mitr=100, etol=1e-6):
        """dict(H, X, LAT, n_energy, n_force, iters) -- CELL_RELX/CELL_MIN."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N).copy()
        LAT = _f64(LAT, 9).copy()
        H = ctypes.c_double()
        counts = np.zeros(3, np.int64)
        self._check(self.lib.mb_relax(self.h, N, NM, ND, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), p_gpa, urep,
                                      rlxt, mitr, etol, ctypes.byref(H), counts.ctypes.data_as(_L)))
        return dict(H=H.value, X=X.reshape(N, 3), LAT=LAT.reshape(3, 3), n_energy=int(counts[0]),
                    n_force=int(counts[1]), iters=int(counts[2]))

    def relax_fmax(self, X, LAT, atmn, ND=3, NM=512, p_gpa=0.0, urep=0.0, rlxt=3, mitr=500, fmax=0.01):
        """dict(H, X, LAT, n_energy, n_force, iters, converged) -- force-criterion relax, FP64, host BFGS."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N).copy()
        LAT = _f64(LAT, 9).copy()
        H = ctypes.c_double()
        counts = np.zeros(3, np.int64)
        conv = ctypes.c_int()
        self._check(self.lib.mb_relax_fmax(self.h, N, NM, ND, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), p_gpa, urep,
                                           rlxt, mitr, fmax, ctypes.byref(H), counts.ctypes.data_as(_L),
                                           ctypes.byref(conv)))
        return dict(H=H.value, X=X.reshape(N, 3), LAT=LAT.reshape(3, 3), n_energy=int(counts[0]),
                    n_force=int(counts[1]), iters=int(counts[2]), converged=bool(conv.value))

    def relax_batch(self, structures, p_gpa=0.0, urep=0.0, rlxt=3, mitr=500, fmax=0.01):
        """Relax a list of dict(X, LAT, atmn) in one persistent launch.
        Returns dict(H[S], X list, LAT[S,3,3], iters[S], status[S], evals, ms)."""
        nat = np.array([len(s["atmn"]) for s in structures], np.int32)
        atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures]))
        X = np.ascontiguousarray(np.concatenate([np.asarray(s["X"], float).reshape(-1, 3) for s in structures]))
        LAT = np.ascontiguousarray(np.stack([np.asarray(s["LAT"], float).reshape(3, 3) for s in structures]))
        S = len(structures)
        H = np.zeros(S)
        iters = np.zeros(S, np.int32)
        status = np.zeros(S, np.int32)
        self._check(self.lib.mb_relax_batch(self.h, S, nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I), _dp(LAT),
                                            _dp(X), p_gpa, urep, rlxt, mitr, fmax, _dp(H),
                                            iters.ctypes.data_as(_I), status.ctypes.data_as(_I)))
        ev, ms = ctypes.c_longlong(), ctypes.c_double()
        self._check(self.lib.mb_batch_stats(self.h, ctypes.byref(ev), ctypes.byref(ms)))
        wk = [ctypes.c_longlong() for _ in range(3)]
        self._check(self.lib.mb_batch_work(self.h, *(ctypes.byref(v) for v in wk)))
        offs = np.concatenate([[0], np.cumsum(nat)])
        return dict(H=H, X=[X[offs[k]:offs[k + 1]] for k in range(S)], LAT=LAT, iters=iters, status=status,
                    evals=int(ev.value), ms=float(ms.value), atom_evals=int(wk[0].value), pairs=int(wk[1].value),
                    triplets=int(wk[2].value))

    def efs_batch(self, structures, p_gpa=0.0, urep=0.0):
        """FP32 batched E/F/S of a list of dict(X, LAT, atmn), no relaxation.
        Returns dict(H[S], F list of [N,3], U[S,6])."""
        nat = np.array([len(s["atmn"]) for s in structures], np.int32)
        atmn = np.ascontiguousarray(np.concatenate([np.asarray(s["atmn"], np.int32) for s in structures]))
        X = np.ascontiguousarray(np.concatenate([np.asarray(s["X"], float).reshape(-1, 3) for s in structures]))
        LAT = np.ascontiguousarray(np.stack([np.asarray(s["LAT"], float).reshape(3, 3) for s in structures]))
        S = len(structures)
        H = np.zeros(S)
        F = np.zeros_like(X)
        U = np.zeros((S, 6))
        self._check(self.lib.mb_efs_batch(self.h, S, nat.ctypes.data_as(_I), atmn.ctypes.data_as(_I), _dp(LAT),
                                          _dp(X), p_gpa, urep, _dp(H), _dp(F), _dp(U)))
        offs = np.concatenate([[0], np.cumsum(nat)])
        return dict(H=H, F=[F[offs[k]:offs[k + 1]] for k in range(S)], U=U)

    def maxwell(self, atmn, T, seed=1):
        """Initial velocities of the reference's Maxwell() for model species atmn."""
        atmn = _i32(atmn)
        amu = np.array([self.lib.mb_atomic_mass(self.spcz[s]) for s in atmn])
        return maxwell(amu, T, seed)

    def md_nvt(self, X, LAT, atmn, V, T, dt=1.0, tau=25.0, nsteps=10, ND=3, NM=512, urep=0.0, xi=0.0,
               trace=True):
        """dict(X, V, xi, H[nsteps], K[nsteps]) -- NVT steps of Dynamics on the GPU."""
        atmn = _i32(atmn)
        N = len(atmn)
        X = _f64(X, 3 * N).copy()
        V = _f64(V, 3 * N).copy()
        LAT = _f64(LAT, 9)
        xi_c = ctypes.c_double(xi)
        Hs = np.zeros(max(nsteps, 1)) if trace else None
        Ks = np.zeros(max(nsteps, 1)) if trace else None
        self._check(self.lib.mb_md_nvt(self.h, N, NM, ND, atmn.ctypes.data_as(_I), _dp(LAT), _dp(X), _dp(V), T, dt,
                                       tau, nsteps, urep, ctypes.byref(xi_c), _dp(Hs), _dp(Ks)))
        out = dict(X=X.reshape(N, 3), V=V.reshape(N, 3), xi=xi_c.value)
        if trace:
            out["H"], out["K"] = Hs[:nsteps], Ks[:nsteps]
        return out

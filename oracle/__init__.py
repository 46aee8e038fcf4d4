"""CPU oracle for the MAISE neural-network potential path (test infrastructure).

Two checkers live here:

* ``Oracle`` -- the C restatement in ``oracle/oracle.c`` (built into
  ``oracle/liboracle.so`` by ``make -C oracle``), which restates the reference
  algorithm in plain FP64 C and materialises the reference's derivative
  blocks.
* ``RefOracle`` -- the reference MAISE sources themselves, compiled by
  ``make -C oracle ref`` into ``oracle/_ref/libmaise_ref.so`` with a GSL
  stand-in.  It exists only where the reference sources were available at
  build time.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  The product (``maise_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmaise_ref.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


# Where the build recipe looks for the reference MAISE sources: the
# MAISE_REFERENCE environment variable, else the read-only mount point of the
# build container.  Besides the build, only CPU tests that pin the oracle to
# the reference's own fixture files read it (and skip without it); nothing
# in the GPU tests, smoke() or the benchmark does.
_REFERENCE_MOUNT = "/root/reference"


def reference_dir():
    """Directory of the reference sources for the build recipe, or None."""
    d = os.environ.get("MAISE_REFERENCE") or _REFERENCE_MOUNT
    return d if os.path.isdir(os.path.join(d, "src")) else None


def build(ref: bool = True) -> None:
    """Compile the restatement (and the reference, when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    src = reference_dir() if ref else None
    if src:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8", "REF=" + src], check=True)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class Oracle:
    """ctypes view of oracle/liboracle.so for one model file."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build(ref=False)
            lib = ctypes.CDLL(ORACLE_SO)
            lib.orc_model_load.restype = ctypes.c_void_p
            lib.orc_model_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
            lib.orc_model_free.argtypes = [ctypes.c_void_p]
            lib.orc_model_info.argtypes = [ctypes.c_void_p, _I, _I, _I, _D, _I, _I]
            common = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I, _D, _D]
            lib.orc_nlist.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D,
                                      ctypes.c_double, _I, _I, _I, _D]
            lib.orc_descriptors_api.argtypes = common + [_D]
            lib.orc_fn_api.argtypes = common + [ctypes.c_int, _I, _I, _D, _D]
            lib.orc_vjp_api.argtypes = common + [_D, _D, _D]
            lib.orc_efs_api.argtypes = common + [ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D, _D, _D, _D]
            lib.orc_cell_volume.restype = ctypes.c_double
            lib.orc_cell_volume.argtypes = [_D]
            cls._lib = lib
        return cls._lib

    def __init__(self, model_path: str):
        err = ctypes.create_string_buffer(512)
        self.h = self.lib().orc_model_load(model_path.encode(), err)
        if not self.h:
            raise ValueError(err.value.decode())
        nspc, D, ng2, ng4 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        spcz = (ctypes.c_int * 10)()
        rc = ctypes.c_double()
        self.lib().orc_model_info(self.h, ctypes.byref(nspc), ctypes.byref(D), spcz, ctypes.byref(rc),
                                  ctypes.byref(ng2), ctypes.byref(ng4))
        self.nspc, self.D, self.rc = nspc.value, D.value, rc.value
        self.ng2, self.ng4 = ng2.value, ng4.value
        self.spcz = list(spcz)[: self.nspc]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().orc_model_free(self.h)
            self.h = None

    @staticmethod
    def _prep(X, LAT, atmn):
        X = np.ascontiguousarray(np.asarray(X, np.float64).reshape(-1)).copy()
        LAT = np.ascontiguousarray(np.asarray(LAT, np.float64).reshape(9))
        atmn = np.ascontiguousarray(np.asarray(atmn, np.int32))
        return X, LAT, atmn

    def nlist(self, X, LAT, atmn, ND, NM=512, rc=0.0):
        X, LAT, atmn = self._prep(X, LAT, atmn)
        N = len(atmn)
        nn = np.zeros(N, np.int32)
        nj = np.zeros(N * NM, np.int32)
        nic = np.zeros(N * NM * 3, np.int32)
        nr = np.zeros(N * NM)
        rv = self.lib().orc_nlist(self.h, N, NM, ND, _dp(LAT), _dp(X), rc, _ip(nn), _ip(nj), _ip(nic), _dp(nr))
        if rv:
            raise RuntimeError("neighbour overflow")
        return nn, nj.reshape(N, NM), nic.reshape(N, NM, 3), nr.reshape(N, NM), X.reshape(N, 3)

    def descriptors(self, X, LAT, atmn, ND, NM=512):
        X, LAT, atmn = self._prep(X, LAT, atmn)
        N = len(atmn)
        G = np.zeros(N * self.D)
        if self.lib().orc_descriptors_api(self.h, N, NM, ND, _ip(atmn), _dp(LAT), _dp(X), _dp(G)):
            raise RuntimeError("neighbour overflow")
        return G.reshape(N, self.D)

    def fn(self, X, LAT, atmn, ND, atom, NM=512):
        """Derivative blocks of one atom: (dni, Fn[dnn+1, D, 3], Sn[D, 6])."""
        X, LAT, atmn = self._prep(X, LAT, atmn)
        N = len(atmn)
        dnn = ctypes.c_int()
        dni = np.zeros(NM + 1, np.int32)
        Fn = np.zeros((NM + 1) * self.D * 3)
        Sn = np.zeros(self.D * 6)
        if self.lib().orc_fn_api(self.h, N, NM, ND, _ip(atmn), _dp(LAT), _dp(X), atom, ctypes.byref(dnn),
                                 _ip(dni), _dp(Fn), _dp(Sn)):
            raise RuntimeError("neighbour overflow")
        k = dnn.value
        return dni[:k].copy(), Fn[: (k + 1) * self.D * 3].reshape(k + 1, self.D, 3), Sn.reshape(self.D, 6)

    def vjp(self, X, LAT, atmn, ND, g, NM=512):
        X, LAT, atmn = self._prep(X, LAT, atmn)
        N = len(atmn)
        g = np.ascontiguousarray(np.asarray(g, np.float64).reshape(N * self.D))
        F = np.zeros(3 * N)
        U = np.zeros(6)
        if self.lib().orc_vjp_api(self.h, N, NM, ND, _ip(atmn), _dp(LAT), _dp(X), _dp(g), _dp(F), _dp(U)):
            raise RuntimeError("neighbour overflow")
        return F.reshape(N, 3), U

    def efs(self, X, LAT, atmn, ND, urep=0.0, p_gpa=0.0, forces=True, NM=512):
        """dict(E, H, EA, F, U, X) following CELL_FRC / CELL_ENE."""
        X, LAT, atmn = self._prep(X, LAT, atmn)
        N = len(atmn)
        E, H = ctypes.c_double(), ctypes.c_double()
        EA = np.zeros(N)
        F = np.zeros(3 * N)
        U = np.zeros(6)
        if self.lib().orc_efs_api(self.h, N, NM, ND, _ip(atmn), _dp(LAT), _dp(X), urep, p_gpa, int(forces),
                                  ctypes.byref(E), ctypes.byref(H), _dp(EA), _dp(F), _dp(U)):
            raise RuntimeError("neighbour overflow")
        return dict(E=E.value, H=H.value, EA=EA, F=F.reshape(N, 3), U=U, X=X.reshape(N, 3))


class RefOracle:
    """ctypes view of the reference sources compiled under oracle/_ref.

    The reference keeps global state (one model at a time, arrays sized by the
    first call); the harness re-initialises when the model directory changes
    or a larger structure arrives.  model_dir must hold a file named 'model'.
    """

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not ref_available():
                raise FileNotFoundError("oracle/_ref/libmaise_ref.so was not built (needs the reference sources)")
            lib = ctypes.CDLL(REF_SO)
            c_i, c_d = ctypes.c_int, ctypes.c_double
            lib.ref_efs.restype = c_d
            lib.ref_efs.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, _D, _D, _D, _D]
            lib.ref_energy.restype = c_d
            lib.ref_energy.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d]
            lib.ref_descriptors.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, _D]
            lib.ref_fn.argtypes = [c_i, _I, _I, _D, _D]
            lib.ref_positions.argtypes = [c_i, _D]
            lib.ref_relax.restype = c_d
            lib.ref_relax.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, c_i, c_i, c_d, _L]
            lib.ref_nvt.restype = c_d
            lib.ref_nvt.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, _D, c_i, ctypes.c_long, c_d,
                                    c_d, c_d, c_i, c_d, _D, _D, c_d]
            lib.ref_maxwell.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, ctypes.c_long, c_d, _D]
            lib.ref_sizes.argtypes = [_I]
            lib.ref_nlist.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, c_i, _I, _I, _I, _D]
            lib.ref_read_cell.argtypes = [ctypes.c_char_p, c_i, _I, _D, _D, _I]
            lib.ref_read_oszi.restype = c_d
            lib.ref_rdf.argtypes = [ctypes.c_char_p, c_i, c_i, c_i, c_i, _I, _D, _D, c_d, c_d, c_d, c_i, _D]
            lib.ref_efile_read.argtypes = [ctypes.c_char_p, c_i, _I, _D, _I, _D]
            lib.ref_efile_block.argtypes = [c_i, _I, _I, _D, _D]
            lib.ref_efile_sn.argtypes = [_D, _D]
            lib.ref_train_terms.restype = c_d
            lib.ref_train_terms.argtypes = [c_i, c_i, c_i, c_i, _D, _D, _D, c_d, c_d, c_d, _D, _D, _D]
            lib.ref_read_oszi.argtypes = [ctypes.c_char_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, model_dir: str, nthreads: int = 0):
        self.dir = os.path.abspath(model_dir).encode()
        self.np = nthreads or os.cpu_count() or 1

    def efs(self, X, LAT, atmn, ND, urep=0.0, p_gpa=0.0, NM=512, XT=1):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        N = len(atmn)
        F = np.zeros(3 * N)
        S = np.zeros(6)
        EA = np.zeros(N)
        E = ctypes.c_double()
        H = self.lib().ref_efs(self.dir, N, NM, ND, self.np, XT, _ip(atmn), _dp(LAT), _dp(X), urep, p_gpa,
                               _dp(F), _dp(S), _dp(EA), ctypes.byref(E))
        Xw = np.zeros(3 * N)
        self.lib().ref_positions(N, _dp(Xw))
        return dict(E=E.value, H=H, EA=EA, F=F.reshape(N, 3), U=S, X=Xw.reshape(N, 3))

    def energy(self, X, LAT, atmn, ND, urep=0.0, p_gpa=0.0, NM=512):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        return self.lib().ref_energy(self.dir, len(atmn), NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), urep, p_gpa)

    def descriptors(self, X, LAT, atmn, ND, NM=512, D=None):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        N = len(atmn)
        G = np.zeros(N * 4096)
        D = self.lib().ref_descriptors(self.dir, N, NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), _dp(G))
        return G[: N * D].reshape(N, D)

    def fn(self, atom, D, NM=512):
        dnn = ctypes.c_int()
        dni = np.zeros(NM + 1, np.int32)
        Fn = np.zeros((NM + 1) * D * 3)
        Sn = np.zeros(D * 6)
        self.lib().ref_fn(atom, ctypes.byref(dnn), _ip(dni), _dp(Fn), _dp(Sn))
        k = dnn.value
        return dni[:k].copy(), Fn[: (k + 1) * D * 3].reshape(k + 1, D, 3), Sn.reshape(D, 6)

    def relax(self, X, LAT, atmn, ND, rlxt=3, mitr=100, etol=1e-6, urep=0.0, p_gpa=0.0, NM=512):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        LAT = LAT.copy()
        counts = np.zeros(3, np.int64)
        # CELL_MIN writes its CONTCAR into the working directory: run it in a
        # scratch directory (the model path is absolute)
        import shutil
        import tempfile
        old = os.getcwd()
        scratch = tempfile.mkdtemp(prefix="ref_relax_")
        os.chdir(scratch)
        try:
            H = self.lib().ref_relax(self.dir, len(atmn), NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), urep,
                                     p_gpa, rlxt, mitr, etol, counts.ctypes.data_as(_L))
        finally:
            os.chdir(old)
            shutil.rmtree(scratch, ignore_errors=True)
        return dict(H=H, X=X.reshape(-1, 3), LAT=LAT.reshape(3, 3), n_energy=int(counts[0]),
                    n_force=int(counts[1]), iters=int(counts[2]))

    def nvt(self, X, LAT, atmn, ND, T, dt, tau, nsteps, seed=1, V=None, urep=0.0, NM=512, xi=0.0):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        N = len(atmn)
        vin = V is not None
        V = np.ascontiguousarray(np.asarray(V, np.float64).reshape(-1)).copy() if vin else np.zeros(3 * N)
        Hs = np.zeros(nsteps)
        Ks = np.zeros(nsteps)
        xi = self.lib().ref_nvt(self.dir, N, NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), _dp(V), int(vin),
                                seed, T, dt, tau, nsteps, urep, _dp(Hs), _dp(Ks), xi)
        return dict(X=X.reshape(N, 3), V=V.reshape(N, 3), H=Hs, K=Ks, xi=xi)

    def nlist(self, X, LAT, atmn, ND, NM=512, cap=None):
        """LIST's neighbour list: (nn[N], nj[N,cap], nic[N,cap,3] integer images, X wrapped)."""
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        N = len(atmn)
        cap = cap or NM
        nn = np.zeros(N, np.int32)
        nj = np.zeros(N * cap, np.int32)
        nic = np.zeros(N * cap * 3, np.int32)
        Xw = np.zeros(3 * N)
        if self.lib().ref_nlist(self.dir, N, NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), cap, _ip(nn), _ip(nj),
                                _ip(nic), _dp(Xw)):
            raise RuntimeError("more neighbours than cap")
        return nn, nj.reshape(N, cap), nic.reshape(N, cap, 3), Xw.reshape(N, 3)

    def read_cell(self, path, cap=4096):
        """READ_CELL of a POSCAR/CONTCAR (a model must have been loaded by an
        earlier call): dict(LAT[3,3], X[N,3] Cartesian, atmn[N])."""
        N = ctypes.c_int()
        lat = np.zeros(9)
        X = np.zeros(3 * cap)
        atmn = np.zeros(cap, np.int32)
        rv = self.lib().ref_read_cell(os.fsencode(path), cap, ctypes.byref(N), _dp(lat), _dp(X), _ip(atmn))
        if rv:
            raise RuntimeError(f"READ_CELL failed on {path} ({rv})")
        n = N.value
        return dict(LAT=lat.reshape(3, 3), X=X[: 3 * n].reshape(n, 3), atmn=atmn[:n].copy())

    def rdf(self, X, LAT, atmn, ND, nspc, rmin=5.8, rmax=6.0, sigma=0.008, normalise=True, NM=512):
        """RDF of RANK_TR's duplicate test: [npair, 3000] for species pairs m <= n."""
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        npair = nspc * (nspc + 1) // 2
        out = np.zeros(npair * 3000)
        nb = self.lib().ref_rdf(self.dir, len(atmn), NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), rmin, rmax,
                                sigma, int(normalise), _dp(out))
        return out.reshape(npair, nb)

    @classmethod
    def read_efile(cls, directory, index, maxN=4096, maxD=1024):
        """A descriptor file read by the reference's LNK_IN: dict(EFS, D, N, NF,
        E, p, DE, atmn, Cn, blocks {atom: (dni, F, Fn[dnn+1, D, 3])}, S, Sn)."""
        lib = cls.lib()
        hdr = np.zeros(4, np.int32)
        eh = np.zeros(3)
        atmn = np.zeros(maxN, np.int32)
        Cn = np.zeros(maxN * maxD)
        if lib.ref_efile_read(os.fsencode(directory), index, _ip(hdr), _dp(eh), _ip(atmn), _dp(Cn)):
            raise RuntimeError("LNK_IN failed")
        EFS, D, N, NF = (int(v) for v in hdr)
        out = dict(EFS=EFS, D=D, N=N, NF=NF, E=eh[0], p=eh[1], DE=eh[2], atmn=atmn[:N].copy(),
                   Cn=Cn[:N * D].reshape(N, D).copy(), blocks={})
        if EFS in (1, 3):
            for i in range(N):
                dnn = ctypes.c_int()
                dni = np.zeros(1024, np.int32)
                F = np.zeros(3)
                fn = np.zeros(1025 * D * 3)
                if lib.ref_efile_block(i, ctypes.byref(dnn), _ip(dni), _dp(F), _dp(fn)) == 0:
                    k = dnn.value
                    out["blocks"][i] = (dni[:k].copy(), F, fn[:(k + 1) * D * 3].reshape(k + 1, D, 3))
        if EFS in (2, 3):
            sn = np.zeros(N * D * 6)
            S = np.zeros(6)
            lib.ref_efile_sn(_dp(sn), _dp(S))
            out["S"], out["Sn"] = S, sn.reshape(N, D, 6)
        return out

    @classmethod
    def train_terms(cls, directory, index, V, nspc, D, h1, h2, rmin, dr, WE=1.0, WF=1.0, w=1.0):
        """The training terms of descriptor file `index` through the reference's
        LNK_IN, ADJT_LNK, FRC_ANN_PARA, DE_ANN_PARA and DF_ANN_PARA:
        (E, f[N, 3] on the marked atoms, gE, gF) with the gradient terms in
        dfunc_gsl's order, not yet divided by the number of structures."""
        lib = cls.lib()
        hdr = np.zeros(4, np.int32)
        eh = np.zeros(3)
        atmn = np.zeros(4096, np.int32)
        Cn = np.zeros(4096 * 1024)
        if lib.ref_efile_read(os.fsencode(directory), index, _ip(hdr), _dp(eh), _ip(atmn), _dp(Cn)):
            raise RuntimeError("LNK_IN failed")
        N = int(hdr[2])
        V = np.ascontiguousarray(V, float)
        rmin = np.ascontiguousarray(rmin, float).reshape(-1)
        dr = np.ascontiguousarray(dr, float).reshape(-1)
        f = np.zeros(3 * N)
        gE = np.zeros(len(V))
        gF = np.zeros(len(V))
        E = lib.ref_train_terms(nspc, D, h1, h2, _dp(V), _dp(rmin), _dp(dr), WE, WF, w, _dp(f), _dp(gE), _dp(gF))
        return float(E), f.reshape(N, 3), gE, gF

    def read_oszi(self, path):
        """The enthalpy Read_OSZI takes from an OSZICAR."""
        return float(self.lib().ref_read_oszi(os.fsencode(path)))

    def maxwell(self, X, LAT, atmn, ND, T, seed=1, NM=512):
        X, LAT, atmn = Oracle._prep(X, LAT, atmn)
        N = len(atmn)
        V = np.zeros(3 * N)
        self.lib().ref_maxwell(self.dir, N, NM, ND, self.np, _ip(atmn), _dp(LAT), _dp(X), seed, T, _dp(V))
        return V.reshape(N, 3)

    def sizes(self):
        out = (ctypes.c_int * 10)()
        self.lib().ref_sizes(out)
        return list(out)

"""mb_efs_noalloc: the entry point for callers that own all device memory and
cannot let the library allocate (see include/maise_b200.h).  It must give the
energy, forces and virial of the CPU oracle (the FP64 restatement of the
reference's CELL_FRC) and of mb_efs, for inputs and outputs held in the
caller's device buffers, on consecutive calls sharing its fixed scratch
array.  Collected last so that a run stopping at the first failure has run
every other test already."""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from oracle import Oracle

pytestmark = pytest.mark.gpu

E_RTOL = 1e-10
F_ATOL = 1e-9


def _model(tmp_path, w, name):
    from maise_b200 import models

    d = tmp_path / name
    d.mkdir()
    models.random_model(str(d / "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3), seed=3)
    return str(d / "model")


def _call_noalloc(pot, w, NM):
    import torch

    lib = pot.lib
    lib.mb_efs_noalloc.restype = ctypes.c_int
    lib.mb_efs_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p]
    N = len(w["atmn"])
    x = torch.tensor(np.asarray(w["X"], float).reshape(-1), dtype=torch.float64, device="cuda")
    spc = torch.tensor(np.asarray(w["atmn"], np.int32), dtype=torch.int32, device="cuda")
    frc = torch.full((3 * N,), np.nan, dtype=torch.float64, device="cuda")
    out = torch.full((8,), np.nan, dtype=torch.float64, device="cuda")
    lat = np.ascontiguousarray(np.asarray(w["LAT"], float).reshape(9))
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.mb_efs_noalloc(pot.h, N, NM, 3, lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), x.data_ptr(),
                            spc.data_ptr(), 0.0, 0.0, frc.data_ptr(), out.data_ptr(), stream)
    assert rc == 0, lib.mb_last_error().decode()
    torch.cuda.synchronize()
    x_after = x.cpu().numpy().reshape(-1, 3)
    np.testing.assert_array_equal(x_after, np.asarray(w["X"], float))  # inputs are not modified
    o = out.cpu().numpy()
    return dict(E=o[0], H=o[1], U=o[2:8], F=frc.cpu().numpy().reshape(N, 3))


def test_noalloc_matches_mb_efs_on_consecutive_calls(tmp_path):
    import maise_b200
    from maise_b200 import workloads

    big = workloads.random_alloy(n=5, a=3.8, seed=21, jitter=0.08)          # 500 atoms, cell-list path
    small = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=22)      # 32 atoms, all-pairs path
    cases = [("big", big, _model(tmp_path, big, "big")), ("small", small, _model(tmp_path, small, "small"))]
    pots = {name: maise_b200.Potential(path) for name, _, path in cases}
    oracle = {name: Oracle(path).efs(w["X"], w["LAT"], w["atmn"], 3, NM=200) for name, w, path in cases}
    # two calls in a row through the shared scratch, then the first structure again
    for name, w, _ in cases + cases[:1]:
        pot = pots[name]
        got = _call_noalloc(pot, w, NM=200)
        ref = oracle[name]
        assert got["H"] == pytest.approx(ref["H"], rel=E_RTOL)
        assert got["E"] == pytest.approx(ref["E"], rel=E_RTOL)
        np.testing.assert_allclose(got["F"], ref["F"], atol=F_ATOL)
        np.testing.assert_allclose(got["U"], ref["U"], rtol=E_RTOL, atol=1e-9)
        want = pot.efs(w["X"], w["LAT"], w["atmn"], ND=3, NM=200)
        assert got["H"] == pytest.approx(want["H"], rel=E_RTOL)
        assert got["E"] == pytest.approx(want["E"], rel=E_RTOL)
        np.testing.assert_allclose(got["F"], want["F"], atol=F_ATOL)
        np.testing.assert_allclose(got["U"], want["U"], rtol=E_RTOL, atol=1e-9)
    for p in pots.values():
        p.close()


def test_noalloc_rejects_oversized_input(tmp_path):
    import maise_b200
    from maise_b200 import workloads

    w = workloads.fcc_supercell(n=2, seed=1)
    pot = maise_b200.Potential(_model(tmp_path, w, "m"))
    lib = pot.lib
    lib.mb_efs_noalloc.restype = ctypes.c_int
    lib.mb_efs_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p]
    lat = np.ascontiguousarray(np.asarray(w["LAT"], float).reshape(9))
    rc = lib.mb_efs_noalloc(pot.h, 5000, 200, 3, lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            1, 1, 0.0, 0.0, 1, 1, 0)
    assert rc == 5  # MB_ERR_CAPACITY
    assert "2048" in lib.mb_last_error().decode()
    pot.close()

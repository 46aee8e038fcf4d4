"""Build libmaise_b200.so in-tree: C host objects (gcc) + sm_100a kernels (nvcc).

    python -m maise_b200._build            # incremental
    python -m maise_b200._build --clean

The library lands in maise_b200/libmaise_b200.so so that it travels with the
source tree; objects go to maise_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmaise_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["host/mb_model.c", "host/mb_bfgs.c", "host/mb_core.c", "host/mb_call_maise.c", "host/mb_batch.c",
                "host/mb_surrogate.c", "host/mb_evos.c", "host/mb_parse.c"]
CUDA_SOURCES = ["cuda/mb_kernels.cu", "cuda/mb_batch.cu", "cuda/mb_diag.cu", "cuda/mb_static.cu",
                "cuda/mb_surrogate.cu", "cuda/mb_rdf.cu", "cuda/mb_train.cu"]
HEADERS = ["mb_internal.h", "host/mb_bfgs.h", "host/mb_batch.h", "host/mb_surrogate_k.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))]
    headers += [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    for src in HOST_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _newer(obj, [path] + headers):
            _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                  "-I" + os.path.join(CUDA, "include"), "-c", path, "-o", obj])
        objs.append(obj)
    for src in CUDA_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if _newer(obj, [path] + headers):
            cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c", path, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(obj)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lm"])
    return LIB


def clean() -> None:
    shutil.rmtree(OBJ, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))

"""Shared fixtures.  Tests marked `gpu` need a B200 and the built library;
everything else runs on the CPU (oracle, host logic, library exports)."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and libmaise_b200.so")


@pytest.fixture(scope="session", autouse=True)
def built_oracle():
    """The C restatement is always buildable from source (gcc)."""
    so = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return so


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=True)


def write_model_dir(tmp_path, text, sub="m"):
    d = tmp_path / sub
    d.mkdir(parents=True, exist_ok=True)
    (d / "model").write_text(str(text))
    return str(d)


@pytest.fixture(scope="session")
def parse_golden():
    return load_golden("parse_cuag.npz")


@pytest.fixture(scope="session")
def parse_model_dir(tmp_path_factory, parse_golden):
    """A Cu-Ag model with the parse test's 30-function basis (82 inputs) and
    random weights: descriptors do not depend on the weights."""
    from maise_b200 import models

    d = tmp_path_factory.mktemp("parse_model")
    D = 82
    lo = np.zeros((2, D))
    hi = np.ones((2, D)) * 100.0
    models.write_model(str(d / "model"), [29, 47], (D, 10, 10), models.random_nets(2, (D, 10, 10), 5), lo, hi,
                       str(parse_golden["basis"]))
    return str(d)


def parse_structures(g):
    """Yield (index, LAT, X, atmn, G) of the golden parse set."""
    off = g["offsets"]
    for s in range(len(g["names"])):
        a, b = off[s], off[s + 1]
        yield s, g["lat"][s], g["x"][a:b], g["atmn"][a:b], g["G"][a:b]


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False

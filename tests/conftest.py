"""Shared fixtures.  `-m "not gpu"` runs the oracle pins and host logic on CPU;
`-m gpu` runs the parity tests through the C ABI on a B200."""
from __future__ import annotations

import importlib.util
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def load_p2z():
    name = "p2z_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "p2z-tests_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def p2z():
    return load_p2z()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O


def read_seed(path):
    lines = [l.split() for l in open(path) if l.strip()]
    t = lines[0]
    trk = ([float(v) for v in t[:6]], [float(v) for v in t[6:27]], int(t[27]))
    hits = [([float(v) for v in l[:3]], [float(v) for v in l[3:9]]) for l in lines[1:]]
    return trk, hits


@pytest.fixture(scope="session")
def kat_seed():
    return read_seed(GOLDEN / "kat_seed.txt")


@pytest.fixture(scope="session")
def readme_seed():
    return read_seed(GOLDEN / "readme_seed.txt")


@pytest.fixture(scope="session")
def ctx(p2z):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = p2z.Context(0)
    yield c
    c.close()


# ---------------------------------------------------------------------------
# comparison metrics (stated once, used by every parity test)
# ---------------------------------------------------------------------------
# Parameters: |a - b| / max(|b|, floor_p), with floors for the elements that
# cross zero or are small: x, y, z in cm (1), ipt in 1/GeV (1e-3), phi and
# theta in rad (1, 1e-2).
PAR_FLOOR = np.array([1.0, 1.0, 1.0, 1e-3, 1.0, 1e-2])
LIVE = [0, 1, 2, 6, 7, 9, 10, 11, 13, 14, 15, 16, 18, 19, 20]


def par_rel(a, b):
    return np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.maximum(np.abs(np.asarray(b, np.float64)),
                                                                                      PAR_FLOOR)


def cov_rel(a, ref):
    """Covariance error normalised by the diagonal: |dC_ij| / sqrt(C_ii C_jj) of ref."""
    a = np.asarray(a, np.float64)
    ref = np.asarray(ref, np.float64)
    out = np.zeros(a.shape)
    for i in range(6):
        for j in range(i + 1):
            k = i * (i + 1) // 2 + j
            ii, jj = i * (i + 1) // 2 + i, j * (j + 1) // 2 + j
            s = np.sqrt(np.abs(ref[:, ii] * ref[:, jj]))
            out[:, k] = np.abs(a[:, k] - ref[:, k]) / np.where(s > 0, s, 1.0)
    return out

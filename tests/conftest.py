"""Shared test set-up: the `gpu` marker, the package loader and fixtures."""
import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "blocked-linearized-coordinate_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    """Import the engine's Python binding under the name blco_b200."""
    if "blco_b200" in sys.modules:
        return sys.modules["blco_b200"]
    spec = importlib.util.spec_from_file_location(
        "blco_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["blco_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def golden_index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def golden_case(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def formula_factors(dims, rank):
    """The factor matrices tests/golden/make_golden.py used (not stored)."""
    out = []
    for m, d in enumerate(dims):
        i = np.arange(int(d), dtype=np.int64)[:, None]
        r = np.arange(rank, dtype=np.int64)[None, :]
        out.append(0.25 + ((i * 2654435761 + r * 40503 + m * 97) % 1000003) / 1000003.0)
    return out


def unique_coords(rng, dims, nnz, zipf=None):
    """nnz distinct coordinates (vectorised; uniform or per-mode Zipf)."""
    dims = [int(d) for d in dims]
    mult = np.cumprod([1] + dims[::-1][:-1])[::-1].astype(np.int64)
    have = np.zeros(0, dtype=np.int64)
    while len(have) < nnz:
        m = 2 * (nnz - len(have)) + 64
        cols = []
        for d in dims:
            if zipf is None:
                cols.append(rng.integers(0, d, size=m))
            else:
                w = 1.0 / np.arange(1, d + 1, dtype=np.float64) ** zipf
                cdf = np.cumsum(w / w.sum())
                cols.append(np.minimum(np.searchsorted(cdf, rng.random(m)), d - 1))
        lin = sum(c.astype(np.int64) * mu for c, mu in zip(cols, mult))
        have = np.concatenate([have, lin])
        _, first = np.unique(have, return_index=True)
        have = have[np.sort(first)]
    have = have[:nnz]
    out = np.zeros((len(dims), nnz), dtype=np.uint64)
    rem = have.copy()
    for n, mu in enumerate(mult):
        out[n] = (rem // mu).astype(np.uint64)
        rem = rem % mu
    return out


def unique_coords_wide(rng, dims, nnz):
    """nnz distinct uniform coordinates for modes whose product exceeds
    2^63 (no linearized integer key), in first-drawn order."""
    dims = [int(d) for d in dims]
    c = np.stack([rng.integers(0, d, size=2 * nnz + 64, dtype=np.uint64) for d in dims])
    _, first = np.unique(c, axis=1, return_index=True)
    first = np.sort(first)
    assert len(first) >= nnz
    return np.ascontiguousarray(c[:, first[:nnz]])


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def blco():
    return load_package()

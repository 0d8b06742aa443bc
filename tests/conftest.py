"""Shared test setup: import paths, the `gpu` marker and helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "chem-kumo_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_points(g) -> np.ndarray:
    """Cartesian points of the sampled grid indices of a golden fixture."""
    idx = g["index"]
    counts = g["counts"]
    ny, nz = int(counts[1]), int(counts[2])
    i = idx // (ny * nz)
    j = (idx // nz) % ny
    k = idx % nz
    ijk = np.stack([i, j, k], 1).astype(float)
    return g["origin"][None, :] + ijk @ g["steps"].T


def scaled_error(a: np.ndarray, ref: np.ndarray) -> float:
    """max |a - ref| / max(1, max |ref|) (tests/density_screening_test.cpp:137-150 of chem-kumo)."""
    if ref.size == 0:
        return 0.0
    return float(np.max(np.abs(a - ref)) / max(1.0, float(np.max(np.abs(ref)))))


@pytest.fixture(scope="session")
def synth_cache(tmp_path_factory):
    d = tmp_path_factory.mktemp("synth")
    os.environ["KUMO_SYNTH_CACHE"] = str(d)
    return str(d)

"""Shared test setup: import paths, the `gpu` marker, scene helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-path-tracer_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); runs the library's kernels")
    # temporary files of the tests stay inside the checkout (ignored by git)
    if not config.option.basetemp:
        config.option.basetemp = os.path.join(ROOT, ".pytest_tmp")


@pytest.fixture(scope="session")
def cuda():
    """Every GPU test depends on this: a missing device is a failure, not a skip."""
    import torch

    assert torch.cuda.is_available(), "gpu-marked test run without a CUDA device"
    major, minor = torch.cuda.get_device_capability()
    assert (major, minor) == (10, 0), f"libcpt.so is built for sm_100a; device is sm_{major}{minor}"
    torch.cuda.set_device(0)
    return torch.device("cuda:0")


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: d[k] for k in d.files}


GOLDEN_CASES = ["random2k_30", "random2k_63", "ties1k_30", "sphere_63", "tiny2_30"]


def quantized(tris, step):
    t = tris.copy()
    for f in ("v0", "v1", "v2"):
        t[f] = (np.round(t[f] / step) * step).astype(np.float32)
    return t


def rays_at(tris, n, seed, spread=(-0.3, 1.3)):
    rng = np.random.default_rng(seed)
    o = rng.uniform(spread[0], spread[1], (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    pick = rng.integers(0, len(tris), n // 2)
    cen = (tris["v0"][pick] + tris["v1"][pick] + tris["v2"][pick]) / 3.0
    d[: n // 2] = (cen - o[: n // 2]).astype(np.float32)
    d[n // 2: n // 2 + n // 8, 1] = 0.0
    return np.concatenate([o, d], 1).astype(np.float32)

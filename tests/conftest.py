import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a) and libhdb_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    O.lib()
    return O


@pytest.fixture(scope="session")
def libpath():
    from gpu_hdbscan_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def ctx(libpath):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpu_hdbscan_b200 import Context
    c = Context(0)
    yield c
    c.close()


def blobs(n, d, seed, blobs=5, noise=0.05, spread=10.0, sigma=1.0):
    """Small seeded blob set for parity cases."""
    rng = np.random.default_rng(seed)
    n_noise = int(n * noise)
    centers = rng.uniform(-spread, spread, size=(blobs, d))
    lab = rng.integers(0, blobs, size=n - n_noise)
    X = centers[lab] + rng.normal(0, sigma, size=(n - n_noise, d))
    lo, hi = X.min(0), X.max(0)
    X = np.concatenate([X, rng.uniform(lo, hi, size=(n_noise, d))]).astype(np.float32)
    return X[rng.permutation(n)]

"""Shared test setup: import paths, the `gpu` marker, device helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "era-boojum-cuda_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

P = 0xFFFFFFFF00000001


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def uniform(rng: np.random.Generator, size) -> np.ndarray:
    """u64 uniform in [0, p)."""
    return rng.integers(0, P, size=size, dtype=np.uint64)


def raw_u64(rng: np.random.Generator, size) -> np.ndarray:
    """Any u64 word, like the reference test's rng.gen() (src/ntt.rs:424)."""
    return rng.integers(0, 2**64, size=size, dtype=np.uint64)


def to_dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def to_host(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


@pytest.fixture(scope="session")
def gpu_ctx():
    """Library context on cuda:0 for the whole session."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import bc_ntt

    torch.cuda.set_device(0)
    ctx = bc_ntt.Context.create(12, 12)
    yield ctx
    torch.cuda.synchronize()

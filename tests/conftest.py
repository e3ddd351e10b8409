"""Shared fixtures: markers, in-tree builds of liboux.so and the CPU oracle."""
import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_builds():
    from ouxsbli_b200 import build as b
    if not b.LIB.exists():
        b.build()
    from oracle import oracle
    oracle.build()


_ensure_builds()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return "cuda:0"

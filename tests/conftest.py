"""Shared fixtures.  `gpu`-marked tests need a CUDA device and the built
library; everything else runs on the CPU (oracle, host logic, ABI checks)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def built_lib():
    from rspacedist_b200 import build, lib
    build.build()
    return lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def make_si8(n=32, sigma=0.0, seed=0):
    from rspacedist_b200 import system as S
    ds = S.load_dataset("si_paw")
    pos = S.diamond_positions(1, 10.26, sigma, seed)
    return S.make_cell(10.26, n, pos, ds)


def make_c8(n=24, sigma=0.03, seed=2):
    from rspacedist_b200 import system as S
    ds = S.load_dataset("c_ncps")
    pos = S.diamond_positions(1, 6.74, sigma, seed)
    return S.make_cell(6.74, n, pos, ds)


@pytest.fixture(scope="session")
def si8(built_lib):
    return make_si8(32, 0.05, 4)


@pytest.fixture(scope="session")
def c8(built_lib):
    return make_c8(24)

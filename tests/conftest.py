"""Shared pytest set-up: the ``gpu`` marker, the repository root on sys.path, golden loaders."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def ref_or_skip():
    from oracle.bindings import Reference, reference_available
    if not reference_available():
        pytest.skip("reference build oracle/_ref/libt3d_ref.so not present")
    Reference.set_threads(1)
    return Reference

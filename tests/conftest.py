import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "nbody-fmm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle import REF_SO, RefLib

    if not os.path.exists(REF_SO):
        pytest.skip("reference not built (oracle/_ref/libref.so)")
    return RefLib()


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def tree_pairs_set(tree, d, kind):
    tk, sk = tree["pairs"][d][kind]
    return set(zip(np.asarray(tk).tolist(), np.asarray(sk).tolist()))

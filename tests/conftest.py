import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def O():
    import oracle_py

    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def mg():
    return importlib.import_module("mg-alphagcd_b200")


@pytest.fixture(scope="session")
def ctx(mg):
    c = mg.Context(0)
    yield c
    c.close()


def two_cliques(k=5):
    """Two k-cliques joined by one edge (hand-checkable fixture)."""
    u, v = [], []
    for base in (0, k):
        for i in range(k):
            for j in range(i + 1, k):
                u.append(base + i)
                v.append(base + j)
    u.append(k - 1)
    v.append(k)
    return 2 * k, np.array(u), np.array(v)


def ring_of_cliques(cliques=6, k=4):
    u, v = [], []
    for c in range(cliques):
        b = c * k
        for i in range(k):
            for j in range(i + 1, k):
                u.append(b + i)
                v.append(b + j)
        u.append(b + k - 1)
        v.append(((c + 1) % cliques) * k)
    return cliques * k, np.array(u), np.array(v)


def star(k=12):
    return k + 1, np.zeros(k, np.int64), np.arange(1, k + 1)


def path(n=20):
    return n, np.arange(n - 1), np.arange(1, n)


def boundary_degree_graph():
    """Vertices whose degrees sit on every bin threshold of the three schemes."""
    degs = [0, 1, 2, 3, 4, 5, 8, 9, 16, 17, 32, 33, 64, 65, 128, 129, 256, 257, 512, 513, 1024, 1025, 2048,
            2049, 4094, 4095, 4096, 4097, 8192, 8193, 12288, 12289]
    n_centers = len(degs)
    leaves = max(degs) + 1
    u, v = [], []
    for i, d in enumerate(degs):
        for j in range(d):
            u.append(i)
            v.append(n_centers + j)
    return n_centers + leaves, np.array(u), np.array(v)


def cuda_available() -> bool:
    import torch

    return torch.cuda.is_available()

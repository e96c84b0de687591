"""Shared fixtures.  GPU tests are marked ``gpu`` (run with ``-m gpu`` on a
B200); everything else runs on the CPU."""
import os
import sys
import warnings

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libvortrace_b200.so")
    config.addinivalue_line("markers", "slow: long-running (large clouds)")


@pytest.fixture(scope="session")
def galaxy():
    """The reference's golden case: snapshot + expected 128x128 projection."""
    g = np.load(os.path.join(GOLDEN, "galaxy_interaction.npz"))
    return {"pos": g["pos"], "dens": g["dens"], "box_size": float(g["box_size"]),
            "proj": g["proj"]}


@pytest.fixture(scope="session")
def small_walks():
    """Segment lists and reductions produced by the reference module."""
    z = np.load(os.path.join(GOLDEN, "small_walks.npz"))
    cases = {}
    for key in z.files:
        case, rest = key.split("/", 1)
        cases.setdefault(case, {})[rest] = z[key]
    return cases


@pytest.fixture(scope="session")
def tie_walks():
    """Exact-tie geometry produced by the reference module: segment lists of
    lattice clouds, k-NN order of tied generators, Slice/BruteProjection
    samples on lattice faces (tests/golden/make_golden.py, ``ties``)."""
    z = np.load(os.path.join(GOLDEN, "tie_walks.npz"))
    cases = {}
    for key in z.files:
        case, rest = key.split("/", 1)
        cases.setdefault(case, {})[rest] = z[key]
    return cases


@pytest.fixture(scope="session")
def ref_module():
    from oracle import oracle as O
    return O.load_reference_module()


def make_cubic_lattice(n=5):
    """n x n x n integer lattice with unit fields and volumes (the reference
    tests' fixture)."""
    c = np.arange(n, dtype=np.float64)
    xx, yy, zz = np.meshgrid(c, c, c, indexing="ij")
    pos = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    return pos, np.ones(len(pos)), np.ones(len(pos)), [-0.5, n - 0.5] * 3


@pytest.fixture
def quiet():
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        yield

"""Slice and BruteProjection (nearest-cell sampling on grids) against the
reference module's own outputs (tests/golden/slice_brute.npz, made by
tests/golden/make_golden.py from Cvortrace.Slice / Cvortrace.BruteProjection):
bit-exact values, the reference's bounds checks and messages."""
import os
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from vortrace_b200 import vortrace as V

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "slice_brute.npz")


@pytest.fixture(scope="module")
def sb():
    return np.load(GOLDEN)


def cloud(z, periodic):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(z["pos"], z["fields"], boundbox=list(z["bb"]), periodic=periodic)


@pytest.mark.parametrize("periodic", [False, True])
def test_slice_bit_exact(sb, periodic):
    pc = cloud(sb, periodic)
    tag = "periodic" if periodic else "open"
    for i in range(3):
        npix = tuple(int(v) for v in sb[f"slice{i}/npix"])
        out = pc.slice(sb[f"slice{i}/extent"], npix, float(sb[f"slice{i}/depth"]))
        assert out.shape == (npix[0], npix[1], 2)
        np.testing.assert_array_equal(out.reshape(-1, 2), sb[f"{tag}/slice{i}"])


def test_brute_projection_bit_exact(sb):
    pc = cloud(sb, False)
    for mode in ("sum", "max", "min"):
        bp = V.BruteProjection([12, 10, 25], [1.0, 9.0, 1.0, 9.0, 0.0, 10.0])
        bp.makeProjection(pc._cloud, mode)
        np.testing.assert_array_equal(bp.returnProjection(), sb[f"open/brute_{mode}"])


def test_slice_and_brute_errors(sb):
    pc = cloud(sb, False)
    with pytest.raises(RuntimeError, match="Slice extent out of bounds of current cloud subbox"):
        pc.slice([-1.0, 5.0, 0.0, 5.0], 8, 1.0)
    with pytest.raises(RuntimeError, match="Slice extent out of bounds"):
        pc.slice([0.0, 5.0, 0.0, 5.0], 8, 11.0)
    bp = V.BruteProjection([4, 4, 4], [1.0, 9.0, 1.0, 9.0, 0.0, 10.0])
    with pytest.raises(ValueError, match="VolumeRender is not supported by BruteProjection"):
        bp.makeProjection(pc._cloud, "volume")
    bp = V.BruteProjection([4, 4, 4], [1.0, 9.0, 1.0, 9.0, 0.0, 11.0])
    with pytest.raises(ValueError, match="Projection extent out of bounds of current cloud subbox"):
        bp.makeProjection(pc._cloud, "sum")
    with pytest.raises(RuntimeError, match="has not yet been made"):
        V.Slice([2, 2], [0, 1, 0, 1], 0.5).returnSlice()

"""Failure detection without a GPU fault: limits are lowered on the host so
the walk kernels return the reference's error statuses, and the context
stays usable afterwards (no trap, no device assert, bounded loops only)."""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from vortrace_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture
def cloud():
    rng = np.random.default_rng(9)
    pos = rng.uniform(0, 10, (5000, 3))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, np.ones(5000), boundbox=[0, 10] * 3)


RAYS = (np.array([[0.2, 0.3, 0.1], [5.0, 5.0, 0.0]]), np.array([[9.8, 9.7, 9.9], [5.0, 5.0, 10.0]]))


@pytest.mark.parametrize("kernel", ["plain", "batched"])
def test_max_iterations(cloud, kernel):
    cloud.kernel = kernel
    good = cloud.projection(*RAYS)
    cloud._cloud.set_param(L.PARAM_MAX_ITERATIONS, 3)
    with pytest.raises(L.VortraceError, match="Ray walk exceeded maximum iteration count") as ei:
        cloud.projection(*RAYS)
    assert ei.value.code == 10
    cloud._cloud.set_param(L.PARAM_MAX_ITERATIONS, 100000)
    np.testing.assert_array_equal(cloud.projection(*RAYS), good)


@pytest.mark.parametrize("kernel", ["plain", "batched"])
def test_hand_over_and_stack_capacity(cloud, kernel):
    cloud.kernel = kernel
    good = cloud.projection(*RAYS)
    assert cloud.last_stats["max_stack"] > 2 and cloud.last_stats["slow_rays"] == 0
    # rays deeper than 2 pending points go to the global-stack kernel:
    # same results, counted as handed over
    cloud._cloud.set_param(L.PARAM_LOCAL_STACK, 2)
    np.testing.assert_array_equal(cloud.projection(*RAYS), good)
    assert cloud.last_stats["slow_rays"] > 0
    # ... whose own capacity is exceeded: the stack error, then recovery
    cloud._cloud.set_param(L.PARAM_STACK_CAP, 2)
    with pytest.raises(L.VortraceError, match="stack capacity") as ei:
        cloud.projection(*RAYS)
    assert ei.value.code == 15
    cloud._cloud.set_param(L.PARAM_STACK_CAP, 4096)
    cloud._cloud.set_param(L.PARAM_LOCAL_STACK, 1 << 30)
    np.testing.assert_array_equal(cloud.projection(*RAYS), good)
    assert cloud.last_stats["slow_rays"] == 0


def test_non_finite_endpoints(cloud):
    s = np.array([[0.2, 0.3, np.nan]])
    with pytest.raises(ValueError, match="finite"):
        cloud.projection(s, np.array([[1.0, 1.0, 1.0]]))
    np.testing.assert_allclose(cloud.projection(*RAYS)[1], 10.0, rtol=1e-9)


def test_bad_parameters(cloud):
    with pytest.raises(ValueError):
        cloud._cloud.set_param(L.PARAM_MAX_ITERATIONS, 0)
    with pytest.raises(ValueError):
        cloud._cloud.set_param(L.PARAM_SMEM_LEVELS, 99)
    with pytest.raises(ValueError):
        cloud._cloud.set_param(12345, 1)


def test_error_detail_reports_first_ray(cloud):
    cloud.kernel = "plain"
    cloud._cloud.set_param(L.PARAM_MAX_ITERATIONS, 1)
    st = np.repeat(RAYS[0], 50, axis=0)
    en = np.repeat(RAYS[1], 50, axis=0)
    with pytest.raises(L.VortraceError) as ei:
        cloud.projection(st, en)
    assert ei.value.code == 10

"""Ray-grid generation (the reference's tests/test_grid.py cases)."""
import numpy as np

from vortrace_b200 import grid as gr


def test_base_grid_square():
    g0 = gr.generate_base_grid([0, 1], 64)
    g1 = gr.generate_base_grid([[0, 1], [0, 1]], (64, 64))
    np.testing.assert_equal(g0, g1)
    assert g0.shape == (64, 64, 3)
    assert g0[0][0][0] == 0.5 / 64.0
    assert g0[-1][-1][0] == 63.5 / 64.0
    assert g0[0][0][1] == 0.5 / 64.0


def test_base_grid_rectangle_and_offset():
    g = gr.generate_base_grid([[0, 1], [0, 3]], (64, 128))
    assert g.shape == (64, 128, 3)
    assert g[0][0][1] == 0.5 / (128.0 / 3.0)
    assert g[-1][-1][1] == 127.5 / (128 / 3.0)
    g0 = gr.generate_base_grid([3, 4], 64)
    assert g0[0][0][0] == 3 + 0.5 / 64.0


def test_named_projections():
    c = [0.5, 0.5, 0.5]
    expect = {
        "xy": [[[0.25, 0.25, 0.0], [0.25, 0.75, 0.0]], [[0.75, 0.25, 0.0], [0.75, 0.75, 0.0]]],
        "yz": [[[0.0, 0.25, 0.25], [0.0, 0.25, 0.75]], [[0.0, 0.75, 0.25], [0.0, 0.75, 0.75]]],
        "zx": [[[0.25, 0.0, 0.25], [0.75, 0.0, 0.25]], [[0.25, 0.0, 0.75], [0.75, 0.0, 0.75]]],
        "yx": [[[0.25, 0.25, 0.0], [0.75, 0.25, 0.0]], [[0.25, 0.75, 0.0], [0.75, 0.75, 0.0]]],
        "zy": [[[0.0, 0.25, 0.25], [0.0, 0.75, 0.25]], [[0.0, 0.25, 0.75], [0.0, 0.75, 0.75]]],
        "xz": [[[0.25, 0.0, 0.25], [0.25, 0.0, 0.75]], [[0.75, 0.0, 0.25], [0.75, 0.0, 0.75]]],
    }
    for proj, want in expect.items():
        gs, _ = gr.generate_projection_grid([0, 1], 2, [0, 1], c,
                                            proj=None if proj == "xy" else proj)
        np.testing.assert_almost_equal(gs, np.array(want))


def test_unknown_projection():
    import pytest
    with pytest.raises(ValueError, match="Unknown projection"):
        gr.generate_projection_grid([0, 1], 2, [0, 1], [0.5] * 3, proj="ab")


def test_bounds_set_z():
    s, e = gr.generate_projection_grid([0, 1], 4, [2.0, 7.0], None)
    assert np.all(s[..., 2] == 2.0) and np.all(e[..., 2] == 7.0)


def _axis_like_device(lo, hi, n):
    """The per-axis arithmetic of the device generator (csrc/grid.cu,
    make_axis / axis_at) in Python doubles."""
    d = (hi - lo) / float(n)
    start, stop = lo + 0.5 * d, hi - 0.5 * d
    delta, div = stop - start, float(n - 1)
    out = []
    for i in range(n):
        if n > 1 and i == n - 1:
            out.append(stop)
        elif n - 1 > 0 and delta / div != 0.0:
            out.append(float(i) * (delta / div) + start)
        elif n - 1 > 0:
            out.append((float(i) / div) * delta + start)
        else:
            out.append(float(i) * delta + start)
    return np.array(out)


def test_device_axis_arithmetic_matches_numpy():
    """The device generator's steps give numpy's pixel centres bit for bit
    (the GPU tests compare the kernel itself)."""
    rng = np.random.default_rng(3)
    cases = [(40.0, 60.0, 1024), (0, 100, 7), (-3.3, 7.1, 1), (1.0, 1.0, 3), (0.0, 1e-300, 5),
             (-1e6, 2.5e6, 997)]
    cases += [(float(a), float(a + w), int(n)) for a, w, n in
              zip(rng.uniform(-1e3, 1e3, 40), rng.lognormal(0.0, 3.0, 40),
                  rng.integers(1, 3000, 40))]
    for lo, hi, n in cases:
        g = gr.generate_base_grid([[lo, hi], [lo, hi]], (n, 1))
        want = g[:, 0, 0]
        got = _axis_like_device(float(lo), float(hi), n)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (lo, hi, n)


def test_device_grid_args():
    from vortrace_b200.vortrace import device_grid_args
    e4, nx, ny, b = device_grid_args([40, 60], 16, [0, 100])
    assert (nx, ny) == (16, 16) and e4.tolist() == [40.0, 60.0, 40.0, 60.0]
    assert b.tolist() == [0.0, 100.0]
    # a named projection whose handedness disagrees with the bounds flips them
    # (vortrace/grid.py:163-172)
    _, _, _, b = device_grid_args([[0, 1], [2, 3]], (4, 5), [0.0, 100.0], proj="xz")
    assert b.tolist() == [100.0, 0.0]
    _, _, _, b = device_grid_args([[0, 1], [2, 3]], (4, 5), [0.0, 100.0], proj="xy")
    assert b.tolist() == [0.0, 100.0]
    # float32 extents and arguments the host generator rejects keep the host path
    assert device_grid_args(np.array([0, 1], np.float32), 4, [0, 1]) is None
    assert device_grid_args([0, 1, 2], 4, [0, 1]) is None
    assert device_grid_args([0, 1], 0, [0, 1]) is None
    assert device_grid_args([0, 1], 4, [0, 1, 2]) is None

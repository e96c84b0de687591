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

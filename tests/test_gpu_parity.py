"""Parity of the CUDA path with the oracle and the reference's fixtures.

Bar: bit-exact cell ids, s values and integrals for integer/index work and
the FP64 walk; volume rendering within 1e-12 relative (CUDA's exp vs
glibc's).  Exact-tie geometry (lattices) is also checked through the
reference's invariants (integral = ray length, sum ds = length) here; its
segment lists are compared bit for bit in test_gpu_ties.py."""
import warnings

import numpy as np
import pytest

from oracle import oracle as O
from vortrace_b200 import grid as gr
from vortrace_b200 import workloads as W

pytestmark = pytest.mark.gpu

KERNELS = ["plain", "batched", "batched_fp64", "thread_fp32"]
VOL_RTOL = 1e-12


def cloud(pos, fields, bb, vol=None, **kw):
    import vortrace_b200 as vt
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, fields, boundbox=bb, vol=vol, **kw)


def oracle(pos, fields, bb, vol=None):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(pos, fields, bb, vol)
    return lp, O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])


# ------------------------------------------------------------------ k-NN
@pytest.fixture(scope="module")
def uniform20k():
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 100, (20000, 3))
    rho = rng.lognormal(0, 1, 20000)
    return pos, rho, cloud(pos, rho, [0, 100] * 3), oracle(pos, rho, [0, 100] * 3)


@pytest.mark.parametrize("k", [1, 2, 3, 10, 100])
def test_knn_bit_exact(uniform20k, k):
    pos, rho, pc, (lp, ot) = uniform20k
    q = np.random.default_rng(k).uniform(-5, 105, (4000, 3))
    ids, r2 = pc._cloud.knn(q, k)
    oids, or2 = ot.knn(q, k)
    np.testing.assert_array_equal(r2, or2)
    np.testing.assert_array_equal(ids, oids)


def test_knn_more_than_npart():
    pos = np.array([[0.1, 0.2, 0.3], [0.9, 0.8, 0.7], [0.5, 0.5, 0.5]])
    pc = cloud(pos, np.ones(3), [0, 1] * 3)
    ids, r2 = pc._cloud.knn(np.array([[0.0, 0.0, 0.0]]), 5)
    assert ids[0, :3].tolist() == [0, 2, 1] and ids[0, 3] == -1 and r2[0, 4] > 1e300


def test_knn_lattice_distances():
    from tests.conftest import make_cubic_lattice
    pos, f, vol, bb = make_cubic_lattice(6)
    pc = cloud(pos, f, bb, vol)
    lp, ot = oracle(pos, f, bb, vol)
    q = np.random.default_rng(2).uniform(-0.5, 5.5, (2000, 3)).round(1)
    for k in (1, 3, 8):
        ids, r2 = pc._cloud.knn(q, k)
        oids, or2 = ot.knn(q, k)
        np.testing.assert_array_equal(r2, or2)
        np.testing.assert_array_equal(ids, oids)   # tied points in nanoflann's order


# ------------------------------------------------------- reference fixtures
@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("case", ["uniform", "plummer", "volume"])
def test_fixture_projection_bit_exact(small_walks, case, kernel):
    c = small_walks[case]
    pc = cloud(c["pos"], c["fields"], c["bb"], c.get("vol"))
    pc.kernel = kernel
    np.testing.assert_array_equal(pc.orig_ids, c["orig_ids"])
    for mode in c["modes"]:
        mode = str(mode)
        out = pc.projection(c["starts"], c["ends"], reduction=mode).reshape(len(c["starts"]), -1)
        want = c[f"{mode}/out"]
        if mode == "volume":
            np.testing.assert_allclose(out, want, rtol=VOL_RTOL, atol=0)
        else:
            np.testing.assert_array_equal(out, want)


@pytest.mark.parametrize("case", ["uniform", "plummer", "volume"])
def test_fixture_segments_bit_exact(small_walks, case):
    c = small_walks[case]
    pc = cloud(c["pos"], c["fields"], c["bb"], c.get("vol"))
    mode = str(c["modes"][0])
    vals, cid, s_enter, ds, off = pc.traced_projection(c["starts"], c["ends"],
                                                       return_midpoint=False, reduction=mode,
                                                       flatten=True)
    np.testing.assert_array_equal(off, c["offsets"])
    np.testing.assert_array_equal(cid, c["orig_ids"][c["cell_ids"]])
    np.testing.assert_array_equal(s_enter, c["s_enter"])
    np.testing.assert_array_equal(ds, c["s_exit"] - c["s_enter"])


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("case", ["lattice", "lattice_f32"])
def test_fixture_lattice_invariants(small_walks, case, kernel):
    c = small_walks[case]
    pc = cloud(c["pos"], c["fields"], c["bb"], c.get("vol"))
    pc.kernel = kernel
    L = np.linalg.norm(c["ends"] - c["starts"], axis=1)
    out = pc.projection(c["starts"], c["ends"])
    rtol = 1e-3 if case == "lattice_f32" else 1e-6
    np.testing.assert_allclose(out, L, rtol=rtol)
    np.testing.assert_allclose(out, c["integrate/out"][:, 0], rtol=rtol)
    _, _, _, ds_list = pc.traced_projection(c["starts"], c["ends"])
    for i, ds in enumerate(ds_list):
        np.testing.assert_allclose(np.sum(ds), L[i], rtol=1e-12)


# ---------------------------------------------------------------- golden
@pytest.mark.parametrize("kernel", KERNELS)
def test_golden_projection(galaxy, kernel):
    # the reference's tests/test_vortrace.py:31-48
    box = galaxy["box_size"]
    pc = cloud(galaxy["pos"], galaxy["dens"], [0.0, box] * 3)
    pc.kernel = kernel
    dat = pc.grid_projection([box / 2 - 37.5, box / 2 + 37.5], 128, [0.0, box], None)
    np.testing.assert_array_almost_equal(dat, galaxy["proj"], decimal=14)
    lp, ot = oracle(galaxy["pos"], galaxy["dens"], [0.0, box] * 3)
    s, e = gr.generate_projection_grid([box / 2 - 37.5, box / 2 + 37.5], 128, [0.0, box], None)
    np.testing.assert_array_equal(dat.ravel(), ot.project(s.reshape(-1, 3), e.reshape(-1, 3))[:, 0])


# -------------------------------------------------------- configurations
def test_uniform_100k_full_image():
    w = W.uniform_100k()
    pc = cloud(w["pos"], w["fields"], w["boundbox"])
    lp, ot = oracle(w["pos"], w["fields"], w["boundbox"])
    ref, (_, _, _, off) = ot.project(w["starts"], w["ends"], segments=True)
    for kernel in KERNELS:
        pc.kernel = kernel
        out = pc.projection(w["starts"], w["ends"])
        np.testing.assert_array_equal(out, ref[:, 0])
        assert pc.last_stats["crossings"] == off[-1]


@pytest.fixture(scope="module")
def clustered():
    w = W.clustered_2m()
    return w, cloud(w["pos"], w["fields"], w["boundbox"]), oracle(w["pos"], w["fields"],
                                                                  w["boundbox"])


def test_clustered_2m_sample_vs_oracle(clustered):
    w, pc, (lp, ot) = clustered
    idx = np.linspace(0, len(w["starts"]) - 1, 4096).astype(np.int64)
    S, E = w["starts"][idx], w["ends"][idx]
    ref = ot.project(S, E)
    for kernel in KERNELS:
        pc.kernel = kernel
        np.testing.assert_array_equal(pc.projection(S, E), ref)


def test_clustered_2m_full_image_kernels_agree(clustered):
    w, pc, _ = clustered
    pc.kernel = "plain"
    a = pc.projection(w["starts"], w["ends"])
    ca = pc.last_stats["crossings"]
    pc.kernel = "batched"
    b = pc.projection(w["starts"], w["ends"])
    np.testing.assert_array_equal(a, b)
    assert pc.last_stats["crossings"] == ca
    # checksum of the full image against a second run (determinism)
    c = pc.projection(w["starts"], w["ends"])
    np.testing.assert_array_equal(b, c)
    assert np.all(np.isfinite(b)) and np.all(b > 0)


def test_volume_2m_sample(clustered):
    w, _, _ = clustered
    rgba = W.transfer_rgba(w["fields"][:, 0])
    pc = cloud(w["pos"], rgba, w["boundbox"])
    lp, ot = oracle(w["pos"], rgba, w["boundbox"])
    s, e = W.z_grid([40.0, 60.0], 512)
    idx = np.linspace(0, len(s) - 1, 2048).astype(np.int64)
    ref = ot.project(s[idx], e[idx], "volume")
    for kernel in KERNELS:
        pc.kernel = kernel
        np.testing.assert_allclose(pc.projection(s[idx], e[idx], reduction="volume"), ref,
                                   rtol=VOL_RTOL, atol=1e-300)


def test_batched_rotations_and_random_rays():
    w = W.batched_1m(n=200_000, nproj=4, npix=64, nrand=2000)
    pc = cloud(w["pos"], w["fields"], w["boundbox"])
    lp, ot = oracle(w["pos"], w["fields"], w["boundbox"])
    ref = ot.project(w["starts"], w["ends"])
    for kernel in KERNELS:
        pc.kernel = kernel
        np.testing.assert_array_equal(pc.projection(w["starts"], w["ends"]), ref[:, 0])


def test_nested_cloud_sample():
    pos, rho, _ = W.nested_cloud(500_000, 5)
    pc = cloud(pos, rho, W.BOX)
    lp, ot = oracle(pos, rho, W.BOX)
    s, e = W.z_grid([45.0, 55.0], 64)
    ref = ot.project(s, e)
    for kernel in KERNELS:
        pc.kernel = kernel
        np.testing.assert_array_equal(pc.projection(s, e), ref[:, 0])


def test_batch_projection_matches_individual(clustered):
    w, pc, _ = clustered
    pc.kernel = "auto"
    grids = [dict(extent=[45, 55], nres=32, bounds=[0, 100], center=None),
             dict(extent=[40, 60], nres=(16, 24), bounds=[0, 100], center=[50, 50, 50],
                  yaw=0.3, pitch=0.2, roll=0.1)]
    rng = np.random.default_rng(1)
    rs, re_ = rng.uniform(0, 100, (500, 3)), rng.uniform(0, 100, (500, 3))
    imgs, vals = pc.batch_projection(grids, (rs, re_))
    for g, img in zip(grids, imgs):
        kw = {k: v for k, v in g.items() if k not in ("extent", "nres", "bounds", "center")}
        np.testing.assert_array_equal(img, pc.grid_projection(g["extent"], g["nres"],
                                                              g["bounds"], g["center"], **kw))
    np.testing.assert_array_equal(vals, pc.projection(rs, re_))
    # a rotated grid first, two device grids after it, no arbitrary rays:
    # the images come back in the order of the grids
    grids2 = [grids[1], dict(extent=[48, 52], nres=(8, 12), bounds=[100, 0], center=None),
              grids[0]]
    imgs2 = pc.batch_projection(grids2)
    # one launch for the whole batch
    assert pc.last_stats["rays"] == 16 * 24 + 8 * 12 + 32 * 32
    assert len(imgs2) == 3
    for g, img in zip(grids2, imgs2):
        kw = {k: v for k, v in g.items() if k not in ("extent", "nres", "bounds", "center")}
        np.testing.assert_array_equal(img, pc.grid_projection(g["extent"], g["nres"],
                                                              g["bounds"], g["center"], **kw))
    assert imgs2[1].shape == (8, 12, 3)


def test_neighbourhood_cache_is_exact(clustered):
    """The batched kernel's per-ray neighbourhood cache answers split queries
    only when it provably holds every candidate: on/off give the same bits."""
    from vortrace_b200 import _lib as L
    w, pc, (lp, ot) = clustered
    idx = np.linspace(0, len(w["starts"]) - 1, 8192).astype(np.int64)
    S, E = w["starts"][idx], w["ends"][idx]
    pc.kernel = "batched"
    S, E = S[:1024], E[:1024]
    pc._cloud.set_param(L.PARAM_CACHE, 1)
    on = pc.projection(S, E)
    assert pc.last_stats["cache_hits"] > 0
    pc._cloud.set_param(L.PARAM_CACHE, 0)
    off = pc.projection(S, E)
    assert pc.last_stats["cache_hits"] == 0
    np.testing.assert_array_equal(on, off)
    np.testing.assert_array_equal(on, ot.project(S, E))


def test_neighbourhood_cache_random_rays_and_segments(clustered):
    """Cache on/off agree bit for bit on arbitrary directions (rays through
    the dense core and across the whole box) and on the per-segment output."""
    from vortrace_b200 import _lib as L
    w, pc, (lp, ot) = clustered
    rng = np.random.default_rng(11)
    S = np.vstack([rng.uniform(0.0, 100.0, (1536, 3)), 50.0 + rng.normal(0.0, 3.0, (512, 3))])
    E = np.vstack([rng.uniform(0.0, 100.0, (1536, 3)), 50.0 + rng.normal(0.0, 3.0, (512, 3))])
    pc.kernel = "batched"
    pc._cloud.set_param(L.PARAM_CACHE, 1)
    try:
        on = pc.projection(S, E)
        hits = pc.last_stats["cache_hits"]
        seg_on = pc.traced_projection(S[:256], E[:256], flatten=True)
    finally:
        pc._cloud.set_param(L.PARAM_CACHE, 0)
    assert hits > 0
    off = pc.projection(S, E)
    np.testing.assert_array_equal(on, off)
    seg_off = pc.traced_projection(S[:256], E[:256], flatten=True)
    for a, b in zip(seg_on, seg_off):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))
    np.testing.assert_array_equal(on, ot.project(S, E))


def _segments_vs_oracle(pc, lp, ot, S, E, reduction, kernel):
    """CSR segments (cells mapped to original ids, entry distances, lengths)
    and values of the CUDA walk against the oracle's, on the same rays."""
    oout, (ocid, ose, osx, ooff) = ot.project(S, E, reduction, segments=True)
    pc.kernel = kernel
    vals, cid, se, ds, off = pc.traced_projection(S, E, return_midpoint=False,
                                                  reduction=reduction, flatten=True)
    np.testing.assert_array_equal(off, ooff)
    np.testing.assert_array_equal(cid, lp["orig_ids"][ocid])
    np.testing.assert_array_equal(se, ose)
    np.testing.assert_array_equal(ds, osx - ose)
    return np.asarray(vals).reshape(len(S), -1), oout.reshape(len(S), -1)


@pytest.mark.parametrize("kernel", KERNELS)
def test_clustered_2m_segments_vs_oracle(clustered, kernel):
    """Segment-level parity on the benchmark cloud: an evenly spaced 2,048-ray
    sample of the 1024x1024 image and of volume_2m's 512x512 image (the same
    cloud), every kernel."""
    w, pc, (lp, ot) = clustered
    for starts, ends in ((w["starts"], w["ends"]), W.z_grid([40.0, 60.0], 512)):
        idx = np.linspace(0, len(starts) - 1, 2048).astype(np.int64)
        S, E = np.ascontiguousarray(starts[idx]), np.ascontiguousarray(ends[idx])
        v, o = _segments_vs_oracle(pc, lp, ot, S, E, "integrate", kernel)
        np.testing.assert_array_equal(v, o)


@pytest.fixture(scope="module")
def batched():
    w = W.batched_1m()
    return w, cloud(w["pos"], w["fields"], w["boundbox"]), oracle(w["pos"], w["fields"],
                                                                  w["boundbox"])


@pytest.mark.parametrize("kernel", ["thread_fp32", "batched_fp64"])
def test_batched_1m_segments_vs_oracle(batched, kernel):
    """Segment-level parity on batched_1m's rays: rotated views whose rays
    start and end outside the cloud, and the 10,000 random rays."""
    w, pc, (lp, ot) = batched
    n = len(w["starts"])
    idx = np.concatenate([np.linspace(0, n - 10_001, 3072).astype(np.int64),
                          np.arange(n - 10_000, n - 10_000 + 1024)])
    S, E = np.ascontiguousarray(w["starts"][idx]), np.ascontiguousarray(w["ends"][idx])
    v, o = _segments_vs_oracle(pc, lp, ot, S, E, "integrate", kernel)
    np.testing.assert_array_equal(v, o)

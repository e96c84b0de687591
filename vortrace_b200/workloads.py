"""Seeded synthetic clouds and rays for the benchmark configurations.

Every free parameter is fixed here and recorded in each workload's ``meta``
dict.  The clouds are synthetic stand-ins with the shapes, sizes and value
distributions of the benchmark definitions; no external dataset is used.

  uniform_100k   N=100,000 uniform in [0,100]^3, rho ~ lognormal(0,1), seed 0;
                 128x128 z-projection over [0,100]^2, bounds [0,100], integrate.
  clustered_2m   N=2,000,000: 90% Plummer (a=2, centre (50,50,50), truncated
                 at r=40, inverse-CDF radii, isotropic directions), 10%
                 uniform in [0,100]^3; rho = (1+r^2/a^2)^-2.5 * lognormal(0,.3);
                 fields [rho, rho*T, rho*Z], T ~ lognormal(0,0.5),
                 Z ~ U[0,0.02]; 1024x1024 z-projection over [40,60]^2,
                 bounds [0,100], integrate, nf=3.
  volume_2m      the clustered_2m cloud; RGBA from three Gaussian bands in
                 log10(rho) (centres -1, 0.5, 2; sigma 0.25); band colours
                 (0.25,0.45,1.0), (0.3,1.0,0.35), (1.0,0.35,0.2);
                 RGB = clip(sum_i band_i*colour_i, 0, 1);
                 alpha = clip(0.05*sum_i band_i, 0, 1); 512x512 over
                 [40,60]^2, bounds [0,100], reduction 'volume'.
  batched_1m     N=1,000,000 with the clustered_2m recipe (90/10), nf=1;
                 64 projections, rotation matrices from a seeded uniform
                 quaternion draw (seed 4), each 256x256 over a 30x30 extent
                 centred on (50,50,50), bounds +-50*sqrt(3) about the
                 centre, plus 10,000 rays with uniform endpoints in [0,100]^3.
  nested_16m     N=16,000,000: 95% in 8 Plummer sub-clumps (a_k log-uniform
                 in [0.05,2], centres (50,50,50) + N(0, 4^2) per axis, equal
                 weights, truncated at 20*a_k), 5% uniform; rho = sum_k
                 a_k^-3 (1+r_k^2/a_k^2)^-2.5 * lognormal(0,0.3), normalised to
                 max 1; 2048x2048 z-projection over [40,60]^2, bounds [0,100].
"""
from __future__ import annotations

import numpy as np

from . import grid as gr

BOX = [0.0, 100.0, 0.0, 100.0, 0.0, 100.0]


def _plummer(rng, n, a, centre, rmax):
    """n points of a Plummer sphere (scale a) truncated at rmax."""
    mmax = rmax ** 3 / (rmax ** 2 + a ** 2) ** 1.5
    m = rng.uniform(0.0, mmax, n)
    m = np.maximum(m, 1e-300)
    r = a / np.sqrt(m ** (-2.0 / 3.0) - 1.0)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return np.asarray(centre, np.float64) + r[:, None] * v


def clustered_cloud(n, seed, nf=3, frac=0.9, a=2.0):
    rng = np.random.default_rng(seed)
    nc = int(round(frac * n))
    centre = np.array([50.0, 50.0, 50.0])
    pos = np.vstack([_plummer(rng, nc, a, centre, 40.0), rng.uniform(0.0, 100.0, (n - nc, 3))])
    r2 = np.sum((pos - centre) ** 2, axis=1)
    rho = (1.0 + r2 / a ** 2) ** -2.5 * rng.lognormal(0.0, 0.3, n)
    if nf == 1:
        return pos, rho
    T = rng.lognormal(0.0, 0.5, n)
    Z = rng.uniform(0.0, 0.02, n)
    return pos, np.column_stack([rho, rho * T, rho * Z])


def z_grid(extent, npix, bounds=(0.0, 100.0)):
    s, e = gr.generate_projection_grid(extent, npix, list(bounds), None)
    return np.ascontiguousarray(s.reshape(-1, 3)), np.ascontiguousarray(e.reshape(-1, 3))


def uniform_100k(seed=0):
    rng = np.random.default_rng(seed)
    n = 100_000
    pos = rng.uniform(0.0, 100.0, (n, 3))
    rho = rng.lognormal(0.0, 1.0, n)
    s, e = z_grid([0.0, 100.0], 128)
    return dict(name="uniform_100k", pos=pos, fields=rho, boundbox=BOX, starts=s, ends=e,
                reduction="integrate", nres=(128, 128),
                meta=dict(n=n, seed=seed, dist="uniform(0,100)^3", rho="lognormal(0,1)",
                          grid="128x128 over [0,100]^2, bounds [0,100]"))


def clustered_2m(seed=1, n=2_000_000, npix=1024):
    pos, f = clustered_cloud(n, seed, nf=3)
    s, e = z_grid([40.0, 60.0], npix)
    return dict(name="clustered_2m", pos=pos, fields=f, boundbox=BOX, starts=s, ends=e,
                reduction="integrate", nres=(npix, npix),
                meta=dict(n=n, seed=seed, plummer_a=2.0, plummer_frac=0.9, rmax=40.0,
                          fields="rho, rho*T, rho*Z", grid=f"{npix}x{npix} over [40,60]^2, "
                          "bounds [0,100]"))


BAND_CENTRES = (-1.0, 0.5, 2.0)
BAND_SIGMA = 0.25
BAND_COLOURS = ((0.25, 0.45, 1.0), (0.3, 1.0, 0.35), (1.0, 0.35, 0.2))


def transfer_rgba(rho):
    lr = np.log10(np.maximum(rho, 1e-300))
    bands = np.stack([np.exp(-0.5 * ((lr - c) / BAND_SIGMA) ** 2) for c in BAND_CENTRES], 1)
    rgb = np.clip(bands @ np.asarray(BAND_COLOURS), 0.0, 1.0)
    alpha = np.clip(0.05 * bands.sum(1), 0.0, 1.0)
    return np.ascontiguousarray(np.column_stack([rgb, alpha]))


def volume_2m(seed=1, n=2_000_000, npix=512):
    pos, f = clustered_cloud(n, seed, nf=3)
    rgba = transfer_rgba(f[:, 0])
    s, e = z_grid([40.0, 60.0], npix)
    return dict(name="volume_2m", pos=pos, fields=rgba, boundbox=BOX, starts=s, ends=e,
                reduction="volume", nres=(npix, npix),
                meta=dict(n=n, seed=seed, band_centres=BAND_CENTRES, band_sigma=BAND_SIGMA,
                          band_colours=BAND_COLOURS, grid=f"{npix}x{npix} over [40,60]^2"))


def random_rotations(k, seed):
    """k rotation matrices from uniformly drawn unit quaternions."""
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    R = np.empty((k, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def batched_1m(seed=3, n=1_000_000, nproj=64, npix=256, nrand=10_000):
    pos, rho = clustered_cloud(n, seed, nf=1)
    centre = np.array([50.0, 50.0, 50.0])
    half = 50.0 * np.sqrt(3.0)
    base = gr.generate_base_grid([35.0, 65.0], npix).reshape(-1, 3)
    S, E = [], []
    for R in random_rotations(nproj, seed + 1):
        s = base.copy()
        e = base.copy()
        s[:, 2] = 50.0 - half
        e[:, 2] = 50.0 + half
        S.append((s - centre) @ R.T + centre)
        E.append((e - centre) @ R.T + centre)
    rng = np.random.default_rng(seed + 2)
    S.append(rng.uniform(0.0, 100.0, (nrand, 3)))
    E.append(rng.uniform(0.0, 100.0, (nrand, 3)))
    return dict(name="batched_1m", pos=pos, fields=rho, boundbox=BOX,
                starts=np.ascontiguousarray(np.concatenate(S)),
                ends=np.ascontiguousarray(np.concatenate(E)), reduction="integrate",
                nres=(npix, npix),
                meta=dict(n=n, seed=seed, nproj=nproj, npix=npix, nrand=nrand,
                          extent="30x30 about (50,50,50)", bounds="+-50*sqrt(3)"))


def nested_cloud(n, seed):
    rng = np.random.default_rng(seed)
    nc = int(round(0.95 * n))
    k = 8
    a = np.exp(rng.uniform(np.log(0.05), np.log(2.0), k))
    centres = 50.0 + rng.normal(0.0, 4.0, (k, 3))
    counts = np.full(k, nc // k)
    counts[: nc - counts.sum()] += 1
    parts = [_plummer(rng, int(counts[i]), a[i], centres[i], 20.0 * a[i]) for i in range(k)]
    pos = np.vstack(parts + [rng.uniform(0.0, 100.0, (n - nc, 3))])
    rho = np.zeros(n)
    for i in range(k):
        r2 = np.sum((pos - centres[i]) ** 2, axis=1)
        rho += a[i] ** -3 * (1.0 + r2 / a[i] ** 2) ** -2.5
    rho *= rng.lognormal(0.0, 0.3, n)
    rho /= rho.max()
    return pos, rho, dict(a=a.tolist(), centres=centres.tolist())


def nested_16m(seed=5, n=16_000_000, npix=2048):
    pos, rho, extra = nested_cloud(n, seed)
    s, e = z_grid([40.0, 60.0], npix)
    return dict(name="nested_16m", pos=pos, fields=rho, boundbox=BOX, starts=s, ends=e,
                reduction="integrate", nres=(npix, npix),
                meta=dict(n=n, seed=seed, grid=f"{npix}x{npix} over [40,60]^2", **extra))


CONFIGS = {"uniform_100k": uniform_100k, "clustered_2m": clustered_2m, "volume_2m": volume_2m,
           "batched_1m": batched_1m, "nested_16m": nested_16m}

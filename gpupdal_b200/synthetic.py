"""Seeded synthetic point clouds for the neighbourhood-geometry workloads.

No public dataset is named for this path; these generators stand in for
airborne-lidar tiles.  Coordinates are produced in metres and stored as LAS
raw int32 at scale 0.01 with offset 0 (``raw = llround(v / 0.01)``); the value
a PDAL reader would see is ``raw * 0.01 + 0.0`` in double.

Workloads (sizes and mixtures of the benchmark configurations):

* ``terrain``      z = 20 sin(x/80) cos(y/60) + N(0, 0.05), x, y ~ U[0, 500)^2
* ``mixture``      60 % terrain, 25 % faces of 400 axis-aligned boxes
                   (10-40 m wide, 5-30 m tall, + N(0, 0.02)), 15 % vegetation
                   blobs (sigma 1-4 m, centred 5-20 m above ground)
* ``stress``       mixture + 2 % exact duplicates of random points + 3 %
                   collinear wire points on random lines at z = 10-25 m
* ``tile``         the mixture on a square whose side keeps the mixture's
                   density (16 points per square metre) for any point count;
                   ``tiles`` makes many (one seed each) in parallel, the
                   batched and served workloads' tiles
"""
from __future__ import annotations

import numpy as np

SCALE = 0.01
DOMAIN = 500.0


def terrain_z(x, y):
    return 20.0 * np.sin(x / 80.0) * np.cos(y / 60.0)


def quantise(x, y, z):
    """metres -> raw int32 at 0.01 m (llround)."""
    out = []
    for v in (x, y, z):
        r = np.rint(np.asarray(v, dtype=np.float64) / SCALE)
        out.append(r.astype(np.int32))
    return out


def _terrain(rng, n, side):
    x = rng.uniform(0.0, side, n)
    y = rng.uniform(0.0, side, n)
    z = terrain_z(x, y) + rng.normal(0.0, 0.05, n)
    return x, y, z


def _buildings(rng, n, side, nbox):
    if n == 0:
        return np.empty(0), np.empty(0), np.empty(0)
    cx = rng.uniform(0.0, side, nbox)
    cy = rng.uniform(0.0, side, nbox)
    wx = rng.uniform(10.0, 40.0, nbox)
    wy = rng.uniform(10.0, 40.0, nbox)
    h = rng.uniform(5.0, 30.0, nbox)
    z0 = terrain_z(cx, cy)
    # faces: roof, wall x-, wall x+, wall y-, wall y+
    areas = np.stack([wx * wy, wy * h, wy * h, wx * h, wx * h], axis=1)
    w = areas.ravel() / areas.sum()
    face = rng.choice(areas.size, size=n, p=w)
    b = face // 5
    f = face % 5
    u = rng.uniform(0.0, 1.0, n)
    v = rng.uniform(0.0, 1.0, n)
    x = np.empty(n)
    y = np.empty(n)
    z = np.empty(n)
    x0 = cx[b] - wx[b] / 2
    y0 = cy[b] - wy[b] / 2
    roof = f == 0
    x[roof] = x0[roof] + u[roof] * wx[b][roof]
    y[roof] = y0[roof] + v[roof] * wy[b][roof]
    z[roof] = z0[b][roof] + h[b][roof]
    for fi, xs in ((1, 0.0), (2, 1.0)):
        m = f == fi
        x[m] = x0[m] + xs * wx[b][m]
        y[m] = y0[m] + u[m] * wy[b][m]
        z[m] = z0[b][m] + v[m] * h[b][m]
    for fi, ys in ((3, 0.0), (4, 1.0)):
        m = f == fi
        x[m] = x0[m] + u[m] * wx[b][m]
        y[m] = y0[m] + ys * wy[b][m]
        z[m] = z0[b][m] + v[m] * h[b][m]
    x += rng.normal(0.0, 0.02, n)
    y += rng.normal(0.0, 0.02, n)
    z += rng.normal(0.0, 0.02, n)
    return x, y, z


def _vegetation(rng, n, side, nblob):
    if n == 0:
        return np.empty(0), np.empty(0), np.empty(0)
    bx = rng.uniform(0.0, side, nblob)
    by = rng.uniform(0.0, side, nblob)
    bz = terrain_z(bx, by) + rng.uniform(5.0, 20.0, nblob)
    bs = rng.uniform(1.0, 4.0, nblob)
    b = rng.integers(0, nblob, n)
    x = bx[b] + rng.normal(0.0, 1.0, n) * bs[b]
    y = by[b] + rng.normal(0.0, 1.0, n) * bs[b]
    z = bz[b] + rng.normal(0.0, 1.0, n) * bs[b]
    return x, y, z


def _mixture(rng, n, side, nbox=400, nblob=None):
    nt = int(round(0.60 * n))
    nb = int(round(0.25 * n))
    nv = n - nt - nb
    if nblob is None:
        nblob = max(8, int(2000 * (side / DOMAIN) ** 2))
    nbox = max(1, int(round(nbox * (side / DOMAIN) ** 2)))
    parts = [_terrain(rng, nt, side), _buildings(rng, nb, side, nbox),
             _vegetation(rng, nv, side, nblob)]
    x = np.concatenate([p[0] for p in parts])
    y = np.concatenate([p[1] for p in parts])
    z = np.concatenate([p[2] for p in parts])
    perm = rng.permutation(n)
    return x[perm], y[perm], z[perm]


def terrain(n=250_000, seed=0):
    """C1: smooth terrain, 500 x 500 m, 0.05 m noise."""
    rng = np.random.default_rng(seed)
    return quantise(*_terrain(rng, n, DOMAIN))


def mixture(n=4_000_000, seed=1):
    """C2: terrain + building faces + vegetation, 500 x 500 m."""
    rng = np.random.default_rng(seed)
    return quantise(*_mixture(rng, n, DOMAIN))


def stress(n=32_000_000, seed=2, nwire=400):
    """C3: mixture + 2 % exact duplicates + 3 % collinear wire points."""
    rng = np.random.default_rng(seed)
    ndup = int(round(0.02 * n))
    nwp = int(round(0.03 * n))
    nbase = n - ndup - nwp
    xi, yi, zi = quantise(*_mixture(rng, nbase, DOMAIN))
    # wires: points along random 3D segments, quantised, no noise
    a = np.stack([rng.uniform(0, DOMAIN, nwire), rng.uniform(0, DOMAIN, nwire),
                  rng.uniform(10.0, 25.0, nwire)], axis=1)
    b = np.stack([rng.uniform(0, DOMAIN, nwire), rng.uniform(0, DOMAIN, nwire),
                  rng.uniform(10.0, 25.0, nwire)], axis=1)
    w = rng.integers(0, nwire, nwp)
    t = rng.uniform(0.0, 1.0, nwp)
    pw = a[w] + (b[w] - a[w]) * t[:, None]
    wx, wy, wz = quantise(pw[:, 0], pw[:, 1], pw[:, 2])
    src = rng.integers(0, nbase, ndup)
    x = np.concatenate([xi, wx, xi[src]])
    y = np.concatenate([yi, wy, yi[src]])
    z = np.concatenate([zi, wz, zi[src]])
    perm = rng.permutation(n)
    return x[perm], y[perm], z[perm]


def tile(n, seed, density=16.0):
    """A mixture tile of n points at `density` points per square metre."""
    rng = np.random.default_rng(seed)
    side = float(np.sqrt(n / density))
    return quantise(*_mixture(rng, n, side))


def _tile_job(args):
    n, seed = args
    return tile(n, seed)


def tiles(sizes, seeds, workers=None):
    """Mixture tiles of the given sizes, one seed each (tile(n, seed)),
    generated in parallel by a pool of fresh (spawned) processes."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import os
    jobs = [(int(n), int(s)) for n, s in zip(sizes, seeds)]
    workers = workers or min(16, os.cpu_count() or 1, max(1, len(jobs)))
    if workers <= 1 or len(jobs) <= 1:
        return [_tile_job(j) for j in jobs]
    with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_tile_job, jobs, chunksize=1))


def served_specs(count=2000, seed=1000, lo=10_000, hi=8_000_000):
    """The served stream's requests: (points, seed, knn, stage kind) each;
    sizes log-uniform in [lo, hi], knn uniform in {8, 16, 32, 64}, the stage
    normal / eigenvalues / covariancefeatures (1 / 2 / 3) in equal shares,
    request i with its own tile seed seed + i."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    knn = rng.choice((8, 16, 32, 64), count)
    kind = rng.integers(1, 4, count)
    return [(int(sizes[i]), seed + i, int(knn[i]), int(kind[i])) for i in range(count)]


def batched_sizes(count=256, seed=100, median=200_000, sigma=1.0, lo=20_000, hi=4_000_000):
    """Tile sizes of the batched workload: log-normal, clipped."""
    rng = np.random.default_rng(seed)
    s = np.exp(rng.normal(np.log(median), sigma, count))
    return np.clip(s, lo, hi).astype(np.int64)


def optimal_columns(n, seed, knn=10):
    """OptimalKNN (= knn) and OptimalRadius (U[0.3, 1.5]) input columns."""
    rng = np.random.default_rng(seed + 7919)
    return np.full(n, float(knn)), rng.uniform(0.3, 1.5, n)


def to_double(raw, scale=SCALE, offset=0.0):
    """The reference's coordinate: raw*scale + offset in double."""
    return raw.astype(np.float64) * scale + offset

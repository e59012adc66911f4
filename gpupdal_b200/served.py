"""The served tile stream and its two ways of running.

A stream is a list of requests shaped like the served configuration: sizes
log-uniform in [10k, 8M] points of the building/vegetation/terrain mixture,
knn uniform in {8, 16, 32, 64}, and the stage normal, eigenvalues or
covariancefeatures (feature_set=all, with OptimalKNN/OptimalRadius columns)
in equal shares.  Requests are uniform subsamples of one pre-generated,
pre-shuffled mixture cloud (so a bounded stream generates in seconds).

run_plain() answers the requests one after another with the plain per-tile
call (upload, nbg_run, free; host buffers in and out).  run_served() submits
them to a Server at Poisson arrival times (rate=None: all at once, which
measures capacity) and reports latency from submission to results.
"""
from __future__ import annotations

import threading
import time

import numpy as np

from . import abi
from . import synthetic as syn

KNNS = (8, 16, 32, 64)


def make_stream(count, seed=1000, pool_points=8_000_000, min_points=10_000,
                max_points=8_000_000):
    rng = np.random.default_rng(seed)
    x, y, z = syn.mixture(pool_points, seed)
    perm = rng.permutation(pool_points)
    x, y, z = x[perm], y[perm], z[perm]
    sizes = np.exp(rng.uniform(np.log(min_points), np.log(min(max_points, pool_points)), count))
    reqs = []
    for i in range(count):
        n = int(sizes[i])
        s0 = int(rng.integers(0, pool_points))
        idx = (s0 + np.arange(n)) % pool_points
        knn = int(rng.choice(KNNS))
        kind = (abi.STAGE_NORMAL, abi.STAGE_EIGENVALUES, abi.STAGE_COVARIANCEFEATURES)[i % 3]
        if kind == abi.STAGE_COVARIANCEFEATURES:
            st = abi.make_opts(kind, knn=knn, feature_mask=abi.FEAT_ALL)
            kopt, ropt = syn.optimal_columns(n, seed + i, knn=knn)
        else:
            st = abi.make_opts(kind, knn=knn)
            kopt = ropt = None
        reqs.append(dict(x=np.ascontiguousarray(x[idx]), y=np.ascontiguousarray(y[idx]),
                         z=np.ascontiguousarray(z[idx]), stages=[st], kopt=kopt, ropt=ropt,
                         knn=knn, kind=kind))
    return reqs


def run_plain(ctx, reqs):
    """Sequential plain per-tile calls; returns seconds per request."""
    secs = []
    for r in reqs:
        t0 = time.perf_counter()
        tile = ctx.tile(r["x"], r["y"], r["z"])
        ctx.run(tile, r["stages"], optimal_knn=r["kopt"], optimal_radius=r["ropt"])
        tile.free()
        secs.append(time.perf_counter() - t0)
    return secs


def run_served(server, reqs, rate=None, seed=0):
    """Submits at Poisson arrival times (rate requests/s; None: all at once)
    and waits for all.  Returns (makespan_s, latencies_s, results)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else np.zeros(len(reqs))
    arrivals = np.cumsum(gaps) - gaps[0]
    tickets = [None] * len(reqs)
    t0 = time.perf_counter()

    def client():
        for i, r in enumerate(reqs):
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets[i] = server.submit(r["x"], r["y"], r["z"], r["stages"],
                                       optimal_knn=r["kopt"], optimal_radius=r["ropt"], tag=i)

    th = threading.Thread(target=client)
    th.start()
    results = [None] * len(reqs)
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        results[i] = server.wait(tickets[i])[2]
    th.join()
    first = min(r.submit_us for r in results)
    last = max(r.end_us for r in results)
    lat = [(r.end_us - r.submit_us) / 1e6 for r in results]
    return (last - first) / 1e6, lat, results

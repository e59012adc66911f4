"""The served tile stream and its two ways of running.

A stream is a list of requests shaped like the served configuration: sizes
log-uniform in [10k, 8M] points of the building/vegetation/terrain mixture,
knn uniform in {8, 16, 32, 64}, and the stage normal, eigenvalues or
covariancefeatures (feature_set=all, with OptimalKNN/OptimalRadius columns)
in equal shares.  make_requests() gives each request its own compact mixture
tile and seed (the configuration's seeds 1000-2999); make_stream() hands out
requests as views of one pre-generated, pre-shuffled mixture cloud instead,
so that a 2,000-request rate sweep (2.4G points) costs host memory only for
the pool and submitting a request copies nothing.

run_plain() answers the requests one after another with the plain per-tile
call (upload, nbg_run, free; host buffers in and out).  pin_requests() gives a
stream pinned host buffers (coordinates, columns and reused output columns).  run_served() submits
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


class Stream:
    """The requests of a stream as views of one cloud: each request is a
    contiguous slice of the (doubled) pool, its OptimalKNN / OptimalRadius
    columns slices of pre-built columns, so taking a request copies nothing
    and a long stream costs host memory only for the pool."""

    def __init__(self, pool, specs, seed, max_points):
        x, y, z = pool
        m = min(max_points, len(x))
        self.x, self.y, self.z = (np.concatenate([v, v[:m]]) for v in (x, y, z))
        rng = np.random.default_rng(seed + 7919)
        self.ropt = rng.uniform(0.3, 1.5, len(self.x))
        self.kopt = {k: np.full(m, float(k)) for k in KNNS}
        self.specs = specs

    def __len__(self):
        return len(self.specs)

    def __getitem__(self, i):
        s0, n, knn, kind = self.specs[i]
        if kind == abi.STAGE_COVARIANCEFEATURES:
            st = abi.make_opts(kind, knn=knn, feature_mask=abi.FEAT_ALL)
            kopt, ropt = self.kopt[knn][:n], self.ropt[s0:s0 + n]
        else:
            st = abi.make_opts(kind, knn=knn)
            kopt = ropt = None
        return dict(x=self.x[s0:s0 + n], y=self.y[s0:s0 + n], z=self.z[s0:s0 + n], stages=[st],
                    kopt=kopt, ropt=ropt, knn=knn, kind=kind)

    def __iter__(self):
        return (self[i] for i in range(len(self)))

    def points(self):
        return sum(s[1] for s in self.specs)


def make_stream(count, seed=1000, pool_points=8_000_000, min_points=10_000,
                max_points=8_000_000, lazy=False):
    """`count` requests (a list, or with lazy=True the Stream itself, which
    hands out each request when it is taken)."""
    rng = np.random.default_rng(seed)
    x, y, z = syn.mixture(pool_points, seed)
    perm = rng.permutation(pool_points)
    x, y, z = x[perm], y[perm], z[perm]
    sizes = np.exp(rng.uniform(np.log(min_points), np.log(min(max_points, pool_points)), count))
    specs = []
    for i in range(count):
        n = int(sizes[i])
        s0 = int(rng.integers(0, pool_points))
        knn = int(rng.choice(KNNS))
        kind = (abi.STAGE_NORMAL, abi.STAGE_EIGENVALUES, abi.STAGE_COVARIANCEFEATURES)[i % 3]
        specs.append((s0, n, knn, kind))
    stream = Stream((x, y, z), specs, seed, max_points)
    return stream if lazy else list(stream)


def make_requests(count, seed=1000, lo=10_000, hi=8_000_000):
    """`count` requests of the served configuration, request i a compact
    mixture tile of its own seed (seed + i: seeds 1000-2999 for the full
    2,000-request stream), its size, knn and stage from syn.served_specs."""
    specs = syn.served_specs(count, seed, lo, hi)
    clouds = syn.tiles([s[0] for s in specs], [s[1] for s in specs])
    reqs = []
    for (n, rseed, knn, kind), (x, y, z) in zip(specs, clouds):
        if kind == abi.STAGE_COVARIANCEFEATURES:
            st = abi.make_opts(kind, knn=knn, feature_mask=abi.FEAT_ALL)
            kopt, ropt = syn.optimal_columns(n, rseed, knn=knn)
        else:
            st = abi.make_opts(kind, knn=knn)
            kopt = ropt = None
        reqs.append(dict(x=x, y=y, z=z, stages=[st], kopt=kopt, ropt=ropt, knn=knn, kind=kind,
                         seed=rseed))
    return reqs


def pin_requests(reqs):
    """The requests with their host buffers in pinned (page-locked) memory, as
    a server keeps its I/O staging: coordinates and OptimalKNN/OptimalRadius
    columns copied into pinned arrays, and each stage's output columns
    allocated pinned once ("out"), reused by every pass.  Pinned buffers are
    copied by DMA directly; pageable ones go through the library's bounce
    buffers and a host memcpy."""
    import torch

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t, t.numpy()

    out = []
    keep = []
    for r in reqs:
        q = dict(r)
        for k in ("x", "y", "z", "kopt", "ropt"):
            if r.get(k) is not None:
                t, q[k] = pinned(r[k])
                keep.append(t)
        n = len(r["x"])
        bufs = []
        for st in r["stages"]:
            t = torch.empty((max(len(abi.stage_dims(st)), 1), n), dtype=torch.float64).pin_memory()
            keep.append(t)
            bufs.append(t.numpy())
        q["out"] = bufs
        out.append(q)
    return out, keep


def run_plain(ctx, reqs):
    """Sequential plain per-tile calls; returns seconds per request."""
    secs = []
    for r in reqs:
        t0 = time.perf_counter()
        tile = ctx.tile(r["x"], r["y"], r["z"])
        ctx.run(tile, r["stages"], optimal_knn=r["kopt"], optimal_radius=r["ropt"],
                out=r.get("out"))
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
    held = [None] * len(reqs)
    t0 = time.perf_counter()

    def client():
        for i in range(len(reqs)):
            r = reqs[i]
            held[i] = r
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets[i] = server.submit(r["x"], r["y"], r["z"], r["stages"],
                                       optimal_knn=r["kopt"], optimal_radius=r["ropt"],
                                       out=r.get("out"), tag=i)

    th = threading.Thread(target=client)
    th.start()
    results = [None] * len(reqs)
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        results[i] = server.wait(tickets[i])[2]
        held[i] = None  # the request's host buffers may go once its result is back
    th.join()
    first = min(r.submit_us for r in results)
    last = max(r.end_us for r in results)
    lat = [(r.end_us - r.submit_us) / 1e6 for r in results]
    return (last - first) / 1e6, lat, results

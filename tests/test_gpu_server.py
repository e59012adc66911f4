"""The served form (nbg_server_*): continuous batching under an HBM budget.

* every request's outputs and row exceptions are identical alone (plain
  per-tile call) and in a mix of concurrent requests
* admission never runs requests together whose charged footprints exceed
  the budget, and a request larger than the budget is refused at submit
* with room for several, requests do overlap on the device
"""
import functools

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from gpupdal_b200.native import NbgError, Server

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=1)
def _requests():
    """12 requests: windows of the 4M mixture of 20k-600k points, knn and
    stage varying as in the served stream."""
    x, y, z = syn.mixture(4_000_000, 1)
    rng = np.random.default_rng(7)
    reqs = []
    kinds = [abi.STAGE_NORMAL, abi.STAGE_EIGENVALUES, abi.STAGE_COVARIANCEFEATURES]
    for i in range(12):
        side = int(rng.integers(3000, 18000))
        x0, y0 = (int(v) for v in rng.integers(0, 50000 - side, 2))
        m = (x >= x0) & (x < x0 + side) & (y >= y0) & (y < y0 + side)
        knn = int(rng.choice([8, 16, 32, 64]))
        kind = kinds[i % 3]
        if kind == abi.STAGE_COVARIANCEFEATURES:
            st = abi.make_opts(kind, knn=knn, feature_mask=abi.FEAT_ALL)
        else:
            st = abi.make_opts(kind, knn=knn)
        kopt, ropt = syn.optimal_columns(int(m.sum()), 100 + i, knn=knn)
        reqs.append((x[m], y[m], z[m], [st], kopt, ropt))
    return reqs


def _same(a, b):
    return all(np.array_equal(u, v, equal_nan=True) for u, v in zip(a, b))


def _sorted_ex(ex):
    return np.sort(ex, order=["point_id", "stage", "code"])


def test_results_are_the_same_alone_and_in_the_mix(nbg):
    reqs = _requests()
    alone = []
    for (x, y, z, st, kopt, ropt) in reqs:
        tile = nbg.tile(x, y, z)
        outs, ex, _ = nbg.run(tile, st, optimal_knn=kopt, optimal_radius=ropt)
        tile.free()
        alone.append((outs, _sorted_ex(ex)))
    srv = Server(0, slots=4)
    try:
        tickets = [srv.submit(x, y, z, st, optimal_knn=kopt, optimal_radius=ropt, tag=i)
                   for i, (x, y, z, st, kopt, ropt) in enumerate(reqs)]
        for i, t in enumerate(tickets):
            outs, ex, res = srv.wait(t)
            assert res.user_tag == i
            assert _same(outs, alone[i][0]), f"request {i}: outputs differ in the mix"
            assert np.array_equal(_sorted_ex(ex), alone[i][1]), f"request {i}: exceptions differ"
    finally:
        srv.close()


def test_requests_overlap_when_slots_and_memory_allow():
    reqs = _requests()
    srv = Server(0, slots=4)
    try:
        tickets = [srv.submit(x, y, z, st, optimal_knn=kopt, optimal_radius=ropt)
                   for (x, y, z, st, kopt, ropt) in reqs]
        spans = [srv.wait(t)[2] for t in tickets]
    finally:
        srv.close()
    overlaps = sum(1 for i, a in enumerate(spans) for b in spans[i + 1:]
                   if a.start_us < b.end_us and b.start_us < a.end_us)
    assert overlaps > 0


def test_admission_holds_the_budget():
    reqs = _requests()
    probe = Server(0, slots=1)
    est = [probe.request_bytes(len(r[0]), r[3]) for r in reqs]
    probe.close()
    budget = int(1.5 * max(est))
    srv = Server(0, slots=4, hbm_budget=budget)
    try:
        tickets = [srv.submit(x, y, z, st, optimal_knn=kopt, optimal_radius=ropt)
                   for (x, y, z, st, kopt, ropt) in reqs]
        res = [srv.wait(t)[2] for t in tickets]
        # at any start, the requests then running fit the budget
        for a in res:
            live = [b for b in res if b.start_us <= a.start_us < b.end_us]
            assert sum(b.est_bytes for b in live) <= budget or len(live) == 1
        x, y, z, st, kopt, ropt = reqs[0]
        big = np.concatenate([x] * 4), np.concatenate([y] * 4), np.concatenate([z] * 4)
        with pytest.raises(NbgError) as e:
            small = Server(0, slots=1, hbm_budget=srv.request_bytes(len(x), st))
            try:
                small.submit(*big, st)
            finally:
                small.close()
        assert e.value.code == abi.NBG_ERR_BUDGET
    finally:
        srv.close()


def test_pinned_buffers_give_the_same_results(nbg):
    """The served stream with its host buffers pinned (served.pin_requests:
    coordinates, OptimalKNN/OptimalRadius and reused output columns in
    page-locked memory, copied by DMA instead of through the bounce buffers)
    answers every request exactly as with pageable buffers, served and plain."""
    from gpupdal_b200 import served
    reqs = [dict(x=x, y=y, z=z, stages=st, kopt=kopt, ropt=ropt)
            for (x, y, z, st, kopt, ropt) in _requests()[:6]]
    preqs, keep = served.pin_requests(reqs)
    srv = Server(0, slots=4)
    try:
        for rs in (reqs, preqs):
            tickets = [srv.submit(r["x"], r["y"], r["z"], r["stages"], optimal_knn=r["kopt"],
                                  optimal_radius=r["ropt"], out=r.get("out"))
                       for r in rs]
            got = [srv.wait(t) for t in tickets]
            if rs is reqs:
                want = [([o.copy() for o in outs], _sorted_ex(ex)) for outs, ex, _ in got]
                continue
            for i, (outs, ex, _) in enumerate(got):
                assert _same(outs, want[i][0]), f"request {i}: pinned outputs differ"
                assert np.array_equal(_sorted_ex(ex), want[i][1]), f"request {i}: exceptions differ"
    finally:
        srv.close()
    # the plain per-tile call writes the same into the pinned output columns
    for r, (outs_want, _) in zip(preqs, want):
        tile = nbg.tile(r["x"], r["y"], r["z"])
        outs, ex, _ = nbg.run(tile, r["stages"], optimal_knn=r["kopt"], optimal_radius=r["ropt"],
                              out=r["out"])
        tile.free()
        assert _same(outs, outs_want)
    del preqs, keep

"""The synthetic workloads that stand in for the reference's benchmark data
hold the shapes their configurations name: the 500 x 500 m terrain surface
and its noise, the stress tile's exact duplicates and wires, the batched
set's clipped log-normal sizes and knn draws, and the served stream's
log-uniform sizes, knn set and equal stage shares."""
import numpy as np

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn


def test_terrain_surface_and_noise():
    x, y, z = syn.terrain(250_000, 0)
    assert len(x) == 250_000 and x.dtype == np.int32
    # 500 x 500 m at 0.01 m: raw 0 .. 50,000 (rounding reaches the upper edge)
    assert x.min() >= 0 and x.max() <= 50_000 and y.min() >= 0 and y.max() <= 50_000
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    resid = Z - 20.0 * np.sin(X / 80.0) * np.cos(Y / 60.0)
    # N(0, 0.05 m) noise plus at most one quantisation step of the inputs
    assert abs(resid.mean()) < 0.005 and 0.045 < resid.std() < 0.056
    # same seed, same cloud
    x2, _, _ = syn.terrain(250_000, 0)
    assert np.array_equal(x, x2)


def test_stress_duplicates_and_wires():
    n = 400_000
    x, y, z = syn.stress(n, 2)
    assert len(x) == n
    triples = np.stack([x, y, z], axis=1)
    uniq = np.unique(triples, axis=0)
    dup = n - len(uniq)
    assert dup >= int(0.02 * n) * 0.95          # the planted exact duplicates (2 %)
    wires = (syn.to_double(z) >= 10.0) & (syn.to_double(z) <= 25.0)
    assert wires.sum() >= 0.03 * n * 0.9        # wire points sit at 10-25 m


def test_batched_set_sizes_and_knn():
    s = syn.batched_sizes(256, 100)
    assert len(s) == 256 and s.min() >= 20_000 and s.max() <= 4_000_000
    assert 120_000 < np.median(s) < 330_000     # log-normal around 200k
    from gpupdal_b200 import batched
    tset = batched.make_set(count=12, seed=100, hi=1_000_000, device="cpu")
    for i, t in enumerate(tset):
        assert t["knn"] in (8, 16, 32)
        kinds = [st.kind for st in t["stages"]]
        assert kinds == [abi.STAGE_NORMAL, abi.STAGE_COVARIANCEFEATURES]
        assert 20_000 <= t["n"] <= 1_000_000
        # tile i: the mixture tile of its own seed 100 + i
        assert t["seed"] == 100 + i
        x, y, z = syn.tile(t["n"], 100 + i)
        assert np.array_equal(t["xyz"][0].numpy(), x)


def test_served_requests_own_seeds():
    from gpupdal_b200 import served
    reqs = served.make_requests(9, seed=1000, hi=300_000)
    for i, r in enumerate(reqs):
        assert r["seed"] == 1000 + i
        x, y, z = syn.tile(len(r["x"]), 1000 + i)
        assert np.array_equal(r["x"], x) and np.array_equal(r["z"], z)
        assert r["knn"] in (8, 16, 32, 64)
        assert 10_000 <= len(r["x"]) <= 300_000


def test_served_stream_mix():
    from gpupdal_b200 import served
    reqs = served.make_stream(240, seed=1000, pool_points=1_000_000, max_points=1_000_000)
    sizes = np.array([len(r["x"]) for r in reqs])
    assert sizes.min() >= 10_000 and sizes.max() <= 1_000_000
    # log-uniform: about half the requests below the geometric middle
    mid = np.sqrt(10_000 * 1_000_000)
    assert 0.35 < (sizes < mid).mean() < 0.65
    knns = {int(r["stages"][0].knn) for r in reqs}
    assert knns <= {8, 16, 32, 64} and len(knns) == 4
    kinds = [int(r["stages"][0].kind) for r in reqs]
    for k in (abi.STAGE_NORMAL, abi.STAGE_EIGENVALUES, abi.STAGE_COVARIANCEFEATURES):
        assert kinds.count(k) == 80


def test_optimal_columns():
    k, r = syn.optimal_columns(10_000, 1, knn=10)
    assert np.all(k == 10.0) and r.min() >= 0.3 and r.max() <= 1.5

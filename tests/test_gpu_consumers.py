"""The other consumers of the kNN index on the sm_100a path, through the C
ABI, against the oracle (the FP64 port, pinned bit for bit to oracle/_ref)
and the reference's own loops (oracle/_ref):

* nndistance (kth / avg), lof (NNDistance, LocalReachabilityDistance,
  LocalOutlierFactor) and outlier radius: bit-exact;
* optimalneighborhood: OptimalKNN exact except rows whose least
  eigenentropy is tied with another k to 1e-12 relative (the device's log
  and the host's differ in the last ulp); OptimalRadius bit-exact where
  OptimalKNN agrees;
* outlier statistical: labels exact except rows whose mean neighbour
  distance lies within 1e-9 (relative) of the threshold (the cloud's mean
  and deviation are exact sums here, serial running moments there);
* approximatecoplanar, estimaterank: statuses exact; values exact except
  rows within 1e-9 (FP64 oracle) or 1e-5 (the reference's float-narrowed
  covariance) of a threshold, relative to the largest eigenvalue.
"""
import math
import os

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu


def _cloud(name):
    if name == "lattice":
        g = U.golden("ties_lattice")
        return g["x"], g["y"], g["z"]
    if name == "terrain":
        return syn.terrain(60_000, 0)
    if name == "mixture":
        x, y, z = syn.mixture(4_000_000, 1)
        m = (x < 9000) & (y < 9000)
        return x[m], y[m], z[m]
    if name == "stress":
        x, y, z = syn.stress(4_000_000, 2)
        m = (x < 9000) & (y < 9000)
        return x[m], y[m], z[m]
    return (np.array([0, 5, 9, 100, 3], np.int32), np.array([0, 1, 2, 3, 4], np.int32),
            np.array([0, 0, 1, 1, 9], np.int32))


CLOUDS = ["lattice", "terrain", "mixture", "stress", "tiny"]


def _bits_equal(a, b):
    return np.all((a == b) | (np.isnan(a) & np.isnan(b)), axis=0)


@pytest.mark.parametrize("cloud", CLOUDS)
def test_list_consumers_bit_exact(nbg, port, ref, cloud):
    x, y, z = _cloud(cloud)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
    for kind, kw in [(abi.STAGE_NNDISTANCE, {}), (abi.STAGE_NNDISTANCE, {"k": 0}),
                     (abi.STAGE_NNDISTANCE, {"k": 24, "mode": "avg"}),
                     (abi.STAGE_LOF, {}), (abi.STAGE_LOF, {"minpts": 31}),
                     (abi.STAGE_OUTLIER, {"method": "radius", "radius": 0.45, "min_k": 3}),
                     (abi.STAGE_OUTLIER, {"method": "radius", "radius": 0.3, "min_k": -1})]:
        o = abi.consumer_opts(kind, **kw)
        outs, ex, stats = nbg.run(tile, [o])
        want, st = tp.run_stage(o, mode=0)
        assert len(ex) == 0 and (st == 0).all()
        bad = ~_bits_equal(outs[0], want)
        assert not bad.any(), (f"{cloud} {kind} {kw}: {bad.sum()} rows differ, first "
                               f"{np.flatnonzero(bad)[:4].tolist()}")
        if kind == abi.STAGE_OUTLIER:
            assert stats.outliers == tp.outliers and stats.inliers == len(x) - tp.outliers
    # and the reference's loops themselves, on one case of each
    for o in (abi.consumer_opts(abi.STAGE_NNDISTANCE, k=7, mode="avg"),
              abi.consumer_opts(abi.STAGE_LOF, minpts=12)):
        outs, _, _ = nbg.run(tile, [o])
        want, _ = tr.run_stage(o, mode=0)
        assert _bits_equal(outs[0], want).all()


def _entropies(tree, X, Y, Z, row, kmax):
    """Eigenentropy of each prefix k of the row's reference-ordered list
    (the loop of OptimalNeighborhoodFilter.cpp:79-150 with numpy's solver)."""
    q = (X[row], Y[row], Z[row])
    ids = tree.neighbors(q, kmax).astype(np.int64)
    P = np.stack([X[ids], Y[ids], Z[ids]], 1)
    out = {}
    for k in range(2, len(ids) + 1):
        ev = np.clip(np.linalg.eigvalsh(np.cov(P[:k].T)), 0, None)
        lam = ev / ev.sum()
        with np.errstate(divide="ignore", invalid="ignore"):
            out[k] = -np.sum(lam * np.log(lam))
    return out


@pytest.mark.parametrize("cloud", CLOUDS)
def test_optimalneighborhood(nbg, port, cloud):
    x, y, z = _cloud(cloud)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    tp = port.tree(X, Y, Z)
    for kw in ({}, {"min_k": 3, "max_k": 40}, {"min_k": 1, "max_k": 8}):
        o = abi.consumer_opts(abi.STAGE_OPTIMALNEIGHBORHOOD, **kw)
        outs, ex, _ = nbg.run(tile, [o])
        want, st = tp.run_stage(o, mode=0)
        got_st = U.status_from_exceptions(len(x), ex)
        assert np.array_equal(got_st, st), f"{cloud} {kw}: status"
        ok = st == 0
        diff = np.flatnonzero(ok & (outs[0][0] != want[0]))
        assert diff.size <= max(2, len(x) // 10000), f"{cloud} {kw}: {diff.size} rows"
        for r in diff:
            ent = _entropies(tp, X, Y, Z, r, o.knn)
            a, b = ent[int(outs[0][0][r])], ent[int(want[0][r])]
            assert abs(a - b) <= 1e-12 * max(abs(a), abs(b)), (cloud, kw, r, a, b)
        same = ok & (outs[0][0] == want[0])
        assert _bits_equal(outs[0][1][same], want[1][same]).all()


@pytest.mark.parametrize("cloud", ["terrain", "mixture", "stress"])
def test_outlier_statistical(nbg, port, ref, cloud):
    x, y, z = _cloud(cloud)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
    for kw in ({}, {"mean_k": 12, "multiplier": 1.25, "cls": 18}):
        o = abi.consumer_opts(abi.STAGE_OUTLIER, **kw)
        outs, ex, stats = nbg.run(tile, [o])
        assert len(ex) == 0
        for tree in (tp, tr):
            want, _ = tree.run_stage(o, mode=0)
            bad = np.flatnonzero(outs[0][0] != want[0])
            if bad.size:
                # rows at the threshold: mean neighbour distance within 1e-9
                avg, _, _ = nbg.run(tile, [abi.consumer_opts(abi.STAGE_NNDISTANCE, k=o.knn,
                                                             mode="avg")])
                d = avg[0][0]
                thr = d.mean() + o.thresh1 * d.std(ddof=1)
                assert (np.abs(d[bad] - thr) <= 1e-9 * thr).all(), (cloud, kw, bad[:4])
            assert abs(int(stats.outliers) - tree.outliers) <= bad.size


@pytest.mark.parametrize("cloud", ["lattice", "terrain", "mixture", "stress", "tiny"])
def test_coplanar_and_rank(nbg, port, ref, cloud):
    x, y, z = _cloud(cloud)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
    for kind, kw in [(abi.STAGE_APPROXIMATECOPLANAR, {}), (abi.STAGE_APPROXIMATECOPLANAR, {"knn": 16}),
                     (abi.STAGE_ESTIMATERANK, {}), (abi.STAGE_ESTIMATERANK, {"knn": 3, "thresh": 0.1})]:
        o = abi.consumer_opts(kind, **kw)
        outs, ex, _ = nbg.run(tile, [o])
        got_st = U.status_from_exceptions(len(x), ex)
        lam, _ = tp.run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, knn=max(o.knn - 1, 0)), mode=1)
        lmax = np.abs(np.nan_to_num(lam, nan=0.0)).max(axis=0)
        for tree, mode, rel in ((tp, 1, 1e-9), (tr, 0, 1e-5)):
            want, st = tree.run_stage(o, mode=mode)
            assert np.array_equal(got_st, st), f"{cloud} {kind} {kw}: status"
            ok = st == 0
            bad = np.flatnonzero(ok & (outs[0][0] != want[0]))
            if kind == abi.STAGE_APPROXIMATECOPLANAR:
                e0, e1, e2 = lam[0][bad], lam[1][bad], lam[2][bad]
                near = ((np.abs(e1 - o.thresh1 * e0) <= rel * o.thresh1 * lmax[bad]) |
                        (np.abs(o.thresh2 * e1 - e2) <= rel * o.thresh2 * lmax[bad]))
            else:
                thr = np.float32(o.thresh1) * lmax[bad]
                near = (np.abs(np.abs(lam[:, bad]) - thr) <= rel * lmax[bad]).any(axis=0)
            assert near.all(), (cloud, kind, kw, mode, bad[~near][:4].tolist())


def test_nndistance_grid_known_answers(nbg):
    # NNDistanceTest.cpp:43-128: integer grid 0..9 on each axis
    g = np.arange(10, dtype=np.int32)
    x, y, z = (v.reshape(-1).astype(np.int32) for v in np.meshgrid(g, g, g, indexing="ij"))
    tile = nbg.tile(x, y, z, scale=(1.0, 1.0, 1.0))
    outs, _, _ = nbg.run(tile, [abi.consumer_opts(abi.STAGE_NNDISTANCE, k=3)])
    assert (outs[0][0] == 1.0).all()
    outs, _, _ = nbg.run(tile, [abi.consumer_opts(abi.STAGE_NNDISTANCE, k=4)])
    corner = np.isin(x, (0, 9)) & np.isin(y, (0, 9)) & np.isin(z, (0, 9))
    assert (outs[0][0][corner] == math.sqrt(2)).all()
    outs, _, _ = nbg.run(tile, [abi.consumer_opts(abi.STAGE_NNDISTANCE, k=6, mode="avg")])
    ends = sum(np.isin(v, (0, 9)).astype(int) for v in (x, y, z))
    want = np.select([ends == 3, ends == 2, ends == 1],
                     [(1 + math.sqrt(2)) / 2.0, (2 + math.sqrt(2)) / 3.0, (5 + math.sqrt(2)) / 6.0],
                     1.0)
    assert (outs[0][0] == want).all()


def test_pipeline_optimal_then_covariancefeatures(nbg, port):
    """filters.optimalneighborhood feeding covariancefeatures (optimized,
    Density), the reference's documented use of the pair."""
    from gpupdal_b200.stages import run_pipeline
    x, y, z = _cloud("mixture")
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    pipe = [{"type": "filters.optimalneighborhood", "min_k": 8, "max_k": 20},
            {"type": "filters.covariancefeatures", "optimized": True,
             "feature_set": "Linearity,Planarity,Density"}]
    dims, log = run_pipeline(nbg, pipe, x, y, z)
    tp = port.tree(X, Y, Z)
    opt, _ = tp.run_stage(abi.consumer_opts(abi.STAGE_OPTIMALNEIGHBORHOOD, min_k=8, max_k=20),
                          mode=0)
    same = dims["OptimalKNN"] == opt[0]
    assert same.mean() > 0.999
    o = abi.make_opts(abi.STAGE_COVARIANCEFEATURES, optimized=True,
                      feature_mask=abi.FEAT_LINEARITY | abi.FEAT_PLANARITY | abi.FEAT_DENSITY)
    want, st = tp.run_stage(o, mode=1, optimal_knn=dims["OptimalKNN"],
                            optimal_radius=dims["OptimalRadius"])
    ok = (st == 0) & same
    for i, name in enumerate(("Linearity", "Planarity", "Density")):
        err = np.abs(dims[name][ok] - want[i][ok])
        scale = 1.0 if name != "Density" else np.abs(want[i][ok])
        assert (err <= 1e-5 * np.maximum(scale, 1e-300)).mean() > 0.999, name


def test_consumer_options_refused(nbg):
    tile = nbg.tile(*_cloud("tiny"))
    from gpupdal_b200.native import NbgError
    for o in (abi.consumer_opts(abi.STAGE_APPROXIMATECOPLANAR, knn=0),
              abi.consumer_opts(abi.STAGE_OPTIMALNEIGHBORHOOD, min_k=9, max_k=4),
              abi.consumer_opts(abi.STAGE_OPTIMALNEIGHBORHOOD, min_k=0, max_k=4)):
        with pytest.raises(NbgError):
            nbg.run(tile, [o])
    # an unrecognised outlier method leaves the column as it was
    o = abi.consumer_opts(abi.STAGE_OUTLIER)
    o.mode = 2
    outs, _, stats = nbg.run(tile, [o])
    assert (outs[0][0] == 0).all() and stats.outliers == 0


def test_pipeline_json_runs_the_consumers(nbg):
    """An existing pipeline naming the consumers runs through the stage layer
    with the filters' own names and options; each dimension equals the
    direct nbg_run of the same options, and filters.outlier's warning is
    logged when no row is an outlier."""
    from gpupdal_b200.stages import run_pipeline
    x, y, z = _cloud("mixture")
    pipe = ["in.las",
            {"type": "filters.nndistance", "mode": "avg", "k": 6},
            {"type": "filters.lof", "minpts": 12},
            {"type": "filters.approximatecoplanar", "knn": 10, "thresh1": 20},
            {"type": "filters.estimaterank", "knn": 9},
            {"type": "filters.outlier", "method": "radius", "radius": 5.0, "min_k": 0},
            "out.las"]
    dims, log = run_pipeline(nbg, pipe, x, y, z)
    assert log[0] == "not run: file" and log[-1] == "not run: file"
    assert any("Filtered cloud has no outliers!" in l for l in log)
    tile = nbg.tile(x, y, z)
    direct = {
        "LocalOutlierFactor": (abi.consumer_opts(abi.STAGE_LOF, minpts=12), 2),
        "Coplanar": (abi.consumer_opts(abi.STAGE_APPROXIMATECOPLANAR, knn=10, thresh1=20.0), 0),
        "Rank": (abi.consumer_opts(abi.STAGE_ESTIMATERANK, knn=9), 0),
        "Classification": (abi.consumer_opts(abi.STAGE_OUTLIER, method="radius", radius=5.0,
                                             min_k=0), 0),
    }
    for name, (o, d) in direct.items():
        outs, _, _ = nbg.run(tile, [o])
        assert np.array_equal(dims[name], outs[0][d], equal_nan=True), name
    # NNDistance was written by nndistance, then by lof (the later stage wins, as in PDAL)
    outs, _, _ = nbg.run(tile, [abi.consumer_opts(abi.STAGE_LOF, minpts=12)])
    assert np.array_equal(dims["NNDistance"], outs[0][0])


FIXTURES = os.path.join(U.GOLDEN, "fixtures")


@pytest.mark.parametrize("name", sorted(f[:-4] for f in os.listdir(FIXTURES) if f.endswith(".npz")))
def test_fork_coplanar_fixtures_on_device(nbg, name):
    # the fork's own approximatecoplanar fixtures, recorded from the reference:
    # six axis points whose spectrum (0.4, 10, 40) puts thresh1 = 25 exactly on
    # the boundary (knn 6, and knn 3 with a distance tie at the k-th
    # neighbour), and four coincident points
    g = dict(np.load(os.path.join(FIXTURES, name + ".npz")))
    tile = nbg.tile(g["x"], g["y"], g["z"])
    n = len(g["x"])
    for key in [k for k in g if k.startswith("nbr_k")]:
        ids, _ = nbg.neighbor_sets(tile, int(key[5:]))
        assert np.array_equal(U.sorted_rows(ids), U.sorted_rows(g[key])), f"{name} {key}"
    for key in [k for k in g if k.endswith("_opts")]:
        sname = key[:-5]
        o = U.opts_from_bytes(g[key])
        outs, ex, _ = nbg.run(tile, [o])
        status = U.status_from_exceptions(n, ex)
        assert np.array_equal(status, g[sname + "_status"]), f"{name}/{sname} status"
        ok = status == 0
        want = g[sname + "_out"][:, ok]
        got = outs[0][:, ok]
        if o.kind in (abi.STAGE_APPROXIMATECOPLANAR, abi.STAGE_ESTIMATERANK):
            assert np.array_equal(got, want), f"{name}/{sname}: {got} vs {want}"
        else:
            lmax = np.abs(want).max(axis=0)
            assert np.all(np.abs(got - want) <= 1e-5 * lmax), f"{name}/{sname}: {got} vs {want}"

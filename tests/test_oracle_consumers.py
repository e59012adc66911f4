"""The oracle of the other kNN consumers (filters.approximatecoplanar,
estimaterank, nndistance, optimalneighborhood, lof, outlier) is pinned on
the CPU:

* the FP64 port against oracle/_ref (the same loops over the reference's own
  nanoflann and Eigen), bit for bit, on lattice ties, terrain, a building /
  vegetation mixture and a cloud smaller than the lists (padding);
* against the known answers of the reference's unit test
  test/unit/filters/NNDistanceTest.cpp:43-128 (10 x 10 x 10 grid).
"""
import math

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

CASES = [
    (abi.STAGE_APPROXIMATECOPLANAR, {"knn": 1}),
    (abi.STAGE_APPROXIMATECOPLANAR, {}),
    (abi.STAGE_APPROXIMATECOPLANAR, {"knn": 16, "thresh1": 10.0, "thresh2": 3.0}),
    (abi.STAGE_ESTIMATERANK, {}),
    (abi.STAGE_ESTIMATERANK, {"knn": 3, "thresh": 0.1}),
    (abi.STAGE_NNDISTANCE, {"k": 0}),
    (abi.STAGE_NNDISTANCE, {}),
    (abi.STAGE_NNDISTANCE, {"k": 33, "mode": "avg"}),
    (abi.STAGE_OPTIMALNEIGHBORHOOD, {}),
    (abi.STAGE_OPTIMALNEIGHBORHOOD, {"min_k": 1, "max_k": 64}),
    (abi.STAGE_LOF, {}),
    (abi.STAGE_LOF, {"minpts": 0}),
    (abi.STAGE_OUTLIER, {}),
    (abi.STAGE_OUTLIER, {"mean_k": 12, "multiplier": 1.25, "cls": 18}),
    (abi.STAGE_OUTLIER, {"method": "radius", "radius": 1.0, "min_k": 6}),
    (abi.STAGE_OUTLIER, {"method": "radius", "radius": 0.5, "min_k": -1}),
]


def clouds():
    g = U.golden("ties_lattice")
    yield "lattice", g["x"], g["y"], g["z"]
    x, y, z = syn.terrain(20_000, 0)
    yield "terrain", x, y, z
    x, y, z = syn.mixture(1_000_000, 1)
    m = (x < 4000) & (y < 4000)
    yield "mixture", x[m], y[m], z[m]
    yield ("tiny", np.array([0, 5, 9, 100, 3], np.int32), np.array([0, 1, 2, 3, 4], np.int32),
           np.array([0, 0, 1, 1, 9], np.int32))


def _same(a, b):
    return np.all((a == b) | (np.isnan(a) & np.isnan(b)))


@pytest.mark.parametrize("cloud", ["lattice", "terrain", "mixture", "tiny"])
def test_port_matches_reference_consumers(port, ref, cloud):
    name, x, y, z = next(c for c in clouds() if c[0] == cloud)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
    for kind, kw in CASES:
        o = abi.consumer_opts(kind, **kw)
        a, sa = tp.run_stage(o, mode=0)
        b, sb = tr.run_stage(o, mode=0)
        assert np.array_equal(sa, sb), (name, kind, kw)
        assert _same(a, b), (name, kind, kw)
        if kind == abi.STAGE_OUTLIER:
            assert tp.outliers == tr.outliers


def _grid10():
    g = np.arange(10, dtype=np.int32)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    return [v.reshape(-1).astype(np.int32) for v in (x, y, z)]


def test_reference_nndistance_grid(port, ref):
    # NNDistanceTest.cpp:43-128: integer grid 0..9 on each axis (scale 1)
    x, y, z = _grid10()
    X, Y, Z = (v.astype(np.float64) for v in (x, y, z))
    for orc in (port, ref):
        t = orc.tree(X, Y, Z)
        out, _ = t.run_stage(abi.consumer_opts(abi.STAGE_NNDISTANCE, k=3), mode=0)
        assert (out[0] == 1.0).all()
        out, _ = t.run_stage(abi.consumer_opts(abi.STAGE_NNDISTANCE, k=4), mode=0)
        corner = np.isin(X, (0, 9)) & np.isin(Y, (0, 9)) & np.isin(Z, (0, 9))
        assert (out[0][corner] == math.sqrt(2)).all()
        out, _ = t.run_stage(abi.consumer_opts(abi.STAGE_NNDISTANCE, k=6, mode="avg"), mode=0)
        ends = sum(np.isin(v, (0, 9)).astype(int) for v in (X, Y, Z))
        want = np.select([ends == 3, ends == 2, ends == 1],
                         [(1 + math.sqrt(2)) / 2.0, (2 + math.sqrt(2)) / 3.0,
                          (5 + math.sqrt(2)) / 6.0], 1.0)
        assert (out[0] == want).all()


def test_outlier_warnings_cases(port):
    # OutlierFilter.cpp:191-226: no labels when every row is an outlier or none is
    x, y, z = syn.terrain(5_000, 3)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    t = port.tree(X, Y, Z)
    out, _ = t.run_stage(abi.consumer_opts(abi.STAGE_OUTLIER, method="radius", radius=0.01,
                                           min_k=100), mode=0)
    assert t.outliers == len(x) and (out[0] == 0).all()
    out, _ = t.run_stage(abi.consumer_opts(abi.STAGE_OUTLIER, method="radius", radius=100.0,
                                           min_k=0), mode=0)
    assert t.outliers == 0 and (out[0] == 0).all()

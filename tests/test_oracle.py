"""The oracle is pinned before it is trusted (CPU only).

* against the golden vectors produced by the reference's own nanoflann and
  Eigen (tests/golden/, see make_golden.py)
* against oracle/_ref directly, when it is built here
* against the known answers of the reference's unit tests
  (test/unit/filters/NormalFilterTest.cpp, CovarianceFeaturesTest.cpp,
  test/unit/KDIndexTest.cpp:118-223)
"""
import math

import os

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U


@pytest.mark.parametrize("name", U.golden_names())
def test_port_matches_golden(port, name):
    _port_matches(port, U.golden(name), name)


FIXTURES = os.path.join(U.GOLDEN, "fixtures")


@pytest.mark.parametrize("name", sorted(f[:-4] for f in os.listdir(FIXTURES) if f.endswith(".npz")))
def test_port_matches_fork_fixtures(port, name):
    # the reference's own approximatecoplanar fixtures (tests/golden/fixtures)
    _port_matches(port, dict(np.load(os.path.join(FIXTURES, name + ".npz"))), name)


def test_fork_boundary_fixture_known_answer():
    # six points at (+-1,0,0), (0,+-5,0), (0,0,+-10): with every point in the
    # neighbourhood the covariance is diag(0.4, 10, 40), so thresh1 = 25 sits
    # exactly on the boundary (10 > 25 * 0.4 is false: not coplanar) and the
    # rank is 3
    g = dict(np.load(os.path.join(FIXTURES, "fork_coplanar_boundary.npz")))
    assert np.array_equal(g["eig5_out"], np.tile([[0.4], [10.0], [40.0]], (1, 6)))
    assert np.array_equal(g["cop6_out"], np.zeros((1, 6)))
    assert np.array_equal(g["rank6_out"], np.full((1, 6), 3.0))


def _port_matches(port, g, name):
    X, Y, Z = U.doubles(g)
    t = port.tree(X, Y, Z)
    for key in [k for k in g if k.startswith("nbr_k")]:
        k = int(key[5:])
        got = t.all_neighbors(k + 1)
        assert np.array_equal(got.astype(np.uint32), g[key]), f"{name} {key}: neighbour lists differ"
    for key in [k for k in g if k.endswith("_opts")]:
        sname = key[:-5]
        o = U.opts_from_bytes(g[key])
        outs, status = t.run_stage(o, mode=0, optimal_knn=g.get("optimal_knn"),
                                   optimal_radius=g.get("optimal_radius"))
        assert np.array_equal(status, g[sname + "_status"]), f"{name}/{sname} status"
        want = g[sname + "_out"]
        ok = status == 0
        both_nan = np.isnan(outs) & np.isnan(want)
        err = np.where(both_nan, 0.0, np.abs(outs - want))[:, ok]
        assert np.all(err <= 1e-12 * np.maximum(1.0, np.nan_to_num(np.abs(want[:, ok])))), f"{name}/{sname} values"


def test_port_matches_reference_on_random_ties(port, ref):
    rng = np.random.default_rng(11)
    for trial in range(12):
        n = int(rng.integers(2, 2500))
        span = int(rng.integers(1, 30))
        x, y, z = (rng.integers(0, span, n).astype(np.int32) for _ in range(3))
        X, Y, Z = (syn.to_double(v) for v in (x, y, z))
        tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
        assert np.array_equal(tp.export()["vind"], tr.export()["vind"])
        for k in (2, 9, 17, 33, 65):
            assert np.array_equal(tp.all_neighbors(k), tr.all_neighbors(k))


def _grid_plane(bounds):
    # FauxReader grid mode (io/FauxReader.cpp:99-130,238-258): count 4
    (x0, x1), (y0, y1), (z0, z1) = bounds
    pts = []
    dx, dy, dz = x1 - x0, y1 - y0, z1 - z0
    for i in range(4):
        x = i % dx if dx else 0
        y = ((i // dx) % dy if dx else i % dy) if dy else 0
        if dz:
            z = i // (dx * dy) if (dx and dy) else (i // dx if dx else i // dy)
        else:
            z = 0
        pts.append((x, y, z))
    return np.array(pts, dtype=np.float64).T


@pytest.mark.parametrize("bounds,normal", [
    (((0, 2), (0, 2), (0, 0)), (0, 0, 1)),
    (((0, 2), (0, 0), (0, 2)), (0, 1, 0)),
    (((0, 0), (0, 2), (0, 2)), (1, 0, 0)),
])
def test_reference_normal_planes(port, bounds, normal):
    X, Y, Z = _grid_plane(bounds)
    t = port.tree(X, Y, Z)
    outs, status = t.run_stage(abi.make_opts(abi.STAGE_NORMAL, knn=3), mode=0)
    assert (status == 0).all()
    for i in range(3):
        np.testing.assert_allclose(np.float32(outs[i]), normal[i], atol=1e-6)
    np.testing.assert_allclose(np.float32(outs[3]), 0.0, atol=1e-6)


@pytest.mark.parametrize("zs,expected", [
    ((0, 0, 1, 1), (-1, 0, 1)),   # RampPlane
    ((0, 1, 0, 1), (0, -1, 1)),   # RampPlane2
])
def test_reference_normal_ramps(port, zs, expected):
    X = np.array([0, 0, 1, 1.0])
    Y = np.array([0, 1, 0, 1.0])
    Z = np.array(zs, dtype=np.float64)
    t = port.tree(X, Y, Z)
    outs, status = t.run_stage(abi.make_opts(abi.STAGE_NORMAL, knn=3), mode=0)
    e = math.sqrt(2.0) / 2.0
    for i in range(3):
        np.testing.assert_allclose(np.float32(outs[i]), np.float32(expected[i] * e), atol=2e-7)
    np.testing.assert_allclose(np.float32(outs[3]), 0.0, atol=1e-7)


FEAT7 = abi.FEAT_DIMENSIONALITY | abi.FEAT_BIT["Omnivariance"] | abi.FEAT_BIT["Anisotropy"] | \
    abi.FEAT_BIT["Eigenentropy"] | abi.FEAT_BIT["EigenvalueSum"] | \
    abi.FEAT_BIT["SurfaceVariation"] | abi.FEAT_BIT["DemantkeVerticality"]


def _features(port, X, Y, Z, knn):
    t = port.tree(np.array(X, float), np.array(Y, float), np.array(Z, float))
    o = abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=knn, feature_mask=FEAT7)
    outs, status = t.run_stage(o, mode=0)
    assert (status == 0).all()
    return {name: np.float32(outs[i]) for i, name in enumerate(abi.stage_dims(o))}


def test_reference_features_linearity(port):
    f = _features(port, [0, 0, 0], [0, 0, 0], [0, 1, 2], 3)
    np.testing.assert_allclose(f["Linearity"], 1, atol=1e-6)
    np.testing.assert_allclose(f["Verticality"], 1, atol=1e-6)
    np.testing.assert_allclose(f["Planarity"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Scattering"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Omnivariance"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Anisotropy"], 1, atol=1e-6)
    assert np.isnan(f["Eigenentropy"]).all()
    np.testing.assert_allclose(f["EigenvalueSum"], 1, atol=1e-6)
    np.testing.assert_allclose(f["SurfaceVariation"], 0, atol=1e-6)
    np.testing.assert_allclose(f["DemantkeVerticality"], 1, atol=1e-6)


def test_reference_features_planarity(port):
    f = _features(port, [0, 1, 1, 0], [0, 0, 1, 1], [0, 0, 0, 0], 10)
    assert (f["Linearity"] <= 0.5).all()
    np.testing.assert_allclose(f["Verticality"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Planarity"], 1, atol=1e-6)
    np.testing.assert_allclose(f["Scattering"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Omnivariance"], 0, atol=1e-6)
    np.testing.assert_allclose(f["Anisotropy"], 1, atol=1e-6)
    assert np.isnan(f["Eigenentropy"]).all()
    np.testing.assert_allclose(f["EigenvalueSum"], 0.667, atol=1e-3)
    np.testing.assert_allclose(f["SurfaceVariation"], 0, atol=1e-6)
    np.testing.assert_allclose(f["DemantkeVerticality"], 0, atol=1e-6)


def test_reference_features_scattering(port):
    f = _features(port, [0, 1, 1, 0], [0, 0, 1, 1], [0, 0, 1, 2], 10)
    assert (f["Linearity"] <= 0.5).all()
    assert (f["Verticality"] >= 0.5).all()
    assert (f["Planarity"] <= 1).all()
    assert (f["Scattering"] >= 0.1).all()
    np.testing.assert_allclose(f["Omnivariance"], 0.458, atol=1e-3)
    np.testing.assert_allclose(f["Anisotropy"], 0.864, atol=1e-3)
    np.testing.assert_allclose(f["Eigenentropy"], 0.488, atol=1e-3)
    np.testing.assert_allclose(f["EigenvalueSum"], 1.583, atol=1e-3)
    np.testing.assert_allclose(f["SurfaceVariation"], 0.095, atol=1e-3)
    np.testing.assert_allclose(f["DemantkeVerticality"], 0.492, atol=1e-3)


def test_reference_kdindex_neighbors3d(port):
    pts = np.array([[0, 0, 0], [1, 1, 1], [3, 3, 3], [6, 6, 6], [10, 10, 10]], dtype=float).T
    t = port.tree(*pts)
    assert t.neighbors((0, 0, 0), 1)[0] == 0
    assert t.neighbors((1.1, 1.1, 1.1), 1)[0] == 1
    assert t.neighbors((3.3, 3.3, 3.3), 1)[0] == 2
    assert t.neighbors((6.1, 6.1, 6.1), 1)[0] == 3
    assert t.neighbors((15, 15, 15), 1)[0] == 4
    assert list(t.neighbors((0, 0, 0), 5)) == [0, 1, 2, 3, 4]
    assert list(t.neighbors((0, 0, 0), 25)) == [0, 1, 2, 3, 4]
    assert list(t.neighbors((3.1, 3.1, 3.1), 5)) == [2, 1, 3, 0, 4]
    assert list(t.neighbors((0, 0, 0), 2, 1)) == [0, 1]
    assert list(t.neighbors((0, 0, 0), 2, 2)) == [0, 2]
    assert list(t.neighbors((0, 0, 0), 2, 3)) == [0, 3]
    assert list(t.neighbors((0, 0, 0), 3, 2)) == [0, 2, 4]


def test_eigen_chain_matches_reference(port, ref):
    rng = np.random.default_rng(3)
    for _ in range(200):
        a = rng.normal(size=(3, 3)) * rng.choice([1e-6, 1, 1e6])
        a = a @ a.T
        if rng.random() < 0.3:
            a[2, :] = a[:, 2] = 0
        okp, evp, vp = port.eigen_chain(a)
        okr, evr, vr = ref.eigen_chain(a)
        assert okp == okr
        np.testing.assert_allclose(evp, evr, rtol=1e-13, atol=1e-13 * np.abs(evr).max())
        np.testing.assert_allclose(vp, vr, atol=1e-10)


def test_f64_mode_close_to_reference(port):
    g = U.golden("c1_terrain")
    t = port.tree(*U.doubles(g))
    o = U.opts_from_bytes(g["normal8_opts"])
    outs, status = t.run_stage(o, mode=1)
    assert np.array_equal(status, g["normal8_status"])
    # the reference narrows the centred coordinates to float: ~1e-7 differences
    assert np.nanmax(np.abs(outs - g["normal8_out"])) < 1e-4


def test_reference_normal_radius(port):
    # NormalFilterTest.cpp:255-313: two tilted 4-point patches, radius 2
    X = np.array([0, 0, 1, 1, 9, 9, 10, 10], np.float64)
    Y = np.array([0, 1, 0, 1, 9, 10, 9, 10], np.float64)
    Z = np.array([0, 1, 0, 1, 9, 10, 9, 10], np.float64)
    t = port.tree(X, Y, Z)
    o = abi.make_opts(abi.STAGE_NORMAL, knn=8, radius=2.0)
    out, status = t.run_stage(o, mode=0)
    e = math.sqrt(2.0) / 2.0
    assert (status == 0).all()
    np.testing.assert_allclose(out[0], 0.0, atol=1e-6)
    np.testing.assert_allclose(out[1], -e, atol=1e-6)
    np.testing.assert_allclose(out[2], e, atol=1e-6)
    np.testing.assert_allclose(out[3], 0.0, atol=1e-6)


def test_port_matches_reference_radius_stages(port, ref):
    """Radius search (KDImpl.hpp:398-415, nanoflann radiusSearch) and the
    stages' radius/min_k branches: same statuses; outputs equal up to the
    order in which equal-distance neighbours are summed."""
    rng = np.random.default_rng(12)
    x, y, z = syn.terrain(250_000, 0)
    m = (x < 3000) & (y < 3000)
    x, y, z = x[m], y[m], z[m]
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tp, tr = port.tree(X, Y, Z), ref.tree(X, Y, Z)
    kopt, ropt = syn.optimal_columns(len(x), 3, knn=10)
    for o in (abi.make_opts(abi.STAGE_NORMAL, radius=1.2),
              abi.make_opts(abi.STAGE_EIGENVALUES, radius=0.9, min_k=8),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, radius=1.5, min_k=5,
                            feature_mask=abi.FEAT_ALL)):
        a, sa = tp.run_stage(o, mode=0, optimal_knn=kopt, optimal_radius=ropt)
        b, sb = tr.run_stage(o, mode=0, optimal_knn=kopt, optimal_radius=ropt)
        assert np.array_equal(sa, sb)
        assert (sa == abi.ROW_RADIUS_FEW).any() or o.kind == abi.STAGE_NORMAL
        ok = sa == 0
        np.testing.assert_allclose(a[:, ok], b[:, ok], rtol=1e-9, atol=1e-12)

"""Parity of the sm_100a path with the oracle, through the C ABI.

* neighbour id sets bit-exact against the reference's (golden vectors made
  by the reference's nanoflann) and against the oracle port on larger clouds
* row status codes exact (the reference's skip / throw decisions)
* stage outputs within the stated tolerances of the FP64 accuracy oracle,
  and of the reference's own (float-narrowed) outputs on well-separated rows
* the device KD replica identical to the reference's tree
"""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu

GOLDEN_NBR = [n for n in U.golden_names()]


def f64_eigen(port, X, Y, Z, knn, stride=1):
    t = port.tree(X, Y, Z)
    o = abi.make_opts(abi.STAGE_EIGENVALUES, knn=knn, stride=stride)
    ev, st = t.run_stage(o, mode=1)
    return ev, st


@pytest.mark.parametrize("name", GOLDEN_NBR)
def test_neighbor_sets_match_reference_golden(nbg, name):
    g = U.golden(name)
    tile = nbg.tile(g["x"], g["y"], g["z"])
    for key in [k for k in g if k.startswith("nbr_k")]:
        knn = int(key[5:])
        ids, stats = nbg.neighbor_sets(tile, knn)
        want = U.sorted_rows(g[key])
        got = U.sorted_rows(ids)
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert bad.size == 0, f"{name} knn={knn}: {bad.size} rows differ, first {bad[:5]}"


@pytest.mark.parametrize("name", GOLDEN_NBR)
def test_stages_match_reference_golden(nbg, port, name):
    g = U.golden(name)
    X, Y, Z = U.doubles(g)
    tile = nbg.tile(g["x"], g["y"], g["z"])
    n = len(X)
    for key in [k for k in g if k.endswith("_opts")]:
        sname = key[:-5]
        o = U.opts_from_bytes(g[key])
        kopt, ropt = g.get("optimal_knn"), g.get("optimal_radius")
        outs, ex, stats = nbg.run(tile, [o], optimal_knn=kopt, optimal_radius=ropt)
        got_status = U.status_from_exceptions(n, ex)
        lam, _ = f64_eigen(port, X, Y, Z, o.knn)
        # accuracy oracle: same neighbour sets, FP64 without narrowing
        want64, st64 = port.tree(X, Y, Z).run_stage(o, mode=1, optimal_knn=kopt,
                                                     optimal_radius=ropt)
        want_ref = g[sname + "_out"]
        free64 = free_ref = None
        if o.kind == abi.STAGE_NORMAL and o.has_viewpoint:
            free64 = U.viewpoint_tangent_rows(o, X, Y, Z, want64)
            free_ref = U.viewpoint_tangent_rows(o, X, Y, Z, want_ref)
        elif o.kind == abi.STAGE_NORMAL and not o.always_up and f"nbr_k{o.knn}" in g:
            nb = g[f"nbr_k{o.knn}"]
            free64 = True
            free_ref = (U.symmetric_rows(g["x"], g["y"], g["z"], nb) |
                        U.sign_unstable_rows(port, g["x"], g["y"], g["z"], nb))
        U.compare_stage(o, outs[0], want64, g[sname + "_status"], got_status, lam=lam,
                        label=f"{name}/{sname} vs f64", sign_free=free64)
        # the reference's own outputs, on rows its float narrowing cannot blur
        U.compare_stage(o, outs[0], want_ref, g[sname + "_status"], got_status, lam=lam,
                        label=f"{name}/{sname} vs reference", gap_min=1e-2, sign_eps=1e-6,
                        sign_free=free_ref)


def test_kd_replica_matches_reference_tree(nbg, port):
    for name in ("c1_terrain", "c3_stress", "ties_lattice", "c2_mixture"):
        g = U.golden(name)
        tile = nbg.tile(g["x"], g["y"], g["z"])
        vind, nodes = nbg.kd_export(tile)
        want = port.tree(*U.doubles(g)).export()
        assert np.array_equal(vind.astype(np.uint64), want["vind"]), f"{name}: point order differs"
        internal = nodes["child1"] >= 0
        got_cuts = sorted(zip(nodes["divfeat"][internal].tolist(), nodes["divlow"][internal].tolist(),
                              nodes["divhigh"][internal].tolist()))
        wi = want["child1"] >= 0
        want_cuts = sorted(zip(want["divfeat"][wi].tolist(), want["divlow"][wi].tolist(),
                               want["divhigh"][wi].tolist()))
        assert got_cuts == want_cuts, f"{name}: split planes differ"
        leaves = sorted(zip(nodes["begin"][~internal].tolist(), nodes["end"][~internal].tolist()))
        want_leaves = sorted(zip(want["left"][~wi].tolist(), want["right"][~wi].tolist()))
        assert leaves == want_leaves, f"{name}: leaves differ"


@pytest.mark.parametrize("workload,knn", [("terrain", 8), ("mixture", 10), ("stress", 16),
                                          ("mixture", 32), ("stress", 64)])
def test_neighbor_sets_match_port_on_windows(nbg, port, workload, knn):
    if workload == "terrain":
        x, y, z = syn.terrain(250_000, 0)
    elif workload == "mixture":
        x, y, z = syn.mixture(4_000_000, 1)
        m = (x < 15000) & (y < 15000)
        x, y, z = x[m], y[m], z[m]
    else:
        x, y, z = syn.stress(4_000_000, 2)
        m = (x < 20000) & (y < 20000)
        x, y, z = x[m], y[m], z[m]
    tile = nbg.tile(x, y, z)
    ids, stats = nbg.neighbor_sets(tile, knn)
    want = port.tree(*(syn.to_double(v) for v in (x, y, z))).all_neighbors(knn + 1)
    bad = np.nonzero((U.sorted_rows(ids) != U.sorted_rows(want)).any(axis=1))[0]
    assert bad.size == 0, f"{workload} knn={knn}: {bad.size}/{len(x)} rows differ"


def test_fused_stages_share_one_pass(nbg, port):
    x, y, z = syn.stress(2_000_000, 2)
    m = (x < 12000) & (y < 12000)
    x, y, z = x[m], y[m], z[m]
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    kopt, ropt = syn.optimal_columns(len(x), 2, knn=16)
    stages = [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16),
              abi.make_opts(abi.STAGE_NORMAL, knn=16),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=16, feature_mask=abi.FEAT_ALL)]
    outs, ex, stats = nbg.run(tile, stages, optimal_knn=kopt, optimal_radius=ropt)
    t = port.tree(X, Y, Z)
    lam, _ = f64_eigen(port, X, Y, Z, 16)
    for i, o in enumerate(stages):
        want, st = t.run_stage(o, mode=1, optimal_knn=kopt, optimal_radius=ropt)
        U.compare_stage(o, outs[i], want, st, U.status_from_exceptions(len(x), ex, i), lam=lam,
                        label=f"fused stage {i}")


def test_host_output_keeps_skipped_rows(nbg):
    # 12 duplicates: every row's covariance is zero and is skipped
    x = np.array([5] * 12, np.int32)
    tile = nbg.tile(x, x, x)
    o = abi.make_opts(abi.STAGE_NORMAL, knn=8)
    buf = [np.full((4, 12), 7.0)]
    outs, ex, _ = nbg.run(tile, [o], fresh=False, out=buf)
    assert (buf[0] == 7.0).all()
    assert set(ex["code"].tolist()) == {abi.ROW_ZERO_COV}
    outs, ex, _ = nbg.run(tile, [o], fresh=True)
    assert (outs[0] == 0.0).all()


def test_invalid_options_fail_loudly(nbg):
    from gpupdal_b200.native import NbgError
    x = np.arange(50, dtype=np.int32)
    tile = nbg.tile(x, x * 3, x * 7)
    with pytest.raises(NbgError) as e:
        nbg.run(tile, [abi.make_opts(abi.STAGE_NORMAL, knn=65)])
    assert e.value.code == abi.NBG_ERR_INVALID
    with pytest.raises(NbgError) as e:
        nbg.run(tile, [abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=8, mode=7)])
    assert e.value.code == abi.NBG_ERR_INVALID
    with pytest.raises(NbgError) as e:
        nbg.run(tile, [abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=8,
                                     feature_mask=abi.FEAT_ALL)])
    assert e.value.code == abi.NBG_ERR_INVALID  # Density without OptimalKNN/Radius
    with pytest.raises(NbgError) as e:
        nbg.tile(x, x, x, scale=(0.01, 0.01, 0.001))
    assert e.value.code == abi.NBG_ERR_UNSUPPORTED


def test_knn_larger_than_cloud(nbg, port):
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 5, 17, 40):
        x, y, z = (rng.integers(0, 1000, n).astype(np.int32) for _ in range(3))
        tile = nbg.tile(x, y, z)
        ids, _ = nbg.neighbor_sets(tile, 64)
        want = port.tree(*(syn.to_double(v) for v in (x, y, z))).all_neighbors(65)
        assert np.array_equal(U.sorted_rows(ids), U.sorted_rows(want))
        for kind in (abi.STAGE_NORMAL, abi.STAGE_EIGENVALUES):
            o = abi.make_opts(kind, knn=64)
            outs, ex, _ = nbg.run(tile, [o])
            _, st = port.tree(*(syn.to_double(v) for v in (x, y, z))).run_stage(o, mode=0)
            assert np.array_equal(U.status_from_exceptions(n, ex), st)


def test_pipeline_json_runs_the_path_stages(nbg):
    from gpupdal_b200.stages import run_pipeline
    g = U.golden("c1_terrain")
    pipe = ('["input.las", {"type": "filters.normal", "knn": 8}, '
            '{"type": "filters.eigenvalues", "knn": 8, "normalize": true}, '
            '{"type": "writers.las", "filename": "out.las"}]')
    dims, log = run_pipeline(nbg, pipe, g["x"], g["y"], g["z"])
    assert "not run: file" in log and "not run: writers.las" in log
    tile = nbg.tile(g["x"], g["y"], g["z"])
    (nrm,), _, _ = nbg.run(tile, [abi.make_opts(abi.STAGE_NORMAL, knn=8)])
    (eig,), _, _ = nbg.run(tile, [abi.make_opts(abi.STAGE_EIGENVALUES, knn=8, normalize=True)])
    for k, name in enumerate(["NormalX", "NormalY", "NormalZ", "Curvature"]):
        assert np.array_equal(dims[name], nrm[k])
    for k in range(3):
        assert np.array_equal(dims[f"Eigenvalue{k}"], eig[k])
    # the golden reference outputs, through the same bars as the direct call
    want = g["normal8_out"]
    o = U.opts_from_bytes(g["normal8_opts"])
    got = np.stack([dims[n] for n in ("NormalX", "NormalY", "NormalZ", "Curvature")])
    lam, _ = f64_eigen(port_for_pipeline(), *U.doubles(g), 8)
    U.compare_stage(o, got, want, g["normal8_status"], g["normal8_status"], lam=lam,
                    label="pipeline normal8 vs reference", gap_min=1e-2, sign_eps=1e-6)


def port_for_pipeline():
    from oracle.oracle import Oracle
    return Oracle("port")


def test_covariancefeatures_optimized_per_point_k(nbg, port):
    """optimized=true: each point's k is its OptimalKNN (rounded, capped at n,
    without the +1 of knn; CovarianceFeaturesFilter.cpp:212-214); k = 0 rows
    have an empty neighbourhood and are skipped as zero covariance."""
    x, y, z = syn.mixture(4_000_000, 1)
    m = (x < 9000) & (y < 9000)
    x, y, z = x[m], y[m], z[m]
    n = len(x)
    rng = np.random.default_rng(5)
    kopt = rng.integers(3, 41, n).astype(np.float64)
    kopt[rng.random(n) < 0.01] = 0.0
    ropt = rng.uniform(0.3, 1.5, n)
    mask = (abi.FEAT_LINEARITY | abi.FEAT_PLANARITY | abi.FEAT_SCATTERING | abi.FEAT_ANISOTROPY |
            abi.FEAT_SURFACEVARIATION | abi.FEAT_DENSITY)
    o = abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10, feature_mask=mask, optimized=True)
    tile = nbg.tile(x, y, z)
    outs, ex, stats = nbg.run(tile, [o], optimal_knn=kopt, optimal_radius=ropt)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    want, st = port.tree(X, Y, Z).run_stage(o, mode=1, optimal_knn=kopt, optimal_radius=ropt)
    got_status = U.status_from_exceptions(n, ex)
    assert np.count_nonzero(st) == np.count_nonzero(kopt == 0)
    U.compare_stage(o, outs[0], want, st, got_status, label="optimized vs f64")


def _radius_lam(port, X, Y, Z, r):
    lam, _ = port.tree(X, Y, Z).run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, radius=r, min_k=0),
                                          mode=1)
    return lam


@pytest.mark.parametrize("workload,r", [("terrain", 1.0), ("mixture", 0.6), ("stress", 0.4)])
def test_radius_stages_match_oracle(nbg, port, ref, workload, r):
    """radius/min_k (KD3Index::radius, KDImpl.hpp:398-415): the set of points
    with squared FP64 distance < r*r; statuses (incl. too few within the
    radius) exact; outputs within the stated bars of the FP64 oracle and of
    the reference's own arithmetic."""
    if workload == "terrain":
        x, y, z = syn.terrain(250_000, 0)
        m = (x < 8000) & (y < 8000)
    elif workload == "mixture":
        x, y, z = syn.mixture(4_000_000, 1)
        m = (x < 7000) & (y < 7000)
    else:
        x, y, z = syn.stress(4_000_000, 2)
        m = (x < 7000) & (y < 7000)
    x, y, z = x[m], y[m], z[m]
    n = len(x)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    kopt, ropt = syn.optimal_columns(n, 4, knn=10)
    lam = _radius_lam(port, X, Y, Z, r)
    tile = nbg.tile(x, y, z)
    for o in (abi.make_opts(abi.STAGE_NORMAL, radius=r),
              abi.make_opts(abi.STAGE_EIGENVALUES, radius=r, min_k=6),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, radius=r, min_k=4, feature_mask=abi.FEAT_ALL)):
        outs, ex, _ = nbg.run(tile, [o], optimal_knn=kopt, optimal_radius=ropt)
        got_status = U.status_from_exceptions(n, ex)
        want64, st64 = port.tree(X, Y, Z).run_stage(o, mode=1, optimal_knn=kopt, optimal_radius=ropt)
        U.compare_stage(o, outs[0], want64, st64, got_status, lam=lam, label=f"{workload} radius vs f64")
        few = ex[ex["code"] == abi.ROW_RADIUS_FEW]
        if o.kind != abi.STAGE_NORMAL:
            assert (st64 == abi.ROW_RADIUS_FEW).sum() == len(few)
        wref, stref = ref.tree(X, Y, Z).run_stage(o, mode=0, optimal_knn=kopt, optimal_radius=ropt)
        U.compare_stage(o, outs[0], wref, stref, got_status, lam=lam,
                        label=f"{workload} radius vs reference", gap_min=1e-2, sign_eps=1e-6,
                        lam0_floor=1e-6)


def test_radius_normal_known_answer(nbg):
    # NormalFilterTest.cpp:255-313: two tilted 4-point patches, radius 2
    x = np.array([0, 0, 1, 1, 9, 9, 10, 10], np.int32)
    y = np.array([0, 1, 0, 1, 9, 10, 9, 10], np.int32)
    z = np.array([0, 1, 0, 1, 9, 10, 9, 10], np.int32)
    tile = nbg.tile(x, y, z, scale=(1.0, 1.0, 1.0))
    (out,), ex, _ = nbg.run(tile, [abi.make_opts(abi.STAGE_NORMAL, radius=2.0)])
    e = np.sqrt(2.0) / 2.0
    assert len(ex) == 0
    np.testing.assert_allclose(out[0], 0.0, atol=1e-6)
    np.testing.assert_allclose(out[1], -e, atol=1e-6)
    np.testing.assert_allclose(out[2], e, atol=1e-6)
    np.testing.assert_allclose(out[3], 0.0, atol=1e-6)


@pytest.mark.parametrize("workload", ["mixture", "stress", "ties_lattice"])
def test_strided_stages_match_oracle(nbg, port, ref, workload):
    """stride > 1 (KD3ImplT::neighbors, KDImpl.hpp:351-381): entries 0,
    stride, 2*stride, ... of the reference's own k*stride ordering (FP64
    distance, then its search's visiting order), so the lattice's many equal
    distances exercise the order inside the list, not only its boundary."""
    if workload == "ties_lattice":
        g = U.golden("ties_lattice")
        x, y, z = g["x"], g["y"], g["z"]
    elif workload == "mixture":
        x, y, z = syn.mixture(4_000_000, 1)
        m = (x < 8000) & (y < 8000)
        x, y, z = x[m], y[m], z[m]
    else:
        x, y, z = syn.stress(4_000_000, 2)
        m = (x < 8000) & (y < 8000)
        x, y, z = x[m], y[m], z[m]
    n = len(x)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    kopt, ropt = syn.optimal_columns(n, 6, knn=10)
    for o in (abi.make_opts(abi.STAGE_EIGENVALUES, knn=8, stride=2),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10, stride=3,
                            feature_mask=abi.FEAT_ALL, mode=abi.MODE_NORMALIZED)):
        outs, ex, _ = nbg.run(tile, [o], optimal_knn=kopt, optimal_radius=ropt)
        got_status = U.status_from_exceptions(n, ex)
        lam, _ = f64_eigen(port, X, Y, Z, o.knn, stride=o.stride)
        want64, st64 = port.tree(X, Y, Z).run_stage(o, mode=1, optimal_knn=kopt, optimal_radius=ropt)
        U.compare_stage(o, outs[0], want64, st64, got_status, lam=lam, label=f"{workload} stride vs f64")
        wref, stref = ref.tree(X, Y, Z).run_stage(o, mode=0, optimal_knn=kopt, optimal_radius=ropt)
        U.compare_stage(o, outs[0], wref, stref, got_status, lam=lam,
                        label=f"{workload} stride vs reference", gap_min=1e-2, sign_eps=1e-6,
                        lam0_floor=1e-6)

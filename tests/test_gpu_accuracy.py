"""Error statistics of every output dimension against the FP64 oracle, on the
three single-tile configurations:

* terrain: filters.normal knn=8 (always_up) on the 250k-point smooth terrain
* mixture: filters.covariancefeatures knn=10, feature_set=all, on the
  4M-point terrain / buildings / vegetation mixture
* stress: filters.eigenvalues knn=16 then filters.normal knn=16 on a
  ~2.9M-point window of the 32M-point stress tile (duplicates, wires)

For each dimension: the rows compared (status 0 on both sides, finite; for
eigenvector-dependent dimensions, rows whose relative eigen-gap is at least
1e-4; normals up to sign where the sign is not determined), the max and the
99.9th percentile of the absolute error, and of the relative error
|got - want| / max(|want|, s) with s the dimension's natural scale (the
largest eigenvalue, or its square root in SQRT mode, for eigenvalues and
eigenvalue-scaled features; 1 for unit-free ones).  The report is written
as JSON to $NBG_ACCURACY_OUT (default: the test's temporary directory); the
parity bars of tests/_util.py gate the test."""
import json
import os

import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu

SCALED = {"Eigenvalue0", "Eigenvalue1", "Eigenvalue2", "Omnivariance", "EigenvalueSum"}
VECTOR = {"NormalX", "NormalY", "NormalZ", "Verticality", "DemantkeVerticality"}


def _stats(opts, got, want, st_got, st_want, lam, tag):
    dims = abi.stage_dims(opts)
    n = got.shape[1]
    lmax = U.eigen_scale(lam)
    gap = (lam[1] - lam[0]) / lmax
    ok = (st_got == 0) & (st_want == 0)
    if opts.kind == abi.STAGE_COVARIANCEFEATURES and opts.mode == abi.MODE_SQRT:
        lscale = np.sqrt(lmax)
    else:
        lscale = lmax
    if opts.kind == abi.STAGE_NORMAL:
        # the sign of a horizontal normal (NormalZ within 1e-9 of 0) is rounding residue
        flat = np.abs(want[2]) < 1e-9
        got = got.copy()
        flip = flat & (np.abs(got[:3] - want[:3]).sum(0) > np.abs(got[:3] + want[:3]).sum(0))
        got[:3, flip] = -got[:3, flip]
    out = {}
    for d, name in enumerate(dims):
        rows = ok & np.isfinite(got[d]) & np.isfinite(want[d])
        if name in VECTOR:
            rows &= gap >= 1e-4
        if name in ("Omnivariance", "Eigenentropy"):
            rows &= lam[0] >= 1e-8 * lmax  # collinear rows: exact zero vs rounding residue
        err = np.abs(got[d][rows] - want[d][rows])
        scale = lscale[rows] if name in SCALED else np.ones(rows.sum())
        if name == "Eigenentropy":
            scale = np.maximum(np.abs(want[d][rows]), 1.0)
        if name in ("Density", "SurfaceVariation"):
            scale = np.maximum(np.abs(want[d][rows]), 1.0 if name == "SurfaceVariation" else 1e-300)
        if opts.normalize and name.startswith("Eigenvalue"):
            scale = np.ones(rows.sum())
        rel = err / np.maximum(np.abs(want[d][rows]), scale)
        out[name] = {
            "rows": int(rows.sum()), "of": int(n),
            "max_abs": float(err.max()) if err.size else 0.0,
            "p999_abs": float(np.quantile(err, 0.999)) if err.size else 0.0,
            "max_rel": float(rel.max()) if rel.size else 0.0,
            "p999_rel": float(np.quantile(rel, 0.999)) if rel.size else 0.0,
        }
    return out


def _config(name):
    if name == "terrain":
        x, y, z = syn.terrain(250_000, 0)
        return (x, y, z), [abi.make_opts(abi.STAGE_NORMAL, knn=8)], None
    if name == "mixture":
        x, y, z = syn.mixture(4_000_000, 1)
        return (x, y, z), [abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10,
                                         feature_mask=abi.FEAT_ALL)], syn.optimal_columns(len(x), 1)
    x, y, z = syn.stress(32_000_000, 2)
    m = (x < 15000) & (y < 15000)
    return (x[m], y[m], z[m]), [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16),
                                abi.make_opts(abi.STAGE_NORMAL, knn=16)], None


@pytest.mark.parametrize("name", ["terrain", "mixture", "stress"])
def test_error_statistics(nbg, port, tmp_path, name):
    (x, y, z), stages, opt = _config(name)
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    kopt, ropt = opt if opt is not None else (None, None)
    outs, ex, stats = nbg.run(tile, stages, optimal_knn=kopt, optimal_radius=ropt)
    tree = port.tree(X, Y, Z)
    report = {"config": name, "points": int(len(x)), "tie_rows": int(stats.tie_rows),
              "resolved_rows": int(stats.resolved_rows), "stages": []}
    for i, o in enumerate(stages):
        lam, _ = tree.run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, knn=o.knn), mode=1)
        want, st = tree.run_stage(o, mode=1, optimal_knn=kopt, optimal_radius=ropt)
        got_st = U.status_from_exceptions(len(x), ex, i)
        assert np.array_equal(got_st, st)
        # the parity bars gate; the statistics are the report
        U.compare_stage(o, outs[i], want, st, got_st, lam=lam, label=f"{name}/{i} vs f64")
        s = _stats(o, outs[i], want, got_st, st, lam, f"{name}/{i}")
        report["stages"].append({"kind": int(o.kind), "knn": int(o.knn), "dims": s})
    out_dir = os.environ.get("NBG_ACCURACY_OUT", str(tmp_path))
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, f"accuracy_{name}.json"), "w") as f:
        json.dump(report, f, indent=1)


def test_plain_fp64_eigensolve(nbg, port):
    # eigen_fp64: every row through the FP64 Eigen chain alone.  Same bars
    # against the FP64 oracle as the default FP32 Jacobi + FP64 polish path,
    # no row counted as handed from the fast solver to the chain, and the
    # eigenvalues of both forms agree to FP64 rounding.
    x, y, z = syn.stress(2_000_000, 2)
    m = (x < 20000) & (y < 20000)
    x, y, z = x[m], y[m], z[m]
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tile = nbg.tile(x, y, z)
    fast = [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16),
            abi.make_opts(abi.STAGE_NORMAL, knn=16),
            abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10, feature_mask=abi.FEAT_ALL
                          & ~abi.FEAT_DENSITY)]
    plain = [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16, eigen_fp64=True),
             abi.make_opts(abi.STAGE_NORMAL, knn=16, eigen_fp64=True),
             abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10, feature_mask=abi.FEAT_ALL
                           & ~abi.FEAT_DENSITY, eigen_fp64=True)]
    got_fast, ex_fast, _ = nbg.run(tile, fast)
    got, ex, stats = nbg.run(tile, plain)
    assert int(stats.resolved_rows) == 0
    tree = port.tree(X, Y, Z)
    for i, o in enumerate(plain):
        lam, _ = tree.run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, knn=o.knn), mode=1)
        want, st = tree.run_stage(o, mode=1)
        got_st = U.status_from_exceptions(len(x), ex, i)
        assert np.array_equal(got_st, st)
        assert np.array_equal(got_st, U.status_from_exceptions(len(x), ex_fast, i))
        U.compare_stage(o, got[i], want, st, got_st, lam=lam, label=f"eigen_fp64/{i} vs f64")
    ok = U.status_from_exceptions(len(x), ex, 0) == 0
    lmax = np.abs(got_fast[0][:, ok]).max(axis=0)
    assert np.all(np.abs(got[0][:, ok] - got_fast[0][:, ok]) <= 1e-12 * lmax)

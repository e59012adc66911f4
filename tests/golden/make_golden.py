"""Generates the golden vectors in tests/golden/ from the reference build.

    python tests/golden/make_golden.py

Inputs are seeded windows of the benchmark workloads, small tie-heavy and
edge-case clouds, and two of the reference's own test fixtures (read where they
lie in the reference tree named by the NBG_REFERENCE environment variable,
which must be set): the fork's
tie / duplicate points and the simple.las tile.  Outputs come from oracle/_ref/libnbg_ref.so, i.e. the
reference's own vendored nanoflann 1.3.1 and Eigen 3.4 compiled here (see
oracle/Makefile); this script must run where that library was built.  Each
fixture stores raw int32 coordinates (scale 0.01, offset 0), the
reference's neighbour lists (in the reference's order), stage outputs and
per-row status codes.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpupdal_b200 import abi  # noqa: E402
from gpupdal_b200 import synthetic as syn  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def window(x, y, z, w):
    m = (x < w * 100) & (y < w * 100)
    return x[m], y[m], z[m]


def stage_set(kind_list):
    out = []
    for name, o in kind_list:
        out.append((name, o))
    return out


REF = os.environ.get("NBG_REFERENCE", "")
if __name__ == "__main__" and not os.path.isdir(REF):
    sys.exit("set NBG_REFERENCE to the reference tree's root")


def record(ref, name, x, y, z, knns, stages, kopt=None, ropt=None, extra=None, out=None):
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    t = ref.tree(X, Y, Z)
    data = dict(x=x.astype(np.int32), y=y.astype(np.int32), z=z.astype(np.int32))
    for k in knns:
        data[f"nbr_k{k}"] = t.all_neighbors(k + 1).astype(np.uint32)
    for sname, o in stages:
        outs, status = t.run_stage(o, mode=0, optimal_knn=kopt, optimal_radius=ropt)
        data[f"{sname}_out"] = outs
        data[f"{sname}_status"] = status
        data[f"{sname}_opts"] = np.frombuffer(bytes(o), dtype=np.uint8)
    if kopt is not None:
        data["optimal_knn"] = kopt
        data["optimal_radius"] = ropt
    if extra:
        data.update(extra)
    os.makedirs(out or OUT, exist_ok=True)
    path = os.path.join(out or OUT, f"{name}.npz")
    np.savez_compressed(path, **data)
    print(path, len(x), os.path.getsize(path))


def main():
    ref = Oracle("reference")
    A = abi
    # C1 window: terrain, filters.normal knn=8 always_up
    x, y, z = syn.terrain(250_000, 0)
    x, y, z = window(x, y, z, 60)
    record(ref, "c1_terrain", x, y, z, [8],
           [("normal8", A.make_opts(A.STAGE_NORMAL, knn=8))])
    # C2 window: mixture, covariancefeatures knn=10 all (+ OptimalKNN/Radius)
    x, y, z = syn.mixture(4_000_000, 1)
    x, y, z = window(x, y, z, 20)
    kopt, ropt = syn.optimal_columns(len(x), 1, knn=10)
    record(ref, "c2_mixture", x, y, z, [10],
           [("cov10all", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=10, feature_mask=A.FEAT_ALL,
                                     mode=A.MODE_SQRT)),
            ("cov10raw", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=10,
                                     feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"],
                                     mode=A.MODE_RAW)),
            ("cov10norm", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=10,
                                      feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"],
                                      mode=A.MODE_NORMALIZED))],
           kopt=kopt, ropt=ropt)
    # C3 window: duplicates + wires, eigenvalues then normal, knn=16
    x, y, z = syn.stress(32_000_000, 2)
    x, y, z = window(x, y, z, 8)
    record(ref, "c3_stress", x, y, z, [16],
           [("eig16", A.make_opts(A.STAGE_EIGENVALUES, knn=16)),
            ("normal16", A.make_opts(A.STAGE_NORMAL, knn=16))])
    # tie-heavy integer lattice with duplicates: every knn the stages accept
    rng = np.random.default_rng(7)
    n = 3000
    x = rng.integers(0, 30, n).astype(np.int32)
    y = rng.integers(0, 30, n).astype(np.int32)
    z = rng.integers(0, 4, n).astype(np.int32)
    dup = rng.integers(0, n, 300)
    x, y, z = np.concatenate([x, x[dup]]), np.concatenate([y, y[dup]]), np.concatenate([z, z[dup]])
    record(ref, "ties_lattice", x, y, z, [1, 8, 16, 32, 64],
           [("normal8", A.make_opts(A.STAGE_NORMAL, knn=8)),
            ("normal8free", A.make_opts(A.STAGE_NORMAL, knn=8, always_up=False)),
            ("normal8vp", A.make_opts(A.STAGE_NORMAL, knn=8, viewpoint=(0.1, 0.2, 5.0))),
            ("eig32n", A.make_opts(A.STAGE_EIGENVALUES, knn=32, normalize=True)),
            ("cov64", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=64,
                                  feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"]))])
    # edge cases: tiny clouds, collinear and coplanar sets
    cases = {
        "n1": ([0], [0], [0]),
        "n2": ([0, 100], [0, 0], [0, 0]),
        "n3_line": ([0, 0, 0], [0, 0, 0], [0, 100, 200]),
        "n4_plane": ([0, 100, 100, 0], [0, 0, 100, 100], [0, 0, 0, 0]),
        "n4_scatter": ([0, 100, 100, 0], [0, 0, 100, 100], [0, 0, 100, 200]),
        "dups": ([5] * 12 + [7], [5] * 12 + [9], [1] * 12 + [2]),
        "line45": (list(range(0, 2000, 100)), list(range(0, 2000, 100)), [0] * 20),
    }
    # the fork's own tie / duplicate fixture (test/data/pdg/neighborhood-points.csv,
    # metres, read as raw = 100 * value at scale 0.01) with the stages of its
    # deterministic-ties pipeline (test/data/pdg/hybrid-neighborhood-deterministic-ties.json)
    pts = np.loadtxt(os.path.join(REF, "test/data/pdg/neighborhood-points.csv"), delimiter=",",
                     skiprows=1)[:, :3]
    raw = np.rint(pts * 100).astype(np.int32)
    record(ref, "fork_neighborhood_points", raw[:, 0], raw[:, 1], raw[:, 2], [1, 2, 3, 7],
           [("normal3free", A.make_opts(A.STAGE_NORMAL, knn=3, always_up=False)),
            ("eig3n", A.make_opts(A.STAGE_EIGENVALUES, knn=3, normalize=True)),
            ("cov3", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=3,
                                 feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"]))])
    # a real LAS tile, the reference's test/data/las/simple.las (LAS 1.2, point
    # format 3, scale 0.01, offset -0): its raw X/Y/Z, and its header block and
    # point records for the LAS ingest tests
    from gpupdal_b200 import las
    lf = las.LasFile(os.path.join(REF, "test/data/las/simple.las"))
    assert lf.scale == (0.01, 0.01, 0.01) and all(o == 0 for o in lf.offset)
    lx, ly, lz = lf.raw_xyz()
    hdr = np.asarray(lf.map[:lf.info["offset_to_points"]]).copy()
    record(ref, "las_simple", lx, ly, lz, [8, 16],
           [("normal8", A.make_opts(A.STAGE_NORMAL, knn=8)),
            ("eig16", A.make_opts(A.STAGE_EIGENVALUES, knn=16)),
            ("cov10", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=10,
                                  feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"]))],
           extra={"las_header": hdr, "las_records": np.asarray(lf.records).copy()})
    # the fork's approximatecoplanar fixtures (test/data/pdg/approximatecoplanar-
    # boundary.csv: six points on the axes whose spectrum puts the thresholds
    # exactly on the boundary, with the options of hybrid-approximatecoplanar-
    # boundary.json and -ties.json; approximatecoplanar-widened.csv: four
    # coincident points).  Kept in fixtures/, outside the device parity sets:
    # the oracle is pinned to them on the CPU.
    fx = os.path.join(OUT, "fixtures")
    for fname, gname, runs in [
            ("approximatecoplanar-boundary.csv", "fork_coplanar_boundary",
             [("cop6", A.consumer_opts(A.STAGE_APPROXIMATECOPLANAR, knn=6, thresh1=25.0, thresh2=5.0)),
              ("cop3", A.consumer_opts(A.STAGE_APPROXIMATECOPLANAR, knn=3, thresh1=25.0, thresh2=6.0)),
              ("rank6", A.consumer_opts(A.STAGE_ESTIMATERANK, knn=6)),
              ("eig5", A.make_opts(A.STAGE_EIGENVALUES, knn=5))]),
            ("approximatecoplanar-widened.csv", "fork_coplanar_coincident",
             [("cop3", A.consumer_opts(A.STAGE_APPROXIMATECOPLANAR, knn=3)),
              ("rank3", A.consumer_opts(A.STAGE_ESTIMATERANK, knn=3))])]:
        pts = np.loadtxt(os.path.join(REF, "test/data/pdg", fname), delimiter=",", skiprows=1)[:, :3]
        raw = np.rint(pts * 100).astype(np.int32)
        record(ref, gname, raw[:, 0], raw[:, 1], raw[:, 2], [1, 2, 3], runs, out=fx)
    for cname, (cx, cy, cz) in cases.items():
        cx, cy, cz = (np.array(v, dtype=np.int32) for v in (cx, cy, cz))
        record(ref, f"edge_{cname}", cx, cy, cz, [3, 8],
               [("normal3", A.make_opts(A.STAGE_NORMAL, knn=3)),
                ("eig3", A.make_opts(A.STAGE_EIGENVALUES, knn=3)),
                ("cov3", A.make_opts(A.STAGE_COVARIANCEFEATURES, knn=3,
                                     feature_mask=A.FEAT_ALL & ~A.FEAT_BIT["Density"]))])


if __name__ == "__main__":
    main()

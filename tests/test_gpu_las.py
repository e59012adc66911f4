"""LAS ingest on the device: a tile made from LAS point records (host-mapped
or already on the device) is the tile made from the same raw coordinates, so
its neighbour sets and stage outputs are identical bit for bit, and they meet
the oracle's bars."""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import las
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu

SCALE = (0.01, 0.01, 0.01)
OFFSET = (512000.0, 4100000.0, 120.0)


def _window(n, seed, side):
    x, y, z = syn.stress(n, seed)
    m = (x < side) & (y < side)
    return x[m], y[m], z[m]


def _stages():
    return [abi.make_opts(abi.STAGE_NORMAL, knn=8, viewpoint=(512100.0, 4100100.0, 300.0)),
            abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10,
                          feature_mask=abi.FEAT_ALL & ~abi.FEAT_DENSITY)]


@pytest.mark.parametrize("version,fmt,extra", [((1, 2), 3, 5), ((1, 4), 6, 0), ((1, 2), 0, 1)])
def test_las_tile_equals_array_tile(nbg, tmp_path, version, fmt, extra):
    import torch
    x, y, z = _window(2_000_000, 2, 9000)
    p = tmp_path / "w.las"
    rng = np.random.default_rng(5)
    base = {0: 20, 1: 28, 2: 26, 3: 34, 6: 30}[fmt]
    fill = rng.integers(0, 256, (len(x), base + extra - 12))
    las.write_las(p, x, y, z, scale=SCALE, offset=OFFSET, version=version, point_format=fmt,
                  extra_bytes=extra, fill=fill)
    f = las.LasFile(p)
    t_arr = nbg.tile(x, y, z, scale=SCALE, offset=OFFSET)
    t_host = nbg.tile_from_las(f)
    dev = torch.from_numpy(np.asarray(f.records).copy()).cuda()
    t_dev = nbg.tile_from_las(f, records=dev)
    want_ids, _ = nbg.neighbor_sets(t_arr, 10)
    want, want_ex, _ = nbg.run(t_arr, _stages())
    for t in (t_host, t_dev):
        assert t.n == len(x)
        ids, _ = nbg.neighbor_sets(t, 10)
        assert np.array_equal(U.sorted_rows(ids), U.sorted_rows(want_ids))
        got, ex, _ = nbg.run(t, _stages())
        for g, w in zip(got, want):
            assert np.array_equal(g, w, equal_nan=True)
        assert np.array_equal(np.sort(ex, order=["stage", "point_id"]),
                              np.sort(want_ex, order=["stage", "point_id"]))


def test_las_host_records_cross_staging_chunks(nbg, tmp_path):
    # 4M records of 38 bytes: three 64 MiB staging chunks
    x, y, z = syn.stress(4_000_000, 3)
    assert len(x) * 38 > (64 << 20)
    p = tmp_path / "big.las"
    las.write_las(p, x, y, z, scale=SCALE, offset=OFFSET, version=(1, 4), point_format=8)
    t_las = nbg.tile_from_las(p)
    t_arr = nbg.tile(x, y, z, scale=SCALE, offset=OFFSET)
    a, _ = nbg.neighbor_sets(t_las, 8)
    b, _ = nbg.neighbor_sets(t_arr, 8)
    assert np.array_equal(U.sorted_rows(a), U.sorted_rows(b))


def test_las_tile_meets_oracle(nbg, port, tmp_path):
    x, y, z = _window(2_000_000, 4, 6000)
    p = tmp_path / "o.las"
    las.write_las(p, x, y, z, scale=SCALE, offset=OFFSET, version=(1, 2), point_format=1)
    tile = nbg.tile_from_las(p)
    X, Y, Z = (syn.to_double(v, SCALE[d], OFFSET[d]) for d, v in enumerate((x, y, z)))
    t = port.tree(X, Y, Z)
    lam, _ = t.run_stage(abi.make_opts(abi.STAGE_EIGENVALUES, knn=8), mode=1)
    outs, ex, _ = nbg.run(tile, _stages()[:1])
    want, st = t.run_stage(_stages()[0], mode=1)
    U.compare_stage(_stages()[0], outs[0], want, st, U.status_from_exceptions(len(x), ex),
                    lam=lam, label="LAS tile vs f64",
                    sign_free=U.viewpoint_tangent_rows(_stages()[0], X, Y, Z, want))


def test_las_rejects_short_records(nbg):
    import ctypes
    h = ctypes.c_void_p()
    sc = (ctypes.c_double * 3)(*SCALE)
    buf = np.zeros(64, np.uint8)
    rc = nbg.lib.nbg_tile_upload_las(nbg.h, buf.ctypes.data, 4, 11, 0, sc, sc, None,
                                     ctypes.byref(h))
    assert rc == abi.NBG_ERR_INVALID and not h.value


def test_reference_las_fixture_matches_reference_outputs(nbg, tmp_path):
    # the reference's simple.las through LAS ingest: neighbour sets bit-exact
    # against the reference's, and stage outputs identical to the array tile's
    # (which the golden parity tests hold to the reference's own outputs)
    g = U.golden("las_simple")
    p = tmp_path / "simple.las"
    p.write_bytes(g["las_header"].tobytes() + g["las_records"].tobytes())
    t = nbg.tile_from_las(las.LasFile(p))
    t_arr = nbg.tile(g["x"], g["y"], g["z"])
    assert t.n == 1065
    for k in (8, 16):
        ids, _ = nbg.neighbor_sets(t, k)
        assert np.array_equal(U.sorted_rows(ids), U.sorted_rows(g[f"nbr_k{k}"]))
    stages = [U.opts_from_bytes(g[f"{s}_opts"]) for s in ("normal8", "eig16", "cov10")]
    got, ex, _ = nbg.run(t, stages)
    want, want_ex, _ = nbg.run(t_arr, stages)
    for i, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b, equal_nan=True)
        assert np.array_equal(U.status_from_exceptions(t.n, ex, i), g[[
            "normal8_status", "eig16_status", "cov10_status"][i]])
    assert np.array_equal(np.sort(ex, order=["stage", "point_id"]),
                          np.sort(want_ex, order=["stage", "point_id"]))

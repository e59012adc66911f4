"""The group select (nbg_group.cu) against the per-thread select and the oracle.

Every setting of the queries-per-group knob (8, 16, 32) and the per-thread
ring search (0) must give the same neighbour sets, the same row statuses and
bit-identical stage outputs: both select kernels compare exact integer squared
distances and hand the same rows to the tie-order resolver and the exact KD
path.  Checked on tiles that stress the group's fallbacks: the stress mixture
(duplicates, wires, sparse vegetation edges), a tiny tile whose boxes cover
the whole tile, a lattice of equal distances, and per-row k (optimized).
"""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from tests import _util as U

pytestmark = pytest.mark.gpu

GROUPS = (0, 1, 2, 8, 16, 32)


def _clouds():
    x, y, z = syn.stress(8_000_000, 7)
    m = (x < 12000) & (y < 12000)
    yield "stress", (x[m], y[m], z[m])
    rng = np.random.default_rng(3)
    yield "tiny", tuple(rng.integers(0, 500, 40).astype(np.int32) for _ in range(3))
    g = np.arange(24, dtype=np.int32) * 7
    gx, gy, gz = np.meshgrid(g, g, g[:6], indexing="ij")
    yield "lattice", (gx.ravel().copy(), gy.ravel().copy(), gz.ravel().copy())


@pytest.mark.parametrize("name,xyz", list(_clouds()), ids=lambda v: v if isinstance(v, str) else "")
def test_group_sizes_agree_with_oracle(nbg, port, name, xyz):
    x, y, z = xyz
    X, Y, Z = (syn.to_double(v) for v in (x, y, z))
    tree = port.tree(X, Y, Z)
    stages = [abi.make_opts(abi.STAGE_EIGENVALUES, knn=16),
              abi.make_opts(abi.STAGE_NORMAL, knn=16),
              abi.make_opts(abi.STAGE_NORMAL, knn=8, always_up=False)]
    want_ids = {k: U.sorted_rows(tree.all_neighbors(k + 1)) for k in (8, 16)}
    base = None
    for G in GROUPS:
        tile = nbg.tile(x, y, z)
        tile.set_select(G)
        for k in (8, 16):
            ids, _ = nbg.neighbor_sets(tile, k)
            bad = np.flatnonzero((U.sorted_rows(ids) != want_ids[k]).any(axis=1))
            assert bad.size == 0, f"{name} G={G} knn={k}: {bad.size} rows differ, first {bad[:5]}"
        outs, ex, stats = nbg.run(tile, stages)
        tile.free()
        if base is None:
            base = (outs, ex)
            continue
        for i in range(len(stages)):
            assert np.array_equal(outs[i], base[0][i], equal_nan=True), f"{name} G={G} stage {i}"
        assert np.array_equal(np.sort(ex, order=["point_id", "stage"]),
                              np.sort(base[1], order=["point_id", "stage"])), f"{name} G={G} rows"


def test_group_optimized_per_row_k(nbg):
    x, y, z = syn.mixture(500_000, 4)
    n = len(x)
    rng = np.random.default_rng(9)
    kopt = rng.integers(0, 30, n).astype(np.float64)
    ropt = rng.uniform(0.3, 1.5, n)
    st = abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=10, optimized=True,
                       feature_mask=abi.FEAT_ALL)
    res = []
    for G in GROUPS:
        tile = nbg.tile(x, y, z)
        tile.set_select(G)
        outs, ex, _ = nbg.run(tile, [st], optimal_knn=kopt, optimal_radius=ropt)
        tile.free()
        res.append((outs[0], np.sort(ex, order=["point_id", "stage"])))
    for G, (o, e) in zip(GROUPS[1:], res[1:]):
        assert np.array_equal(o, res[0][0], equal_nan=True), f"G={G}"
        assert np.array_equal(e, res[0][1]), f"G={G} rows"


def test_group_setting_refused(nbg):
    x, y, z = syn.terrain(10_000, 0)
    tile = nbg.tile(x, y, z)
    from gpupdal_b200.native import NbgError
    with pytest.raises(NbgError):
        tile.set_select(12)
    with pytest.raises(NbgError):
        tile.set_select(32, first_margin=0.0)

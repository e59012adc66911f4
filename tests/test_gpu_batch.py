"""The batched form (nbg_run_batch): tiles of uneven size and knn in one
graph-captured queue give, tile by tile, exactly the plain per-tile results;
a replay of the captured graph and the uncaptured launch agree too."""
import numpy as np
import pytest

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn
from gpupdal_b200.native import record_columns

pytestmark = pytest.mark.gpu


def _batch(nbg, count=12, seed=100):
    import torch
    x, y, z = syn.mixture(4_000_000, 1)
    rng = np.random.default_rng(seed)
    tiles, stages, outs, cols, optimal, raw = [], [], [], [], [], []
    for i in range(count):
        side = int(rng.integers(2000, 20000))
        x0, y0 = (int(v) for v in rng.integers(0, 50000 - side, 2))
        m = (x >= x0) & (x < x0 + side) & (y >= y0) & (y < y0 + side)
        knn = int(rng.choice([8, 16, 32]))
        st = [abi.make_opts(abi.STAGE_NORMAL, knn=knn),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=knn, feature_mask=abi.FEAT_ALL)]
        n = int(m.sum())
        dev = [torch.from_numpy(np.ascontiguousarray(v[m])).cuda() for v in (x, y, z)]
        tiles.append(nbg.tile(*dev))
        raw.append((x[m], y[m], z[m]))
        rec = torch.full((n, 16), float("nan"), dtype=torch.float64, device="cuda")
        outs.append(rec)
        cols.append(record_columns(rec.data_ptr(), st, 128, 1))
        kopt, ropt = syn.optimal_columns(n, seed + i, knn=knn)
        optimal.append((torch.from_numpy(kopt).cuda(), torch.from_numpy(ropt).cuda()))
        stages.append(st)
    return tiles, stages, outs, cols, optimal, raw


def _plain(nbg, raw, st, kopt, ropt):
    t = nbg.tile(*raw)
    res, ex, _ = nbg.run(t, st, optimal_knn=kopt, optimal_radius=ropt)
    t.free()
    return np.concatenate([r for r in res]), np.sort(ex, order=["point_id", "stage", "code"])


def test_batch_matches_plain_per_tile(nbg):
    tiles, stages, outs, cols, optimal, raw = _batch(nbg)
    ex_g, stats = nbg.run_batch(tiles, stages, cols, optimal, graph=True)
    assert stats.points == sum(len(r[0]) for r in raw)
    first = [o.cpu().numpy().copy() for o in outs]
    for o in outs:
        o.fill_(float("nan"))
    ex_r, _ = nbg.run_batch(tiles, stages, cols, optimal, graph=True)   # graph replay
    replay = [o.cpu().numpy().copy() for o in outs]
    for o in outs:
        o.fill_(float("nan"))
    ex_e, _ = nbg.run_batch(tiles, stages, cols, optimal, graph=False)  # eager launches
    eager = [o.cpu().numpy().copy() for o in outs]
    for i in range(len(tiles)):
        kopt, ropt = (v.cpu().numpy() for v in optimal[i])
        want, wex = _plain(nbg, raw[i], stages[i], kopt, ropt)
        nd = want.shape[0]
        for name, got, ex in (("graph", first, ex_g), ("replay", replay, ex_r),
                              ("eager", eager, ex_e)):
            g = got[i][:, :nd].T
            # rows a stage skips keep the output's previous value (NaN here, 0 in plain)
            skip = np.zeros(g.shape[1], bool)
            skip[ex[i]["point_id"]] = True
            assert np.array_equal(g[:, ~skip], want[:, ~skip], equal_nan=True), f"tile {i} {name}"
            assert np.array_equal(np.sort(ex[i], order=["point_id", "stage", "code"]), wex), \
                f"tile {i} {name}: exceptions differ"

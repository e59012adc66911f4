"""The batched tile set and its two ways of running.

A set is `count` tiles with log-normal sizes (median 200k points, sigma 1.0,
clipped to [20k, 4M]) of the building/vegetation/terrain mixture, knn uniform
in {8, 16, 32} per tile, and each tile running filters.normal plus
filters.covariancefeatures (feature_set=all, with OptimalKNN/OptimalRadius
columns).  Tiles are uniform subsamples of one pre-generated, pre-shuffled
mixture cloud, so a set of ~10^8 points generates in seconds.

Coordinates, OptimalKNN/OptimalRadius and outputs stay device-resident; a
step uploads every tile from its resident coordinates (a fresh tile: grid and
KD replica are built inside the step), runs it, and frees it:
  plain    one nbg_run per tile, tile after tile
  batched  one nbg_run_batch over all tiles (graph-captured queue)
"""
from __future__ import annotations

import numpy as np

from . import abi
from . import synthetic as syn
from .native import record_columns

RECORD = 128  # bytes per point: NormalX..Curvature (4) + 11 features, padded


def make_set(count=256, seed=100, pool_points=8_000_000, median=200_000, sigma=1.0,
             lo=20_000, hi=4_000_000, device="cuda"):
    import torch
    rng = np.random.default_rng(seed)
    x, y, z = syn.mixture(pool_points, seed)
    perm = rng.permutation(pool_points)
    x, y, z = x[perm], y[perm], z[perm]
    sizes = np.clip(np.exp(rng.normal(np.log(median), sigma, count)), lo, min(hi, pool_points))
    tiles = []
    for i in range(count):
        n = int(sizes[i])
        s0 = int(rng.integers(0, pool_points))
        idx = (s0 + np.arange(n)) % pool_points
        knn = int(rng.choice((8, 16, 32)))
        st = [abi.make_opts(abi.STAGE_NORMAL, knn=knn),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=knn, feature_mask=abi.FEAT_ALL)]
        kopt, ropt = syn.optimal_columns(n, seed + i, knn=knn)
        dev = [torch.from_numpy(np.ascontiguousarray(v[idx])).to(device) for v in (x, y, z)]
        rec = torch.empty((n, RECORD // 8), dtype=torch.float64, device=device)
        tiles.append(dict(xyz=dev, n=n, knn=knn, stages=st, rec=rec,
                          cols=record_columns(rec.data_ptr(), st, RECORD, 1),
                          optimal=(torch.from_numpy(kopt).to(device), torch.from_numpy(ropt).to(device))))
    return tiles


def step_plain(ctx, tset):
    stats = []
    for t in tset:
        tile = ctx.tile(*t["xyz"])
        _, st = ctx.run_columns(tile, t["stages"], t["cols"], optimal_knn=t["optimal"][0],
                                optimal_radius=t["optimal"][1], aux_on_device=True)
        tile.free()
        stats.append(st)
    return stats


def step_batched(ctx, tset, graph=True, autotune=False):
    tiles = [ctx.tile(*t["xyz"]) for t in tset]
    _, st = ctx.run_batch(tiles, [t["stages"] for t in tset], [t["cols"] for t in tset],
                          [t["optimal"] for t in tset], graph=graph, autotune=autotune)
    for tile in tiles:
        tile.free()
    return st

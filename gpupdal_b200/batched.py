"""The batched tile set and its two ways of running.

A set is `count` tiles with log-normal sizes (median 200k points, sigma 1.0,
clipped to [20k, 4M]) of the building/vegetation/terrain mixture, knn uniform
in {8, 16, 32} per tile, and each tile running filters.normal plus
filters.covariancefeatures (feature_set=all, with OptimalKNN/OptimalRadius
columns).  Tile i is a compact mixture tile of its own seed (seed + i, the
seeds 100-355 of the batched configuration by default), generated in
parallel worker processes.

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


def make_set(count=256, seed=100, median=200_000, sigma=1.0, lo=20_000, hi=4_000_000,
             device="cuda"):
    """`count` compact tiles: tile i is syn.tile(n_i, seed + i) (the mixture at
    16 points per square metre, its own seed), n_i log-normal (median, sigma)
    clipped to [lo, hi], knn uniform in {8, 16, 32}."""
    import torch
    rng = np.random.default_rng(seed)
    sizes = syn.batched_sizes(count, seed, median, sigma, lo, hi)
    clouds = syn.tiles(sizes, [seed + i for i in range(count)])
    tiles = []
    for i, (x, y, z) in enumerate(clouds):
        n = len(x)
        knn = int(rng.choice((8, 16, 32)))
        st = [abi.make_opts(abi.STAGE_NORMAL, knn=knn),
              abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=knn, feature_mask=abi.FEAT_ALL)]
        kopt, ropt = syn.optimal_columns(n, seed + i, knn=knn)
        dev = [torch.from_numpy(np.ascontiguousarray(v)).to(device) for v in (x, y, z)]
        rec = torch.empty((n, RECORD // 8), dtype=torch.float64, device=device)
        tiles.append(dict(xyz=dev, n=n, knn=knn, stages=st, rec=rec, seed=seed + i,
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

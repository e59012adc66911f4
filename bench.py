#!/usr/bin/env python
"""Benchmark of the neighbourhood-geometry path on B200.

Workload (one "step"): filters.eigenvalues knn=16 followed by filters.normal
knn=16 on one 32,000,000-point tile of the stress mixture (terrain, building
faces, vegetation, 2 % exact duplicates, 3 % collinear wire points; seeded
synthetic, int32 at 0.01 m) — index build, kNN, covariance, eigensolve and
all seven output dimensions, the tie rows answered by the exact KD replica.

  value  Mpts/s with the tile's coordinates resident in HBM when the timed
         region starts (device-to-device tile upload + nbg_run, device outputs)
  e2e    the same through the C ABI with pinned host buffers: H2D of the
         coordinates, nbg_run, D2H of the outputs inside the timed region

Multi-GPU (torchrun): one replica tile per rank (different seeds), no
collective on the data path; value = all ranks' points / max-over-ranks time.

--impl reference times the reference's CPU implementation (oracle/_ref:
nanoflann 1.3.1 + Eigen 3.4 built from the reference's sources; the oracle
port when that library is absent) on the host cores, on a bounded window of
the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpts/s k=16 normals+eigen, served vs plain @<=1e-5 rel err; p50/p99 latency"
BYTES_PER_POINT = 20 + 8 * 7 + 1  # sorted xyz+id, id permutation, 7 f64 outputs, status
# Per select kernel (the one the autotuner chose for the timed tile): the query
# kernels, their DRAM bytes per point (read + write) and the select kernel's
# active lanes per warp instruction and issue-slot fraction, from one ncu
# capture per kernel of the same workload at 4M points (64-byte device
# records), summarised under profiles/.
QUERY_PROFILES = {
    0: {"kernel": "knn_select_kernel+knn_finish_kernel",
        # (182.3 + 628.9) MB / 4e6
        "traffic": 202.8, "lanes": 8.91, "issue": 0.793, "dram_pct": 0.54},
    2: {"kernel": "knn_select_loc_kernel+knn_retry_finish_kernel+knn_finish_kernel",
        # select (70.4 + 99.3) + handed-back rows (10.1 + 0.1) + finish (363.1 + 255.5) MB / 4e6
        "traffic": 199.6, "lanes": 10.13, "issue": 0.662, "dram_pct": 0.58},
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)  # ~1.2 s timed: several clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=32_000_000)
    ap.add_argument("--knn", type=int, default=16)
    ap.add_argument("--select", type=int, default=None,
                    help="select kernel for the main line's tiles instead of the autotuner's "
                         "choice (nbg_tile_set_select: 0, 1, 2, 8, 16, 32)")
    ap.add_argument("--cell-factor", type=float, default=None,
                    help="cell factor for the main line's tiles instead of the autotuner's "
                         "choice (nbg_tile_tune)")
    ap.add_argument("--cpu-sample", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the plain FP64 eigensolve comparison leg")
    ap.add_argument("--served-requests", type=int, default=64)
    ap.add_argument("--served-rate", type=float, default=20.0)
    ap.add_argument("--served-slots", type=int, default=4)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-sweep", default="",
                    help="comma-separated request rates (req/s, 0: all at once): run only the "
                         "served stream (--served-requests requests) at each rate, one JSON "
                         "line per rate")
    ap.add_argument("--batch-tiles", type=int, default=256)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the extra stages / consumers / LAS ingest leg")
    ap.add_argument("--cpu-only", action="store_true",
                    help="(internal) time the CPU baselines in this fresh process and print them "
                         "as one JSON object")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (read-only queries)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(points, seed):
    from gpupdal_b200 import synthetic as syn
    return syn.stress(points, seed)


def stages(knn):
    from gpupdal_b200 import abi
    return [abi.make_opts(abi.STAGE_EIGENVALUES, knn=knn),
            abi.make_opts(abi.STAGE_NORMAL, knn=knn, always_up=True)]


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference(x, y, z, knn, sample, kind=None, single_thread=False, reps=1):
    """Times the reference's CPU path (KD build + eigenvalues + normal) on a
    spatially contiguous window of `sample` points: all host threads for the
    rows in fixed contiguous chunks, and the KD build on min(8, cores)
    threads; with reps > 1, after one untimed run, the median of `reps` runs.
    With `single_thread`, also one thread for both (the stage's own
    semantics: one thread per view) on a window of a quarter of the points,
    after one untimed run."""
    from gpupdal_b200 import synthetic as syn
    from oracle import oracle as orc
    if kind is None:
        kind = "reference" if orc.available("reference") else "port"
    if not orc.available(kind):
        orc.build()
    o = orc.Oracle(kind)

    def window(count):
        # square window from the tile's corner holding about `count` points
        side = int(round(50000 * np.sqrt(min(1.0, count / len(x)))))
        m = (x < side) & (y < side)
        return side, tuple(syn.to_double(v[m]) for v in (x, y, z))

    def timed_run(xyz, threads):
        t0 = time.perf_counter()
        t = o.tree(*xyz, build_threads=threads if threads == 1 else 0)
        for st in stages(knn):
            t.run_stage(st, mode=0, threads=threads)
        return time.perf_counter() - t0

    threads = os.cpu_count() or 1
    side, xyz = window(sample)
    if reps > 1:
        timed_run(xyz, threads)
        dt = statistics.median(timed_run(xyz, threads) for _ in range(reps))
    else:
        dt = timed_run(xyz, threads)
    n = len(xyz[0])
    out = {"value": n / dt / 1e6, "unit": "Mpts/s", "cores": threads,
           "kind": kind, "sample": f"{n}-point window ({side / 100:.0f} x "
                                   f"{side / 100:.0f} m) of the same tile: KD build "
                                   f"(min(8, cores) threads) + eigenvalues + normal, "
                                   f"{threads} threads",
           "seconds": dt, "cpu_model": cpu_model(), "nproc": threads}
    if single_thread:
        side1, xyz1 = window(sample // 4)
        if reps > 1:
            timed_run(xyz1, 1)
        dt1 = timed_run(xyz1, 1)
        n1 = len(xyz1[0])
        out["single_thread"] = {"value": n1 / dt1 / 1e6, "unit": "Mpts/s", "cores": 1,
                                "seconds": dt1,
                                "sample": f"{n1}-point window ({side1 / 100:.0f} x "
                                          f"{side1 / 100:.0f} m): KD build + eigenvalues "
                                          f"+ normal, one thread"}
    return out


def fp64_leg(ctx, args, dxyz, drec, sts, steps):
    """The main workload with every row solved by the FP64 Eigen chain alone
    (eigen_fp64: a plain FP64 eigensolve) against the FP32 Jacobi + FP64
    polish path whose outputs `drec` holds: device time per step, and the
    largest difference of the two outputs (eigenvalues relative to the row's
    largest, normals on rows whose relative eigen-gap is at least 1e-4)."""
    import ctypes
    import torch
    from gpupdal_b200.native import record_columns
    s64 = []
    for o in sts:
        c = type(o)()
        ctypes.memmove(ctypes.addressof(c), ctypes.addressof(o), ctypes.sizeof(o))
        c.eigen_fp64 = 1
        s64.append(c)
    n = drec.shape[0]
    rec64 = torch.empty_like(drec)
    cols64 = record_columns(rec64.data_ptr(), s64, 64, 1)

    def step():
        tile = ctx.tile(*dxyz)
        ex, st = ctx.run_columns(tile, s64, cols64)
        tile.free()
        return st

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        st = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    lam, lam64 = drec[:, 0:3], rec64[:, 0:3]
    lmax = lam.abs().amax(dim=1).clamp_min(1e-300)
    ok = torch.isfinite(lam).all(dim=1) & torch.isfinite(lam64).all(dim=1)
    dl = ((lam - lam64).abs().amax(dim=1) / lmax)[ok]
    gap = ((lam[:, 1] - lam[:, 0]) / lmax) >= 1e-4
    nv, nv64 = drec[:, 3:6], rec64[:, 3:6]
    okn = ok & gap & torch.isfinite(nv).all(dim=1) & torch.isfinite(nv64).all(dim=1)
    dn = (nv - nv64).abs().amax(dim=1)[okn]
    return {"ms_per_step": ms, "value": n / (ms / 1e3) / 1e6, "unit": "Mpts/s",
            "resolved_rows": int(st.resolved_rows),
            "max_rel_diff_eigenvalues": float(dl.max()) if dl.numel() else 0.0,
            "max_abs_diff_normal": float(dn.max()) if dn.numel() else 0.0,
            "rows_compared": int(ok.sum()), "normal_rows_compared": int(okn.sum())}


def target_leg(ctx, dxyz, seed, steps):
    """filters.normal knn=16 + filters.covariancefeatures knn=16 feature_set=all on the main
    tile (one grid, one fused pass for both stages): device inputs, one 128-byte device
    record per point (4 + 11 dims), OptimalKNN / OptimalRadius input columns as in the
    4M-point covariancefeatures configuration."""
    import torch
    from gpupdal_b200 import abi
    from gpupdal_b200 import synthetic as syn
    from gpupdal_b200.native import record_columns
    n = int(dxyz[0].shape[0])
    dev = dxyz[0].device
    sts = [abi.make_opts(abi.STAGE_NORMAL, knn=16),
           abi.make_opts(abi.STAGE_COVARIANCEFEATURES, knn=16, feature_mask=abi.FEAT_ALL)]
    kopt, ropt = syn.optimal_columns(n, seed, knn=16)
    dk, dr = (torch.from_numpy(v).to(dev) for v in (kopt, ropt))
    rec = torch.empty((n, 16), dtype=torch.float64, device=dev)
    cols = record_columns(rec.data_ptr(), sts, 128, 1)

    def step():
        tile = ctx.tile(*dxyz)
        _, st = ctx.run_columns(tile, sts, cols, optimal_knn=dk, optimal_radius=dr,
                                aux_on_device=True)
        tile.free()
        return st

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    stats = [step() for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    q = statistics.mean(s.query_ms for s in stats)
    bpp = 16 + 4 + 8 * 15 + 1
    hbm, _ = peaks()
    return {"workload": f"stress tile {n} points, normal knn=16 + covariancefeatures knn=16 "
                        "feature_set=all, one fused pass",
            "ms_per_step": ms, "value": n / ms / 1e3, "unit": "Mpts/s", "query_ms": q,
            "bytes_per_point": bpp, "query_hbm_frac": n * bpp / (q / 1e3) / 1e9 / hbm}


def extras_cases():
    """The stage options beyond the main path (radius, stride, optimized) and
    the other consumers of the index, each as one stage on the 4M mixture."""
    from gpupdal_b200 import abi
    c = abi.consumer_opts
    return [
        ("normal radius=0.5", abi.make_opts(abi.STAGE_NORMAL, radius=0.5)),
        ("eigenvalues knn=8 stride=2", abi.make_opts(abi.STAGE_EIGENVALUES, knn=8, stride=2)),
        ("covariancefeatures optimized all", abi.make_opts(abi.STAGE_COVARIANCEFEATURES,
                                                           optimized=True, feature_mask=abi.FEAT_ALL)),
        ("approximatecoplanar knn=8", c(abi.STAGE_APPROXIMATECOPLANAR)),
        ("estimaterank knn=8", c(abi.STAGE_ESTIMATERANK)),
        ("nndistance k=10 avg", c(abi.STAGE_NNDISTANCE, mode="avg")),
        ("optimalneighborhood 10..14", c(abi.STAGE_OPTIMALNEIGHBORHOOD)),
        ("lof minpts=10", c(abi.STAGE_LOF)),
        ("outlier statistical mean_k=8", c(abi.STAGE_OUTLIER)),
        ("outlier radius=1 min_k=2", c(abi.STAGE_OUTLIER, method="radius")),
    ]


def cpu_reference_stage(x, y, z, st, kopt, ropt, sample=250_000):
    """The reference's CPU loop of one stage (oracle/_ref, all host threads) on
    a spatially contiguous window of about `sample` points of the tile."""
    from gpupdal_b200 import synthetic as syn
    from oracle import oracle as orc
    kind = "reference" if orc.available("reference") else "port"
    o = orc.Oracle(kind)
    side = int(round(np.sqrt(sample / len(x)) * (x.max() + 1)))
    m = (x < side) & (y < side)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    t = o.tree(*(syn.to_double(v) for v in (x[m], y[m], z[m])))
    t.run_stage(st, mode=0, threads=threads,
                optimal_knn=None if kopt is None else kopt[m],
                optimal_radius=None if ropt is None else ropt[m])
    dt = time.perf_counter() - t0
    return {"value": int(m.sum()) / dt / 1e6, "unit": "Mpts/s", "cores": threads, "kind": kind,
            "sample": f"{int(m.sum())}-point window of the same tile: KD build + the stage"}


def extras_cpu(sample=250_000):
    """The reference's CPU loop of every extra stage on its window of the 4M
    mixture (run in the CPU-only process)."""
    from gpupdal_b200 import synthetic as syn
    x, y, z = syn.mixture(4_000_000, 1)
    kopt, ropt = syn.optimal_columns(len(x), 1, knn=10)
    return {label: cpu_reference_stage(x, y, z, st, kopt, ropt, sample)
            for label, st in extras_cases()}


def extras_leg(ctx, args, cpu=None):
    """The remaining stage options and the other kNN consumers measured: each
    extra stage on the 4M mixture (device inputs, one fresh tile per step),
    beside the reference's CPU loop timed in the CPU-only process (`cpu`),
    and LAS ingest of the same points."""
    import tempfile
    import torch
    from gpupdal_b200 import las
    from gpupdal_b200 import synthetic as syn
    x, y, z = syn.mixture(4_000_000, 1)
    n = len(x)
    kopt, ropt = syn.optimal_columns(n, 1, knn=10)
    dev = torch.device("cuda", ctx.device)
    dx, dy, dz = (torch.from_numpy(v).to(dev) for v in (x, y, z))
    dk, dr = torch.from_numpy(kopt).to(dev), torch.from_numpy(ropt).to(dev)
    out = {"workload": f"mixture tile {n} points (seed 1), one stage per entry, device inputs "
                       "and outputs, a fresh tile every step; cpu: oracle/_ref on a 250k-point "
                       "window, all host threads"}

    def timed_ms(fn, steps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    for label, st in extras_cases():
        def step():
            tile = ctx.tile(dx, dy, dz)
            ctx.run(tile, [st], optimal_knn=dk, optimal_radius=dr, device_out=True)
            tile.free()
        try:
            ms = timed_ms(step)
            e = {"ms": round(ms, 3), "mpts_s": round(n / ms / 1e3, 1)}
            cb = (cpu or {}).get(label)
            if cb:
                e["cpu_mpts_s"] = round(cb["value"], 3)
                e["vs_cpu"] = round(e["mpts_s"] / cb["value"], 1)
        except Exception as exc:  # recorded, not fatal to the main line
            e = {"error": str(exc)}
        out[label] = e
    # LAS ingest: point format 7 records (36 bytes, scale 0.01), host-mapped and
    # device-resident
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tile.las")
        las.write_las(path, x, y, z, version=(1, 4), point_format=7)
        f = las.LasFile(path)
        rec = np.ascontiguousarray(f.records)
        drec = torch.from_numpy(rec.copy()).to(dev)  # the mapped records are read-only
        nbytes = rec.nbytes

        def up_host():
            ctx.tile_from_las(f).free()

        def up_dev():
            ctx.tile_from_las(f, records=drec).free()
        for label, fn in (("las ingest host records", up_host), ("las ingest device records", up_dev)):
            ms = timed_ms(fn)
            out[label] = {"ms": round(ms, 3), "mpts_s": round(n / ms / 1e3, 1),
                          "gb_s": round(nbytes / ms / 1e6, 1), "record_bytes": int(f.record_length)}
    return out


def batched_leg(ctx, args):
    """The batched tile set: plain per-tile launches against one
    nbg_run_batch (graph-captured queue), with fixed and autotuned cells."""
    import torch
    from gpupdal_b200 import batched
    tset = batched.make_set(args.batch_tiles, seed=100)
    pts = sum(t["n"] for t in tset)
    torch.cuda.synchronize()

    def timed(fn, steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = [fn() for _ in range(steps)]
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, out

    steps = max(1, min(args.steps, 3))
    batched.step_plain(ctx, tset)
    plain_ms, _ = timed(lambda: batched.step_plain(ctx, tset), steps)
    batched.step_batched(ctx, tset)
    fixed_ms, st_fixed = timed(lambda: batched.step_batched(ctx, tset), steps)
    batched.step_batched(ctx, tset, autotune=True)  # tunes each size/knn class once
    tuned_ms, st_tuned = timed(lambda: batched.step_batched(ctx, tset, autotune=True), steps)
    return {
        "set": (f"{len(tset)} compact mixture tiles, seeds 100-{99 + len(tset)}, sizes "
                "log-normal (median 200k, sigma 1) in [20k, 4M], knn in {8,16,32}, "
                "normal + covariancefeatures(all), device-resident, one graph-captured launch"),
        "points": int(pts),
        "plain": round(pts / plain_ms / 1e3, 1),
        "batched": round(pts / fixed_ms / 1e3, 1),
        "autotuned": round(pts / tuned_ms / 1e3, 1),
        "batched_vs_plain": round(plain_ms / fixed_ms, 2),
        "query_ms": round(st_fixed[-1].query_ms, 2), "kd_build_ms": round(st_fixed[-1].kd_build_ms, 2),
    }


def served_leg(ctx, args):
    """The served stream (bounded sample): sequential plain per-tile calls
    against the request loop, all requests at once (capacity: the median of
    three passes) and at Poisson arrivals (latency)."""
    from gpupdal_b200 import served
    from gpupdal_b200.native import Server
    reqs = served.make_requests(args.served_requests, seed=1000)
    pts = sum(len(r["x"]) for r in reqs)
    served.run_plain(ctx, reqs)  # warm-up pass: the plain context's block cache
    plain_s = sum(served.run_plain(ctx, reqs))
    srv = Server(0, slots=args.served_slots, hbm_budget=120 * 10**9)
    try:
        # warm-up: requests land on whichever worker is free and waves mix
        # them differently every pass, so early passes still meet buffer sizes
        # a worker's block cache lacks; capacity is the median of three passes
        # after three warm-up passes (all three are reported)
        for _ in range(3):
            served.run_served(srv, reqs)
        caps = sorted(served.run_served(srv, reqs)[0] for _ in range(3))
        cap_s = caps[1]
        rate_s, lat, res = served.run_served(srv, reqs, rate=args.served_rate, seed=1)
        # the same stream with pinned host buffers (outputs allocated once and
        # reused), as a server keeps its I/O staging: copies go by DMA
        preqs, keep = served.pin_requests(reqs)
        served.run_plain(ctx, preqs)
        pplain_s = sum(served.run_plain(ctx, preqs))
        for _ in range(3):
            served.run_served(srv, preqs)
        pcaps = sorted(served.run_served(srv, preqs)[0] for _ in range(3))
        del preqs, keep
    finally:
        srv.close()
    lat_ms = np.sort(np.array(lat) * 1e3)
    return {
        "stream": (f"bounded sample of the 2,000-request stream: requests 0-{len(reqs) - 1} "
                   f"(own tile seeds 1000-{999 + len(reqs)}), sizes log-uniform 10k-8M, knn in "
                   "{8,16,32,64}, normal/eigenvalues/covariancefeatures(all); host buffers; "
                   "120 GB budget"),
        "points": int(pts),
        "plain_mpts_s": round(pts / plain_s / 1e6, 1),
        "served_mpts_s": round(pts / cap_s / 1e6, 1),
        "served_passes_mpts_s": [round(pts / c / 1e6, 1) for c in reversed(caps)],
        "served_vs_plain": round(plain_s / cap_s, 2),
        "rate_req_s": args.served_rate,
        "p50_ms": round(float(np.percentile(lat_ms, 50)), 2),
        "p99_ms": round(float(np.percentile(lat_ms, 99)), 2),
        "rate_mpts_s": round(pts / rate_s / 1e6, 1),
        "pinned": {"plain_mpts_s": round(pts / pplain_s / 1e6, 1),
                   "served_mpts_s": round(pts / pcaps[1] / 1e6, 1),
                   "served_passes_mpts_s": [round(pts / c / 1e6, 1) for c in reversed(pcaps)],
                   "served_vs_plain": round(pplain_s / pcaps[1], 2)},
    }


def served_sweep(ctx, args):
    """The served stream at each rate of --served-sweep: p50/p99 latency from
    submission to results and Mpts/s, beside the plain per-tile calls' Mpts/s
    on the same stream (requests materialised one at a time)."""
    from gpupdal_b200 import served
    from gpupdal_b200.native import Server
    reqs = served.make_stream(args.served_requests, seed=1000, lazy=True)
    pts = reqs.points()
    warm = served.make_stream(24, seed=999)
    served.run_plain(ctx, warm)
    plain_s = sum(served.run_plain(ctx, reqs))
    stream = (f"{len(reqs)} requests, sizes log-uniform 10k-8M of the mixture (subsamples of one "
              "8M cloud, seed 1000), knn in {8,16,32,64}, normal/eigenvalues/"
              "covariancefeatures(all) in equal shares; host buffers in and out; Poisson arrivals")
    srv = Server(0, slots=args.served_slots, hbm_budget=120 * 10**9)
    try:
        for _ in range(2):
            served.run_served(srv, warm)
        for rate in [float(r) for r in args.served_sweep.split(",") if r]:
            # rate 0: every request at once (the server's capacity)
            span_s, lat, _ = served.run_served(srv, reqs, rate=rate or None, seed=int(rate))
            lat_ms = np.sort(np.array(lat) * 1e3)
            print(json.dumps({
                "metric": "served stream latency and throughput", "rate_req_s": rate,
                "requests": len(reqs), "points": pts, "slots": args.served_slots,
                "hbm_budget_gb": 120, "p50_ms": float(np.percentile(lat_ms, 50)),
                "p99_ms": float(np.percentile(lat_ms, 99)), "max_ms": float(lat_ms[-1]),
                "served_mpts_s": pts / span_s / 1e6, "plain_mpts_s": pts / plain_s / 1e6,
                "stream": stream}), flush=True)
    finally:
        srv.close()


def dist_setup():
    """One process per GPU (torchrun env); NCCL on GPUs, gloo without (host-logic tests)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def rank_max(v, ws):
    """Max of a float over the ranks (the timing rule: slowest rank)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, ws, rank):
    if rank != 0:
        return
    x, y, z = workload(args.points, 2)
    for _ in range(args.warmup):
        cpu_reference(x, y, z, args.knn, args.cpu_sample)
    vals = [cpu_reference(x, y, z, args.knn, args.cpu_sample) for _ in range(args.steps)]
    v = statistics.median(r["value"] for r in vals)
    base = dict(vals[-1])
    base["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "Mpts/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(r["seconds"] for r in vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"stress tile {args.points} points (seed 2), eigenvalues "
                                   f"knn={args.knn} then normal knn={args.knn}",
                       "sample": base["sample"]},
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                  "cpu_model", "nproc")},
            "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_only(args):
    """The CPU baselines, timed in a process that has touched no GPU and runs
    nothing else: the main workload's window (all host threads, and one
    thread) and each extra stage's window.  Printed as one JSON object."""
    x, y, z = workload(args.points, 2)
    # warm and repeated as the reference arm's steps are (a single cold run
    # read 16 % below the arm on the same box)
    out = {"main": cpu_reference(x, y, z, args.knn, args.cpu_sample, single_thread=True, reps=3)}
    del x, y, z
    if not args.no_extras:
        out["extras"] = extras_cpu()
    print(json.dumps(out), flush=True)


def run_cpu_child(args):
    """Runs cpu_only() in a fresh interpreter before this process starts any
    GPU work (an in-process timing after the GPU legs read 40 % low: CUDA
    contexts and their host threads share the cores)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-only", "--points", str(args.points),
           "--knn", str(args.knn), "--cpu-sample", str(args.cpu_sample)]
    if args.no_extras:
        cmd.append("--no-extras")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=env)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        return json.loads(lines[-1]) if lines else {"error": r.stderr[-400:]}
    except Exception as exc:  # recorded, not fatal to the main line
        return {"error": str(exc)}


def main():
    args = parse()
    if args.cpu_only:
        cpu_only(args)
        return
    ws, rank, local = dist_setup()
    cpu = None
    if (args.impl == "ours" and rank == 0 and ws == 1 and not args.no_cpu_baseline
            and not args.served_sweep):
        cpu = run_cpu_child(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from gpupdal_b200.native import Context
    from gpupdal_b200 import abi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.served_sweep:
        served_sweep(Context(local), args)
        return
    x, y, z = workload(args.points, 2 + rank)
    n = len(x)
    ctx = Context(local)
    sts = stages(args.knn)
    nd = [len(abi.stage_dims(s)) for s in sts]
    from gpupdal_b200.native import record_columns
    # device-resident inputs; outputs as one 64-byte record per point
    # (Eigenvalue0..2, NormalX/Y/Z, Curvature, unused), sector aligned
    dx, dy, dz = (torch.from_numpy(v).to(dev) for v in (x, y, z))
    drec = torch.empty((n, 8), dtype=torch.float64, device=dev)
    dcols = record_columns(drec.data_ptr(), sts, 64, 1)
    # pinned host inputs and packed 56-byte host records for the end-to-end form
    hx, hy, hz = (torch.from_numpy(v).pin_memory() for v in (x, y, z))
    hrec = torch.empty((n, 7), dtype=torch.float64).pin_memory()
    hcols = record_columns(hrec.data_ptr(), sts, 56, 2)
    hxn, hyn, hzn = hx.numpy(), hy.numpy(), hz.numpy()

    fixed = args.select is not None or args.cell_factor is not None

    def configure(tile):
        if args.cell_factor is not None:
            tile.tune(args.cell_factor)
        if args.select is not None:
            tile.set_select(args.select)
        return tile

    def step_device():
        tile = configure(ctx.tile(dx, dy, dz))
        ex, st = ctx.run_columns(tile, sts, dcols)
        tile.free()
        return st

    def step_e2e():
        tile = configure(ctx.tile(hxn, hyn, hzn))
        ex, st = ctx.run_columns(tile, sts, hcols)
        tile.free()
        return st

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(v):
        return rank_max(v, ws)

    def timed(fn, steps):
        stats = []
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            stats.append(fn())
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1), stats

    # the context's autotuner measures this tile's size / knn class once (cell
    # factor and select kernel); every fresh tile of the steps below then takes
    # the cached choice in nbg_run, as tiles of a loaded tuning file do
    if fixed:
        tuning = [{"cell_factor": args.cell_factor if args.cell_factor is not None else 4.0,
                   "select_kernel": args.select if args.select is not None else 0}]
    else:
        tune_tile = ctx.tile(dx, dy, dz)
        tune_tile.autotune(args.knn)
        tune_tile.free()
        tuning = ctx.tuning_cache()
    for _ in range(max(args.warmup, 3)):
        step_device()
    clocks = ClockSampler(local)
    clocks.start()
    ms, stats = timed(step_device, args.steps)
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    per_step = ms / args.steps
    value = ws * n / (per_step / 1e3) / 1e6
    query_ms = statistics.mean(s.query_ms for s in stats)
    launches = int(sum(s.kernel_launches for s in stats))
    hbm, peak_kind = peaks()
    achieved = n * BYTES_PER_POINT / (query_ms / 1e3) / 1e9
    sel_kernel = tuning[0]["select_kernel"] if len(tuning) == 1 else 0
    qp = QUERY_PROFILES.get(sel_kernel, QUERY_PROFILES[0])
    # end to end through the C ABI with host buffers
    for _ in range(2):
        step_e2e()
    ms_e2e, stats_e2e = timed(step_e2e, args.steps)
    ms_e2e = max_over_ranks(ms_e2e)
    e2e_value = ws * n / (ms_e2e / args.steps / 1e3) / 1e6
    last = stats[-1]
    fp64 = None
    if ws == 1 and not args.no_fp64:
        step_device()  # drec: the FP32 + FP64-polish outputs
        fp64 = fp64_leg(ctx, args, (dx, dy, dz), drec, sts, args.steps)
        fp64["speedup_of_default"] = fp64["ms_per_step"] / per_step
    line = {
        "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+i64+f64", "data": "synthetic",
        "config": {"workload": f"stress tile {n} points per GPU (seed 2+rank), filters.eigenvalues "
                               f"knn={args.knn} then filters.normal knn={args.knn}, one grid",
                   "points_per_gpu": n, "knn": args.knn, "form": "plain per-tile launch",
                   "tuning": {"source": ("fixed by --select / --cell-factor" if fixed else
                                         "context autotuner, one measurement of this size/knn "
                                         "class before the warm-up, applied by nbg_run to each "
                                         "fresh tile"), "entries": tuning},
                   "l2": "inputs larger than L2 (tile 384 MB + sorted copy 512 MB per step)",
                   "tie_rows": int(last.tie_rows), "deferred_rows": int(last.deferred_rows),
                   "resolved_rows": int(last.resolved_rows), "replay_rows": int(last.replay_rows),
                   "grid_ms": last.grid_ms, "query_ms": last.query_ms, "tree_ms": last.tree_ms},
        "e2e": {"value": e2e_value, "unit": "Mpts/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 8 * sum(nd) * n, "ms_per_step": ms_e2e / args.steps,
                "output_chunks": int(stats_e2e[-1].output_chunks),
                "run_device_ms": statistics.mean(s.total_ms for s in stats_e2e),
                "run_query_ms": statistics.mean(s.query_ms for s in stats_e2e),
                "form": "tile upload from pinned host arrays + nbg_run writing one pinned "
                        "56-byte host record per point (copied back chunk by chunk while "
                        "later chunks run when output_chunks > 0)"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": qp["traffic"] * n,
                     "traffic_source": "ncu dram bytes of the query kernels on the 4M-point "
                                       "tile, scaled per point",
                     "kernel": qp["kernel"], "peak_source": peak_kind,
                     "bytes_per_point": BYTES_PER_POINT,
                     "issue_efficiency": round(qp["lanes"] / 32 * qp["issue"], 3),
                     "limiter": (f"instruction issue, not HBM: ncu on the 4M-point stress tile shows "
                                 f"the select kernel with {100 * qp['issue']:.1f} % of issue slots "
                                 f"busy, {qp['lanes']:.2f} of 32 lanes active per instruction "
                                 f"(issue efficiency = lanes/32 x issue fraction) and "
                                 f"{qp['dram_pct']:.2f} % DRAM throughput")},
        "clocks": clk,
    }
    if cpu is not None:
        cb = cpu.get("main")
        if cb:
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                       "cpu_model", "nproc", "single_thread")}
            line["cpu_baseline"]["process"] = ("fresh process, before any GPU work; one untimed "
                                               "run, then the median of three")
        else:
            line["cpu_baseline"] = {"error": cpu.get("error", "no result")}
    # the large legs first, the compact summaries last (the end of the line
    # is what a log tail keeps)
    if ws == 1 and not args.no_extras:
        line["extras"] = extras_leg(ctx, args, (cpu or {}).get("extras"))
    if fp64 is not None:
        line["eigen_fp64"] = fp64
    if ws == 1 and not args.no_extras:
        try:
            line["normal_plus_features"] = target_leg(ctx, (dx, dy, dz), 2 + rank, args.steps)
        except Exception as exc:  # recorded, not fatal to the main line
            line["normal_plus_features"] = {"error": str(exc)}
    if ws == 1 and not args.no_batched:
        line["batched"] = batched_leg(ctx, args)
    if ws == 1 and not args.no_served:
        line["served"] = served_leg(ctx, args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

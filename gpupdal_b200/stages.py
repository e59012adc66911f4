"""PDAL stage layer over the C ABI (nbg_filter_*, nbg_pipeline_*): run the
path's stages of an existing pipeline JSON on one tile.

    from gpupdal_b200.stages import run_pipeline
    dims, log = run_pipeline(ctx, pipeline_json, x, y, z)

`dims` maps each registered dimension name (NormalX, Eigenvalue0, Linearity,
Coplanar, NNDistance, OptimalKNN, ...) to a float64 array in point order;
rows a stage skips hold 0, as in a freshly added PDAL dimension.  `log` holds the lines the stages logged.  A
check or row the reference throws on raises StageError with its message.
Stages outside this path (readers, writers, other filters) are not run;
their types are returned in `log` as "not run: <type>"."""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import abi

PATH_STAGES = ("filters.normal", "filters.eigenvalues", "filters.covariancefeatures",
               "filters.approximatecoplanar", "filters.estimaterank", "filters.nndistance",
               "filters.optimalneighborhood", "filters.lof", "filters.outlier")


class StageError(RuntimeError):
    pass


class Filter:
    def __init__(self, stage_type, options=None, has_optimal_knn=False, has_optimal_radius=False):
        self.lib = abi.load_library()
        text = options if isinstance(options, str) else json.dumps(options or {})
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        rc = self.lib.nbg_filter_create(stage_type.encode(), text.encode(), int(has_optimal_knn),
                                        int(has_optimal_radius), ctypes.byref(h), err, len(err))
        if rc != abi.NBG_OK:
            raise StageError(err.value.decode())
        self.h = h
        self.type = stage_type

    def options(self):
        o = abi.StageOpts()
        rc = self.lib.nbg_filter_options(self.h, ctypes.byref(o))
        return o, rc

    def dims(self):
        buf = ctypes.create_string_buffer(512)
        self.lib.nbg_filter_dims(self.h, buf, len(buf))
        return [d for d in buf.value.decode().split(",") if d]

    def log(self):
        return [l for l in self.lib.nbg_filter_log(self.h).decode().split("\n") if l]

    def report(self, exceptions, stage_index=0):
        n = len(exceptions)
        arr = (abi.RowException * max(n, 1))()
        from .native import EXC_DTYPE
        if n and exceptions.dtype == np.dtype(EXC_DTYPE):
            ctypes.memmove(arr, np.ascontiguousarray(exceptions).ctypes.data, n * ctypes.sizeof(abi.RowException))
        else:
            for i, e in enumerate(exceptions):
                arr[i].point_id, arr[i].stage, arr[i].code = (int(e["point_id"]), int(e["stage"]),
                                                              int(e["code"]))
                if "reserved" in e.dtype.names:
                    arr[i].reserved = int(e["reserved"])
        err = ctypes.create_string_buffer(1024)
        rc = self.lib.nbg_filter_report(self.h, arr, n, int(stage_index), err, len(err))
        if rc != abi.NBG_OK:
            raise StageError(err.value.decode())

    def outcome(self, stats):
        """filters.outlier's warnings for a run's counts (appended to the log)."""
        self.lib.nbg_filter_outcome(self.h, ctypes.byref(stats))

    def close(self):
        if getattr(self, "h", None):
            self.lib.nbg_filter_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_pipeline(text):
    """[(type, options dict)] of a pipeline JSON."""
    lib = abi.load_library()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(1024)
    rc = lib.nbg_pipeline_parse(text.encode(), ctypes.byref(h), err, len(err))
    if rc != abi.NBG_OK:
        raise StageError(err.value.decode())
    try:
        out = []
        for i in range(lib.nbg_pipeline_size(h)):
            out.append((lib.nbg_pipeline_type(h, i).decode(),
                        json.loads(lib.nbg_pipeline_options(h, i).decode())))
        return out
    finally:
        lib.nbg_pipeline_free(h)


def run_pipeline(ctx, pipeline, x, y, z, scale=(0.01, 0.01, 0.01), offset=(0.0, 0.0, 0.0),
                 optimal_knn=None, optimal_radius=None):
    stages = parse_pipeline(pipeline if isinstance(pipeline, str) else json.dumps(pipeline))
    tile = ctx.tile(x, y, z, scale=scale, offset=offset)
    dims, log = {}, []
    try:
        for stype, opts in stages:
            if stype not in PATH_STAGES:
                log.append(f"not run: {stype}")
                continue
            f = Filter(stype, opts, optimal_knn is not None, optimal_radius is not None)
            o, rc = f.options()
            if rc != abi.NBG_OK:
                raise StageError(f"{stype}: stride * (knn + 1) above 65 is not supported "
                                 "by this library")
            outs, ex, stats = ctx.run(tile, [o], optimal_knn=optimal_knn,
                                      optimal_radius=optimal_radius)
            f.report(ex, 0)
            f.outcome(stats)
            for name, col in zip(f.dims(), outs[0]):
                dims[name] = col
            # filters.optimalneighborhood's dimensions feed later stages
            # (covariancefeatures optimized / Density)
            if "OptimalKNN" in dims:
                optimal_knn = np.ascontiguousarray(dims["OptimalKNN"])
                optimal_radius = np.ascontiguousarray(dims["OptimalRadius"])
            log += [f"({stype}) {l}" for l in f.log()]
            f.close()
    finally:
        tile.free()
    return dims, log

"""Python handle on the native library (C ABI in include/nbg_b200.h).

Host buffers are numpy arrays; device buffers are torch CUDA tensors (torch is
used only for device memory and streams).  Every call goes to the sm_100a
library; a missing library raises instead of falling back to the CPU.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import abi


class NbgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"nbg error {code}: {msg}")
        self.code = code


def _dptr(a):
    return ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())


# row exceptions as returned: the point, the stage index, the NBG_ROW_* code and
# the code's detail (the neighbour count of NBG_ROW_RADIUS_FEW rows)
EXC_DTYPE = [("point_id", np.uint32), ("stage", np.uint8), ("code", np.uint8), ("reserved", np.uint16)]


def exceptions_array(buf, count):
    """The first `count` nbg_row_exception records of a ctypes array as a
    structured numpy array (the record is EXC_DTYPE byte for byte)."""
    if count == 0:
        return np.zeros(0, dtype=EXC_DTYPE)
    return np.frombuffer(buf, dtype=np.dtype(EXC_DTYPE), count=count).copy()


def record_columns(base_ptr, stages, record_bytes, on_device):
    """abi.Columns for `stages` sharing one record per point: the stages'
    dims are laid out one after another from offset 0."""
    cols, off = [], 0
    for st in stages:
        c = abi.Columns()
        c.base = base_ptr
        c.point_stride = record_bytes
        dims = abi.stage_dims(st)
        c.ndims = len(dims)
        c.on_device = on_device
        for d in range(len(dims)):
            c.offset[d] = off
            off += 8
        cols.append(c)
    if off > record_bytes:
        raise ValueError("record too small for the stages' dims")
    return cols


class Context:
    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = abi.load_library()
        h = ctypes.c_void_p()
        rc = self.lib.nbg_create(ctypes.byref(h), int(device), int(hbm_budget))
        if rc != abi.NBG_OK:
            raise NbgError(rc, "nbg_create failed (no sm_100 device?)")
        self.h = h
        self.device = device
        self._tls = threading.local()

    def _exceptions(self, cap):
        """This thread's row-exception buffer of `cap` records (a context may
        be shared by threads; each reads its own call's exceptions)."""
        buf = getattr(self._tls, "exc", None)
        if buf is None or len(buf) != cap:
            buf = (abi.RowException * cap)()
            self._tls.exc = buf
        return buf

    def tuning_cache(self):
        """The autotuner's cached choices: a list of {"size_class", "slots",
        "cell_factor", "select_kernel"} (nbg_autotune_cache_get)."""
        count = ctypes.c_int32(0)
        self._check(self.lib.nbg_autotune_cache_get(self.h, None, 0, ctypes.byref(count)))
        buf = (abi.TuneEntry * max(count.value, 1))()
        self._check(self.lib.nbg_autotune_cache_get(self.h, buf, count.value, ctypes.byref(count)))
        return [{"size_class": int(e.size_class), "slots": int(e.slots),
                 "cell_factor": float(e.cell_factor),
                 "select_kernel": int(e.select_kernel)} for e in buf[:count.value]]

    def set_tuning_cache(self, entries):
        """Adds or replaces autotuner choices (nbg_autotune_cache_set)."""
        buf = (abi.TuneEntry * max(len(entries), 1))()
        for e, d in zip(buf, entries):
            e.size_class = int(d["size_class"])
            e.slots = int(d["slots"])
            e.cell_factor = float(d["cell_factor"])
            e.select_kernel = int(d.get("select_kernel", 0))
        self._check(self.lib.nbg_autotune_cache_set(self.h, buf, len(entries)))

    def save_tuning(self, path):
        """Writes the autotuner's choices to a JSON tuning file, keyed by the
        device's name (a file tuned on one GPU model is not applied to another)."""
        import json
        with open(path, "w") as f:
            json.dump({"device": self.device_name(), "entries": self.tuning_cache()}, f, indent=1)

    def load_tuning(self, path):
        """Applies a tuning file written by save_tuning on the same GPU model;
        returns the number of entries applied (0 for another model)."""
        import json
        with open(path) as f:
            d = json.load(f)
        if d.get("device") != self.device_name():
            return 0
        self.set_tuning_cache(d["entries"])
        return len(d["entries"])

    def device_name(self):
        import torch
        return torch.cuda.get_device_name(self.device)

    def close(self):
        if getattr(self, "h", None):
            self.lib.nbg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != abi.NBG_OK:
            raise NbgError(rc, self.lib.nbg_last_error(self.h).decode())

    def tile(self, x, y, z, scale=(0.01, 0.01, 0.01), offset=(0.0, 0.0, 0.0), stream=None):
        return Tile(self, x, y, z, scale, offset, stream)

    def tile_from_las(self, src, records=None, stream=None):
        """A tile straight from LAS point records (nbg_tile_upload_las).

        `src` is a path or a las.LasFile; its records are copied from the
        mapped file and decoded on the device.  `records` overrides them with
        the same records already on the device (a uint8 torch tensor of
        point_count x point_record_length bytes)."""
        from . import las
        f = src if isinstance(src, las.LasFile) else las.LasFile(src)
        rec = f.records if records is None else records
        if records is not None and int(records.numel()) != f.n * f.record_length:
            raise ValueError("device records do not match the file's record extent")
        sc = (ctypes.c_double * 3)(*f.scale)
        of = (ctypes.c_double * 3)(*f.offset)
        h = ctypes.c_void_p()
        rc = self.lib.nbg_tile_upload_las(self.h, _dptr(rec), f.n, f.record_length,
                                          int(records is not None), sc, of,
                                          ctypes.c_void_p(stream) if stream else None,
                                          ctypes.byref(h))
        self._check(rc)
        return Tile._adopt(self, h, f.n, (f, rec))

    # -- stages -----------------------------------------------------------
    def run(self, tile, stages, optimal_knn=None, optimal_radius=None, device_out=False,
            fresh=True, exception_capacity=None, stream=None, out=None):
        """Runs `stages` (list of abi.StageOpts) over `tile`.

        Returns (outputs, exceptions, stats): outputs[i] is a (ndims, n)
        array (numpy, or a torch tensor when device_out) for stage i;
        exceptions is a structured numpy array (point_id, stage, code)."""
        n = tile.n
        ns = len(stages)
        opts = (abi.StageOpts * max(ns, 1))(*stages)
        cols = (abi.Columns * max(ns, 1))()
        outs = []
        for i, st in enumerate(stages):
            nd = len(abi.stage_dims(st))
            if out is not None:
                buf = out[i]
            elif device_out:
                import torch
                buf = torch.zeros((max(nd, 1), n), dtype=torch.float64, device=f"cuda:{self.device}")
            else:
                buf = np.zeros((max(nd, 1), n), dtype=np.float64)
            outs.append(buf)
            c = cols[i]
            c.base = _dptr(buf).value
            c.point_stride = 8
            c.ndims = nd
            c.on_device = 1 if device_out else (2 if fresh else 0)
            for d in range(nd):
                c.offset[d] = d * n * 8
        cap = exception_capacity if exception_capacity is not None else max(1024, n)
        exc = self._exceptions(cap)
        nexc = ctypes.c_uint32(0)
        stats = abi.RunStats()
        kp = rp = None
        aux_dev = 0
        if optimal_knn is not None:
            if isinstance(optimal_knn, np.ndarray):
                optimal_knn = np.ascontiguousarray(optimal_knn, dtype=np.float64)
                optimal_radius = np.ascontiguousarray(optimal_radius, dtype=np.float64)
            else:
                aux_dev = 1
            kp, rp = _dptr(optimal_knn), _dptr(optimal_radius)
        rc = self.lib.nbg_run(self.h, tile.h, opts, ns, cols, kp, rp, aux_dev, exc, cap,
                              ctypes.byref(nexc), ctypes.byref(stats),
                              ctypes.c_void_p(stream) if stream else None)
        self._check(rc)
        m = min(nexc.value, cap)
        ex = exceptions_array(exc, m)
        return [o[: len(abi.stage_dims(s))] for o, s in zip(outs, stages)], ex, stats

    def run_columns(self, tile, stages, columns, optimal_knn=None, optimal_radius=None,
                    aux_on_device=False, exception_capacity=1 << 16, stream=None):
        """nbg_run with caller-built abi.Columns (e.g. one record per point
        shared by several stages).  Returns (exceptions, stats)."""
        ns = len(stages)
        opts = (abi.StageOpts * max(ns, 1))(*stages)
        cols = (abi.Columns * max(ns, 1))(*columns)
        cap = exception_capacity
        exc = self._exceptions(cap)
        nexc = ctypes.c_uint32(0)
        stats = abi.RunStats()
        kp = None if optimal_knn is None else _dptr(optimal_knn)
        rp = None if optimal_radius is None else _dptr(optimal_radius)
        rc = self.lib.nbg_run(self.h, tile.h, opts, ns, cols, kp, rp, int(aux_on_device), exc,
                              cap, ctypes.byref(nexc), ctypes.byref(stats),
                              ctypes.c_void_p(stream) if stream else None)
        self._check(rc)
        m = min(nexc.value, cap)
        ex = exceptions_array(exc, m)
        return ex, stats

    def run_batch(self, tiles, stages, outputs, optimal=None, graph=True, autotune=False,
                  exception_capacity=1 << 16, stream=None):
        """nbg_run_batch over `tiles` (list of Tile); stages[i] is the stage
        list of tile i, outputs[i] its device abi.Columns list, optimal[i]
        an (OptimalKNN, OptimalRadius) pair of device tensors or None.
        Returns (exceptions per tile, stats)."""
        m = len(tiles)
        arr = (abi.BatchItem * max(m, 1))()
        keep = []
        nex = (ctypes.c_uint32 * max(m, 1))()
        excs = []
        for i, t in enumerate(tiles):
            opts = (abi.StageOpts * len(stages[i]))(*stages[i])
            cols = (abi.Columns * len(stages[i]))(*outputs[i])
            exc = (abi.RowException * exception_capacity)()
            keep += [opts, cols]
            excs.append(exc)
            it = arr[i]
            it.tile = t.h.value
            it.n_stages = len(stages[i])
            it.exception_capacity = exception_capacity
            it.stages = opts
            it.outputs = cols
            if optimal is not None and optimal[i] is not None:
                it.optimal_knn = _dptr(optimal[i][0]).value
                it.optimal_radius = _dptr(optimal[i][1]).value
            it.exceptions = ctypes.addressof(exc)
            it.n_exceptions = ctypes.cast(ctypes.addressof(nex) + 4 * i,
                                          ctypes.POINTER(ctypes.c_uint32))
        stats = abi.RunStats()
        flags = (abi.BATCH_GRAPH if graph else 0) | (abi.BATCH_AUTOTUNE if autotune else 0)
        rc = self.lib.nbg_run_batch(self.h, arr, m, flags,
                                    ctypes.byref(stats), ctypes.c_void_p(stream) if stream else None)
        self._check(rc)
        out = []
        for i in range(m):
            k = min(nex[i], exception_capacity)
            ex = exceptions_array(excs[i], k)
            out.append(ex)
        return out, stats

    def kd_export(self, tile):
        """The device KD replica: (vind, nodes dict) for parity tests."""
        n = tile.n
        cap = max(16, n // 10 + 64)
        vind = np.zeros(n, np.uint32)
        nn = ctypes.c_uint32(0)
        arr = dict(child1=np.zeros(cap, np.int32), child2=np.zeros(cap, np.int32),
                   divfeat=np.zeros(cap, np.int32), divlow=np.zeros(cap), divhigh=np.zeros(cap),
                   begin=np.zeros(cap, np.uint32), end=np.zeros(cap, np.uint32))
        rc = self.lib.nbg_debug_kd_export(
            self.h, tile.h, _dptr(vind), ctypes.byref(nn), *[_dptr(arr[k]) for k in
                                                            ("child1", "child2", "divfeat",
                                                             "divlow", "divhigh", "begin", "end")],
            cap)
        self._check(rc)
        m = min(nn.value, cap)
        return vind, {k: v[:m] for k, v in arr.items()}

    def neighbor_sets(self, tile, knn):
        k1 = min(tile.n, knn + 1)
        ids = np.zeros((tile.n, k1), dtype=np.uint32)
        stats = abi.RunStats()
        rc = self.lib.nbg_neighbor_sets(self.h, tile.h, int(knn), _dptr(ids), 0,
                                        ctypes.byref(stats), None)
        self._check(rc)
        return ids, stats


class Tile:
    def __init__(self, ctx: Context, x, y, z, scale, offset, stream=None):
        self.ctx = ctx
        on_device = not isinstance(x, np.ndarray)
        if not on_device:
            x = np.ascontiguousarray(x, dtype=np.int32)
            y = np.ascontiguousarray(y, dtype=np.int32)
            z = np.ascontiguousarray(z, dtype=np.int32)
        self._keep = (x, y, z)
        self.n = int(len(x))
        sc = (ctypes.c_double * 3)(*scale)
        of = (ctypes.c_double * 3)(*offset)
        h = ctypes.c_void_p()
        rc = ctx.lib.nbg_tile_upload(ctx.h, _dptr(x), _dptr(y), _dptr(z), self.n, sc, of,
                                     int(on_device), ctypes.c_void_p(stream) if stream else None,
                                     ctypes.byref(h))
        ctx._check(rc)
        self.h = h

    @classmethod
    def _adopt(cls, ctx, h, n, keep):
        t = cls.__new__(cls)
        t.ctx, t.h, t.n, t._keep = ctx, h, int(n), keep
        return t

    def tune(self, cell_factor=4.0, fixed_cell=0):
        self.ctx._check(self.ctx.lib.nbg_tile_tune(self.ctx.h, self.h, float(cell_factor),
                                                   int(fixed_cell)))

    def set_select(self, kernel=0, first_margin=0.5):
        """Select kernel (nbg_tile_set_select): 0 two-pass ring search
        (default), 1 the same in block-local Morton order, 2 single-pass ring
        search, 8 / 16 / 32 queries sharing one candidate list; results are
        identical."""
        self.ctx._check(self.ctx.lib.nbg_tile_set_select(self.ctx.h, self.h, int(kernel),
                                                         float(first_margin)))

    def autotune(self, knn, candidates=None, use_cache=False):
        """Cell factor chosen by the library's autotuner (applied to the tile)."""
        cand = None
        cnt = 0
        if candidates is not None:
            cand = (ctypes.c_float * len(candidates))(*candidates)
            cnt = len(candidates)
        out = ctypes.c_float(0)
        self.ctx._check(self.ctx.lib.nbg_tile_autotune(self.ctx.h, self.h, int(knn), cand, cnt,
                                                       int(use_cache), ctypes.byref(out), None))
        return out.value

    def free(self):
        if getattr(self, "h", None) and self.ctx.h:
            self.ctx.lib.nbg_tile_free(self.ctx.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """The served form (nbg_server_*): requests are queued FIFO and admitted
    onto `slots` workers while the HBM budget holds their footprint; admitted
    requests overlap on the device.

    submit() takes one tile's raw coordinates and its stages and returns a
    ticket; wait() returns (outputs, exceptions, result) once it finished."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: int = 0):
        self.lib = abi.load_library()
        h = ctypes.c_void_p()
        rc = self.lib.nbg_server_create(ctypes.byref(h), int(device), int(slots), int(hbm_budget))
        if rc != abi.NBG_OK:
            raise NbgError(rc, "nbg_server_create failed")
        self.h = h
        self.device = device
        self._pending = {}

    def submit(self, x, y, z, stages, scale=(0.01, 0.01, 0.01), offset=(0.0, 0.0, 0.0),
               optimal_knn=None, optimal_radius=None, out=None, device_out=False,
               exception_capacity=None, tag=0):
        on_device = not isinstance(x, np.ndarray)
        if not on_device:
            x, y, z = (np.ascontiguousarray(v, dtype=np.int32) for v in (x, y, z))
        n = int(len(x))
        ns = len(stages)
        opts = (abi.StageOpts * ns)(*stages)
        cols = (abi.Columns * ns)()
        outs = []
        for i, st in enumerate(stages):
            nd = len(abi.stage_dims(st))
            if out is not None:
                buf = out[i]
            elif device_out:
                import torch
                buf = torch.zeros((max(nd, 1), n), dtype=torch.float64, device=f"cuda:{self.device}")
            else:
                buf = np.zeros((max(nd, 1), n), dtype=np.float64)
            outs.append(buf)
            c = cols[i]
            c.base = _dptr(buf).value
            c.point_stride = 8
            c.ndims = nd
            c.on_device = 1 if device_out else 2
            for d in range(nd):
                c.offset[d] = d * n * 8
        cap = exception_capacity if exception_capacity is not None else max(1024, n)
        exc = (abi.RowException * cap)()
        aux = []
        if optimal_knn is not None:
            aux = [np.ascontiguousarray(optimal_knn, dtype=np.float64),
                   np.ascontiguousarray(optimal_radius, dtype=np.float64)]
        r = abi.Request()
        r.x, r.y, r.z = _dptr(x).value, _dptr(y).value, _dptr(z).value
        r.n = n
        for k in range(3):
            r.scale[k] = scale[k]
            r.offset[k] = offset[k]
        r.on_device = int(on_device)
        r.n_stages = ns
        r.stages = opts
        r.outputs = cols
        r.optimal_knn = aux[0].ctypes.data if aux else None
        r.optimal_radius = aux[1].ctypes.data if aux else None
        r.aux_on_device = 0
        r.exception_capacity = cap
        r.exceptions = ctypes.addressof(exc)
        r.user_tag = int(tag)
        t = ctypes.c_uint64(0)
        rc = self.lib.nbg_server_submit(self.h, ctypes.byref(r), ctypes.byref(t))
        if rc != abi.NBG_OK:
            raise NbgError(rc, self.lib.nbg_server_last_error(self.h).decode())
        # everything the worker reads stays referenced until wait()
        self._pending[t.value] = (x, y, z, opts, cols, outs, exc, aux, stages, r)
        return t.value

    def request_bytes(self, n, stages):
        r = abi.Request()
        r.n = int(n)
        r.n_stages = len(stages)
        cols = (abi.Columns * len(stages))()
        for i, st in enumerate(stages):
            cols[i].ndims = len(abi.stage_dims(st))
        opts = (abi.StageOpts * len(stages))(*stages)
        r.outputs = cols
        r.stages = opts
        return int(self.lib.nbg_request_bytes(ctypes.byref(r)))

    def wait(self, ticket, timeout_ms=-1):
        res = abi.RequestResult()
        rc = self.lib.nbg_server_wait(self.h, int(ticket), int(timeout_ms), ctypes.byref(res))
        if rc != abi.NBG_OK:
            raise NbgError(rc, "nbg_server_wait")
        x, y, z, opts, cols, outs, exc, aux, stages, r = self._pending.pop(ticket)
        if res.status != abi.NBG_OK:
            raise NbgError(res.status, self.lib.nbg_server_last_error(self.h).decode())
        m = min(res.n_exceptions, len(exc))
        ex = exceptions_array(exc, m)
        return [o[: len(abi.stage_dims(s))] for o, s in zip(outs, stages)], ex, res

    def close(self):
        if getattr(self, "h", None):
            self.lib.nbg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

ctypes wrapper over the CPU oracle: ``port`` (oracle/_build/libnbg_oracle.so,
the restatement in nbg_oracle.cpp) or ``reference`` (oracle/_ref/libnbg_ref.so,
the same entry points over the reference's own nanoflann and Eigen).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "_build", "libnbg_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libnbg_ref.so")


def build(ref_root: str | None = None) -> None:
    """Compile the port (always) and the reference shim when a reference tree
    is given (`ref_root`, else the NBG_REFERENCE environment variable)."""
    ref_root = ref_root or os.environ.get("NBG_REFERENCE", "")
    subprocess.check_call(["make", "-s", "-C", HERE, "all", f"REF={ref_root}"])


def available(kind: str = "port") -> bool:
    return os.path.exists(PORT_PATH if kind == "port" else REF_PATH)


class Oracle:
    def __init__(self, kind: str = "port"):
        path = PORT_PATH if kind == "port" else REF_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind = kind
        lib = ctypes.CDLL(path)
        vp, u64 = ctypes.c_void_p, ctypes.c_uint64
        dp = ctypes.POINTER(ctypes.c_double)
        lib.orc_impl_name.restype = ctypes.c_char_p
        lib.orc_tree_build.argtypes = [dp, dp, dp, u64]
        lib.orc_tree_build.restype = vp
        lib.orc_tree_build_t.argtypes = [dp, dp, dp, u64, ctypes.c_int]
        lib.orc_tree_build_t.restype = vp
        lib.orc_tree_free.argtypes = [vp]
        lib.orc_tree_neighbors.argtypes = [vp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, u64, u64,
                                           ctypes.POINTER(ctypes.c_uint64)]
        lib.orc_tree_neighbors.restype = u64
        lib.orc_all_neighbors.argtypes = [vp, u64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
        lib.orc_tree_num_nodes.argtypes = [vp]
        lib.orc_tree_num_nodes.restype = u64
        lib.orc_tree_export.argtypes = [vp] + [ctypes.c_void_p] * 8
        lib.orc_eigen_chain.argtypes = [dp, dp, dp]
        lib.orc_eigen_chain.restype = ctypes.c_int
        lib.orc_run_stage.argtypes = [vp, ctypes.c_void_p, dp, dp, ctypes.c_int,
                                      ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_uint8),
                                      ctypes.c_int]
        lib.orc_run_stage.restype = ctypes.c_int
        self.lib = lib

    def tree(self, x, y, z, build_threads=0) -> "Tree":
        """build_threads 0 leaves the KD build its own thread count."""
        return Tree(self, x, y, z, build_threads)

    def eigen_chain(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
        ev = np.zeros(3)
        vec = np.zeros(9)
        dp = ctypes.POINTER(ctypes.c_double)
        ok = self.lib.orc_eigen_chain(a.ctypes.data_as(dp), ev.ctypes.data_as(dp),
                                      vec.ctypes.data_as(dp))
        return ok, ev, vec.reshape(3, 3).T  # columns are eigenvectors


class Tree:
    """A KD3-style index over double coordinates (x, y, z in metres)."""

    def __init__(self, orc: Oracle, x, y, z, build_threads=0):
        self.orc = orc
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.z = np.ascontiguousarray(z, dtype=np.float64)
        self.n = len(self.x)
        dp = ctypes.POINTER(ctypes.c_double)
        self.h = orc.lib.orc_tree_build_t(self.x.ctypes.data_as(dp), self.y.ctypes.data_as(dp),
                                          self.z.ctypes.data_as(dp), self.n, int(build_threads))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.orc.lib.orc_tree_free(h)
            self.h = None

    def neighbors(self, q, k, stride=1):
        out = np.zeros(max(1, k * stride), dtype=np.uint64)
        cnt = self.orc.lib.orc_tree_neighbors(
            self.h, float(q[0]), float(q[1]), float(q[2]), int(k), int(stride),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return out[:cnt].copy()

    def all_neighbors(self, k, threads=None):
        k1 = min(self.n, k)
        out = np.zeros((self.n, k1), dtype=np.uint64)
        self.orc.lib.orc_all_neighbors(self.h, int(k), out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_uint64)), int(threads or os.cpu_count() or 1))
        return out

    def export(self):
        """Preorder node arrays of the port's tree (vind for both kinds)."""
        nn = self.orc.lib.orc_tree_num_nodes(self.h)
        vind = np.zeros(self.n, dtype=np.uint64)
        c1 = np.zeros(nn, np.int64)
        c2 = np.zeros(nn, np.int64)
        feat = np.zeros(nn, np.int32)
        lo = np.zeros(nn)
        hi = np.zeros(nn)
        le = np.zeros(nn, np.uint64)
        ri = np.zeros(nn, np.uint64)
        self.orc.lib.orc_tree_export(self.h, *[a.ctypes.data for a in
                                               (vind, c1, c2, feat, lo, hi, le, ri)])
        return dict(vind=vind, child1=c1, child2=c2, divfeat=feat, divlow=lo, divhigh=hi,
                    left=le, right=ri)

    def run_stage(self, opts, mode=0, optimal_knn=None, optimal_radius=None, threads=None,
                  ndims=None):
        """Per-point loop of one stage; returns (outputs[ndims, n], status[n]).

        Rows the reference skips keep NaN in `outputs`; an outlier stage's
        Classification starts at 0 (a fresh dimension) and the number of
        outliers found is left in `self.outliers`."""
        from gpupdal_b200.abi import STAGE_OUTLIER, stage_dims
        nd = ndims if ndims is not None else len(stage_dims(opts))
        outs = np.full((max(nd, 1), self.n), 0.0 if opts.kind == STAGE_OUTLIER else np.nan)
        status = np.zeros(self.n, dtype=np.uint8)
        dp = ctypes.POINTER(ctypes.c_double)
        cols = (dp * max(nd, 1))(*[outs[i].ctypes.data_as(dp) for i in range(max(nd, 1))])
        kopt = None if optimal_knn is None else np.ascontiguousarray(optimal_knn, np.float64)
        ropt = None if optimal_radius is None else np.ascontiguousarray(optimal_radius, np.float64)
        rc = self.orc.lib.orc_run_stage(
            self.h, ctypes.addressof(opts),
            kopt.ctypes.data_as(dp) if kopt is not None else None,
            ropt.ctypes.data_as(dp) if ropt is not None else None,
            int(mode), cols, status.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            int(threads or os.cpu_count() or 1))
        if opts.kind == STAGE_OUTLIER and rc >= 0:
            self.outliers = rc
        elif rc != 0:
            raise RuntimeError(f"orc_run_stage failed ({rc})")
        return outs[:nd], status

"""ctypes mirror of include/nbg_b200.h and the loader of the native library.

The product path is the in-tree shared library ``gpupdal_b200/_lib/libnbg_b200.so``
(hand-written sm_100a CUDA behind a C ABI).  Loading fails loudly when it is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libnbg_b200.so")

NBG_OK = 0
NBG_ERR_INVALID = 1
NBG_ERR_OOM = 2
NBG_ERR_BUDGET = 3
NBG_ERR_CUDA = 4
NBG_ERR_TIMEOUT = 5
NBG_ERR_UNSUPPORTED = 6
NBG_ERR_NO_DEVICE = 7
NBG_ERR_EXCEPTIONS = 8

STAGE_NORMAL = 1
STAGE_EIGENVALUES = 2
STAGE_COVARIANCEFEATURES = 3
STAGE_APPROXIMATECOPLANAR = 4
STAGE_ESTIMATERANK = 5
STAGE_NNDISTANCE = 6
STAGE_OPTIMALNEIGHBORHOOD = 7
STAGE_LOF = 8
STAGE_OUTLIER = 9

# covariance feature bits, reference order of feature_set "all"
FEATURES = [
    "Linearity",
    "Planarity",
    "Scattering",
    "Verticality",
    "Omnivariance",
    "Anisotropy",
    "Eigenentropy",
    "EigenvalueSum",
    "SurfaceVariation",
    "DemantkeVerticality",
    "Density",
]
FEAT_BIT = {name: 1 << i for i, name in enumerate(FEATURES)}
globals().update({"FEAT_" + name.upper(): 1 << i for i, name in enumerate(FEATURES)})
FEAT_DIMENSIONALITY = 0x0F
FEAT_ALL = 0x7FF

MODE_RAW = 0
MODE_SQRT = 1
MODE_NORMALIZED = 2

ROW_TOO_FEW = 1
ROW_ZERO_COV = 2
ROW_EIGEN_FAIL = 3
ROW_ZERO_LAMBDA = 4
ROW_RADIUS_FEW = 5

MAX_DIMS = 16
NOALLOC_MAX_POINTS = 524288

NORMAL_DIMS = ["NormalX", "NormalY", "NormalZ", "Curvature"]
EIGENVALUE_DIMS = ["Eigenvalue0", "Eigenvalue1", "Eigenvalue2"]
CONSUMER_DIMS = {
    STAGE_APPROXIMATECOPLANAR: ["Coplanar"],
    STAGE_ESTIMATERANK: ["Rank"],
    STAGE_NNDISTANCE: ["NNDistance"],
    STAGE_OPTIMALNEIGHBORHOOD: ["OptimalKNN", "OptimalRadius"],
    STAGE_LOF: ["NNDistance", "LocalReachabilityDistance", "LocalOutlierFactor"],
    STAGE_OUTLIER: ["Classification"],
}


class StageOpts(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("knn", ctypes.c_int32),
        ("always_up", ctypes.c_int32),
        ("has_viewpoint", ctypes.c_int32),
        ("viewpoint", ctypes.c_double * 3),
        ("refine", ctypes.c_int32),
        ("normalize", ctypes.c_int32),
        ("feature_mask", ctypes.c_uint32),
        ("mode", ctypes.c_int32),
        ("stride", ctypes.c_int32),
        ("optimized", ctypes.c_int32),
        ("use_radius", ctypes.c_int32),
        ("min_k", ctypes.c_int32),
        ("radius", ctypes.c_double),
        ("thresh1", ctypes.c_double),
        ("thresh2", ctypes.c_double),
        ("label", ctypes.c_int32),
        ("eigen_fp64", ctypes.c_int32),
    ]


class Columns(ctypes.Structure):
    _fields_ = [
        ("base", ctypes.c_void_p),
        ("point_stride", ctypes.c_int64),
        ("ndims", ctypes.c_int32),
        ("on_device", ctypes.c_int32),
        ("offset", ctypes.c_int64 * MAX_DIMS),
    ]


class RowException(ctypes.Structure):
    _fields_ = [
        ("point_id", ctypes.c_uint32),
        ("stage", ctypes.c_uint8),
        ("code", ctypes.c_uint8),
        ("reserved", ctypes.c_uint16),
    ]


class RunStats(ctypes.Structure):
    _fields_ = [
        ("points", ctypes.c_uint64),
        ("tie_rows", ctypes.c_uint64),
        ("deferred_rows", ctypes.c_uint64),
        ("resolved_rows", ctypes.c_uint64),
        ("grid_ms", ctypes.c_double),
        ("query_ms", ctypes.c_double),
        ("tree_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("replay_rows", ctypes.c_uint64),
        ("kd_build_ms", ctypes.c_double),
        ("outliers", ctypes.c_uint64),
        ("inliers", ctypes.c_uint64),
        ("output_chunks", ctypes.c_uint64),
        ("retry_rows", ctypes.c_uint64),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("tile", ctypes.c_void_p),
        ("n_stages", ctypes.c_int32),
        ("exception_capacity", ctypes.c_uint32),
        ("stages", ctypes.POINTER(StageOpts)),
        ("outputs", ctypes.POINTER(Columns)),
        ("optimal_knn", ctypes.c_void_p),
        ("optimal_radius", ctypes.c_void_p),
        ("exceptions", ctypes.c_void_p),
        ("n_exceptions", ctypes.POINTER(ctypes.c_uint32)),
    ]


BATCH_GRAPH = 1
BATCH_AUTOTUNE = 2


class Request(ctypes.Structure):
    _fields_ = [
        ("x", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("n", ctypes.c_uint64),
        ("scale", ctypes.c_double * 3),
        ("offset", ctypes.c_double * 3),
        ("on_device", ctypes.c_int32),
        ("n_stages", ctypes.c_int32),
        ("stages", ctypes.POINTER(StageOpts)),
        ("outputs", ctypes.POINTER(Columns)),
        ("optimal_knn", ctypes.c_void_p),
        ("optimal_radius", ctypes.c_void_p),
        ("aux_on_device", ctypes.c_int32),
        ("exception_capacity", ctypes.c_uint32),
        ("exceptions", ctypes.c_void_p),
        ("user_tag", ctypes.c_uint64),
    ]


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("n_exceptions", ctypes.c_uint32),
        ("user_tag", ctypes.c_uint64),
        ("submit_us", ctypes.c_double),
        ("start_us", ctypes.c_double),
        ("end_us", ctypes.c_double),
        ("est_bytes", ctypes.c_uint64),
        ("stats", RunStats),
    ]


class TuneEntry(ctypes.Structure):
    _fields_ = [
        ("size_class", ctypes.c_int32),
        ("slots", ctypes.c_int32),
        ("cell_factor", ctypes.c_float),
        ("select_kernel", ctypes.c_int32),
    ]


class LasInfo(ctypes.Structure):
    _fields_ = [
        ("version_major", ctypes.c_uint8),
        ("version_minor", ctypes.c_uint8),
        ("point_format", ctypes.c_uint8),
        ("compressed", ctypes.c_uint8),
        ("point_record_length", ctypes.c_uint16),
        ("reserved", ctypes.c_uint16),
        ("offset_to_points", ctypes.c_uint32),
        ("point_count", ctypes.c_uint64),
        ("scale", ctypes.c_double * 3),
        ("offset", ctypes.c_double * 3),
        ("min", ctypes.c_double * 3),
        ("max", ctypes.c_double * 3),
    ]


def stage_dims(opts: StageOpts) -> list:
    """Output dimension names of one stage, in the library's order."""
    if opts.kind == STAGE_NORMAL:
        return list(NORMAL_DIMS)
    if opts.kind == STAGE_EIGENVALUES:
        return list(EIGENVALUE_DIMS)
    if opts.kind in CONSUMER_DIMS:
        return list(CONSUMER_DIMS[opts.kind])
    return [f for i, f in enumerate(FEATURES) if opts.feature_mask & (1 << i)]


def make_opts(kind, knn=8, always_up=True, viewpoint=None, refine=False,
              normalize=False, feature_mask=FEAT_DIMENSIONALITY, mode=MODE_SQRT,
              stride=1, optimized=False, radius=None, min_k=3, thresh1=0.0, thresh2=0.0,
              label=0, eigen_fp64=False) -> StageOpts:
    o = StageOpts()
    o.kind = int(kind)
    o.knn = int(knn)
    o.always_up = int(bool(always_up))
    o.has_viewpoint = int(viewpoint is not None)
    if viewpoint is not None:
        for i in range(3):
            o.viewpoint[i] = float(viewpoint[i])
    o.refine = int(bool(refine))
    o.normalize = int(bool(normalize))
    o.feature_mask = int(feature_mask)
    o.mode = int(mode)
    o.stride = int(stride)
    o.optimized = int(bool(optimized))
    o.use_radius = int(radius is not None)
    o.radius = float(radius) if radius is not None else 0.0
    o.min_k = int(min_k)
    o.thresh1 = float(thresh1)
    o.thresh2 = float(thresh2)
    o.label = int(label)
    o.eigen_fp64 = int(bool(eigen_fp64))
    return o


def consumer_opts(kind, **kw) -> StageOpts:
    """Options of a kNN-consumer stage under the reference's option names
    and defaults (ApproximateCoplanarFilter.cpp:66-71, EstimateRankFilter.cpp:
    66-70, NNDistanceFilter.cpp:95-99, OptimalNeighborhoodFilter.cpp:62-66,
    LOFFilter.cpp:62-65, OutlierFilter.cpp:62-71)."""
    if kind == STAGE_APPROXIMATECOPLANAR:
        return make_opts(kind, knn=kw.get("knn", 8), thresh1=kw.get("thresh1", 25.0),
                         thresh2=kw.get("thresh2", 6.0))
    if kind == STAGE_ESTIMATERANK:
        return make_opts(kind, knn=kw.get("knn", 8), thresh1=kw.get("thresh", 0.01))
    if kind == STAGE_NNDISTANCE:
        return make_opts(kind, knn=kw.get("k", 10), mode={"kth": 0, "avg": 1}[kw.get("mode", "kth")])
    if kind == STAGE_OPTIMALNEIGHBORHOOD:
        return make_opts(kind, knn=kw.get("max_k", 14), min_k=kw.get("min_k", 10))
    if kind == STAGE_LOF:
        return make_opts(kind, knn=kw.get("minpts", 10))
    if kind == STAGE_OUTLIER:
        method = kw.get("method", "statistical")
        o = make_opts(kind, knn=kw.get("mean_k", 8), min_k=kw.get("min_k", 2),
                      thresh1=kw.get("multiplier", 2.0), label=kw.get("cls", 7),
                      mode={"statistical": 0, "radius": 1}[method])
        o.radius = float(kw.get("radius", 1.0))
        return o
    raise ValueError(f"not a consumer stage kind: {kind}")


_LIB = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the native library; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(
            f"native library {path} is missing; build it with "
            "`python -m gpupdal_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    u64 = ctypes.c_uint64
    i32 = ctypes.c_int32
    lib.nbg_version.restype = ctypes.c_char_p
    lib.nbg_device_count.restype = ctypes.c_int
    lib.nbg_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, u64]
    lib.nbg_create.restype = ctypes.c_int
    lib.nbg_destroy.argtypes = [vp]
    lib.nbg_destroy.restype = ctypes.c_int
    lib.nbg_last_error.argtypes = [vp]
    lib.nbg_last_error.restype = ctypes.c_char_p
    lib.nbg_tile_upload.argtypes = [vp, vp, vp, vp, u64, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), i32, vp,
                                    ctypes.POINTER(vp)]
    lib.nbg_tile_upload.restype = ctypes.c_int
    lib.nbg_las_header.argtypes = [vp, ctypes.c_size_t, ctypes.POINTER(LasInfo)]
    lib.nbg_las_header.restype = ctypes.c_int
    lib.nbg_tile_upload_las.argtypes = [vp, vp, u64, ctypes.c_uint32, i32,
                                        ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double), vp, ctypes.POINTER(vp)]
    lib.nbg_tile_upload_las.restype = ctypes.c_int
    lib.nbg_tile_free.argtypes = [vp, vp]
    lib.nbg_tile_free.restype = ctypes.c_int
    lib.nbg_tile_tune.argtypes = [vp, vp, ctypes.c_float, i32]
    lib.nbg_tile_tune.restype = ctypes.c_int
    lib.nbg_tile_set_select.argtypes = [vp, vp, i32, ctypes.c_float]
    lib.nbg_tile_set_select.restype = ctypes.c_int
    lib.nbg_tile_autotune.argtypes = [vp, vp, i32, ctypes.POINTER(ctypes.c_float), i32, i32,
                                      ctypes.POINTER(ctypes.c_float), vp]
    lib.nbg_tile_autotune.restype = ctypes.c_int
    lib.nbg_autotune_cache_get.argtypes = [vp, ctypes.POINTER(TuneEntry), i32,
                                           ctypes.POINTER(ctypes.c_int32)]
    lib.nbg_autotune_cache_get.restype = ctypes.c_int
    lib.nbg_autotune_cache_set.argtypes = [vp, ctypes.POINTER(TuneEntry), i32]
    lib.nbg_autotune_cache_set.restype = ctypes.c_int
    lib.nbg_tile_size.argtypes = [vp]
    lib.nbg_tile_size.restype = u64
    lib.nbg_run.argtypes = [vp, vp, ctypes.POINTER(StageOpts), i32, ctypes.POINTER(Columns),
                            vp, vp, i32, ctypes.POINTER(RowException), ctypes.c_uint32,
                            ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(RunStats), vp]
    lib.nbg_run.restype = ctypes.c_int
    lib.nbg_neighbor_sets.argtypes = [vp, vp, i32, vp, i32, ctypes.POINTER(RunStats), vp]
    lib.nbg_neighbor_sets.restype = ctypes.c_int
    lib.nbg_stage_noalloc.argtypes = [vp, vp, vp, u64, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(StageOpts),
                                      ctypes.POINTER(Columns), vp, vp, vp,
                                      ctypes.POINTER(ctypes.c_uint32), vp, ctypes.c_uint32,
                                      ctypes.POINTER(ctypes.c_uint32), vp, ctypes.c_char_p,
                                      ctypes.c_size_t]
    lib.nbg_stage_noalloc.restype = ctypes.c_int
    lib.nbg_debug_kd_export.argtypes = [vp, vp] + [vp] * 9 + [ctypes.c_uint32]
    lib.nbg_debug_kd_export.restype = ctypes.c_int
    cp = ctypes.c_char_p
    lib.nbg_filter_create.argtypes = [cp, cp, i32, i32, ctypes.POINTER(vp), cp, ctypes.c_size_t]
    lib.nbg_filter_create.restype = ctypes.c_int
    lib.nbg_filter_options.argtypes = [vp, ctypes.POINTER(StageOpts)]
    lib.nbg_filter_options.restype = ctypes.c_int
    lib.nbg_filter_dims.argtypes = [vp, cp, ctypes.c_size_t]
    lib.nbg_filter_dims.restype = ctypes.c_int
    lib.nbg_filter_log.argtypes = [vp]
    lib.nbg_filter_log.restype = cp
    lib.nbg_filter_report.argtypes = [vp, ctypes.POINTER(RowException), ctypes.c_uint32, i32, cp,
                                      ctypes.c_size_t]
    lib.nbg_filter_report.restype = ctypes.c_int
    lib.nbg_filter_outcome.argtypes = [vp, ctypes.POINTER(RunStats)]
    lib.nbg_filter_outcome.restype = ctypes.c_int
    lib.nbg_filter_free.argtypes = [vp]
    lib.nbg_filter_free.restype = None
    lib.nbg_pipeline_parse.argtypes = [cp, ctypes.POINTER(vp), cp, ctypes.c_size_t]
    lib.nbg_pipeline_parse.restype = ctypes.c_int
    lib.nbg_pipeline_size.argtypes = [vp]
    lib.nbg_pipeline_size.restype = i32
    lib.nbg_pipeline_type.argtypes = [vp, i32]
    lib.nbg_pipeline_type.restype = cp
    lib.nbg_pipeline_options.argtypes = [vp, i32]
    lib.nbg_pipeline_options.restype = cp
    lib.nbg_pipeline_free.argtypes = [vp]
    lib.nbg_pipeline_free.restype = None
    lib.nbg_run_batch.argtypes = [vp, ctypes.POINTER(BatchItem), i32, ctypes.c_uint32,
                                  ctypes.POINTER(RunStats), vp]
    lib.nbg_run_batch.restype = ctypes.c_int
    lib.nbg_server_create.argtypes = [ctypes.POINTER(vp), i32, i32, u64]
    lib.nbg_server_create.restype = ctypes.c_int
    lib.nbg_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]
    lib.nbg_server_submit.restype = ctypes.c_int
    lib.nbg_server_wait.argtypes = [vp, ctypes.c_uint64, i32, ctypes.POINTER(RequestResult)]
    lib.nbg_server_wait.restype = ctypes.c_int
    lib.nbg_request_bytes.argtypes = [ctypes.POINTER(Request)]
    lib.nbg_request_bytes.restype = u64
    lib.nbg_server_last_error.argtypes = [vp]
    lib.nbg_server_last_error.restype = ctypes.c_char_p
    lib.nbg_server_destroy.argtypes = [vp]
    lib.nbg_server_destroy.restype = ctypes.c_int
    _LIB = lib
    return lib

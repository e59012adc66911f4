// nbg_noalloc.cu — one stage over one tile without any device allocation.
//
// Some callers cannot allocate device memory at the time they need
// neighbourhood geometry: code running inside another framework's memory
// pool or allocator (a host application that owns every device byte), a
// real-time loop that must not call cudaMalloc/cudaFree (they can block the
// device), or a plug-in whose host forbids allocation in its processing
// callback.  nbg_stage_noalloc serves them: the caller passes device inputs
// and outputs, and every byte of working memory (the uniform grid: cell keys,
// cell table, points in cell order, the scan's temporary storage and the
// counters) comes from one file-scope device array of fixed size.
//
// What it runs: the grid build and the fused kNN + covariance + eigensolve +
// projection kernel of the regular path.  Rows whose neighbour set depends on
// the reference's tie order, or whose search did not finish within the ring
// limit, need the exact KD replica, whose working memory grows with the tile;
// this entry point does not build it and instead returns those point ids to
// the caller (who can answer them later with nbg_run).
//
// The array is shared by every call in the process on a given device and
// keeps the last call's contents; the entry point clears what must start at
// zero.  Calls whose work overlaps on the same device race on it, so calls on
// one device must be serialised (for example, all issued on one stream).
// Every call looks up the array's device address with the device current;
// the first call on a device also loads the library's device code there, so
// make it outside any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "nbg_internal.h"

namespace nbg {
namespace {

constexpr uint64_t kMaxPoints = NBG_NOALLOC_MAX_POINTS;
constexpr uint64_t kColsCap = 2 * kMaxPoints + 1024;
constexpr uint64_t kTableCap = 4 * kMaxPoints + 1024;
constexpr size_t kTmpReserve = 1u << 20;  // CUB scan storage
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffBbox = 0;
constexpr size_t kOffGp = kOffBbox + 256;
constexpr size_t kOffCounters = kOffGp + align256(sizeof(GridParams));
constexpr size_t kOffTable = kOffCounters + 256;
constexpr size_t kOffColinfo = kOffTable + 256;
constexpr size_t kOffExt = kOffColinfo + align256(kColsCap * 16);
constexpr size_t kOffKeys = kOffExt + align256((kColsCap + 1) * 4);
constexpr size_t kOffCstart = kOffKeys + align256(kMaxPoints * 4);
constexpr size_t kOffCursor = kOffCstart + align256(kTableCap * 4);
constexpr size_t kOffSorted = kOffCursor + align256(kTableCap * 4);
constexpr size_t kOffTmp = kOffSorted + align256(kMaxPoints * 16);
constexpr size_t kArenaBytes = kOffTmp + kTmpReserve;

// All working memory of nbg_stage_noalloc (about 49 MB); held by every
// device that loads this library until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_arena[kArenaBytes];

int set_msg(char* buf, size_t len, int code, const char* msg) {
    if (buf && len) {
        std::strncpy(buf, msg, len - 1);
        buf[len - 1] = '\0';
    }
    return code;
}

}  // namespace
}  // namespace nbg

using namespace nbg;

extern "C" int nbg_stage_noalloc(const int32_t* x, const int32_t* y, const int32_t* z, uint64_t n,
                                 const double scale[3], const double offset[3],
                                 const nbg_stage_opts* opts, const nbg_columns* out,
                                 const double* optimal_knn, const double* optimal_radius,
                                 uint32_t* unresolved, uint32_t* n_unresolved,
                                 nbg_row_exception* exceptions, uint32_t exception_capacity,
                                 uint32_t* n_exceptions, void* stream_v, char* err_msg,
                                 size_t err_len) {
    if (n_unresolved) *n_unresolved = 0;
    if (n_exceptions) *n_exceptions = 0;
    if (!opts || !out || !scale || !offset || !n_unresolved || !n_exceptions)
        return set_msg(err_msg, err_len, NBG_ERR_INVALID, "null argument");
    if (n > kMaxPoints)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED,
                       "tile larger than NBG_NOALLOC_MAX_POINTS; use nbg_tile_upload + nbg_run");
    if (n > 0 && (!x || !y || !z || !unresolved))
        return set_msg(err_msg, err_len, NBG_ERR_INVALID, "null device array");
    if (exception_capacity > 0 && !exceptions)
        return set_msg(err_msg, err_len, NBG_ERR_INVALID, "null exception array with a capacity");
    if (scale[0] != scale[1] || scale[0] != scale[2] || !(scale[0] > 0.0))
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED, "needs one positive scale for x, y, z");
    {
        // the regular path's option checks first (same codes and messages)
        Context vctx;
        bool need_aux = false;
        const int vrc = validate_stages(&vctx, opts, 1, out, &need_aux);
        if (vrc) return set_msg(err_msg, err_len, vrc, vctx.err.c_str());
    }
    // then what this entry point does not run
    if (opts->kind > NBG_STAGE_COVARIANCEFEATURES)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED,
                       "only normal, eigenvalues and covariancefeatures run without allocation");
    if (opts->kind != NBG_STAGE_NORMAL && opts->stride > 1)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED, "stride > 1 is not supported");
    if (opts->kind == NBG_STAGE_COVARIANCEFEATURES && opts->optimized)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED, "optimized is not supported");
    if (opts->use_radius)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED,
                       "radius neighbourhoods are not supported by this entry point");
    const int ndims = out->ndims;
    if (out->on_device != 1)
        return set_msg(err_msg, err_len, NBG_ERR_INVALID, "outputs must be device columns");
    if (opts->kind == NBG_STAGE_COVARIANCEFEATURES && (opts->feature_mask & NBG_FEAT_DENSITY) &&
        (!optimal_knn || !optimal_radius))
        return set_msg(err_msg, err_len, NBG_ERR_INVALID, "Density needs OptimalKNN and OptimalRadius");
    if (n == 0) return NBG_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0)
        return set_msg(err_msg, err_len, NBG_ERR_NO_DEVICE, "no current device");
    // The array's device address on the current device (the host-side symbol
    // is not a device address).  Looked up on every call: a cached address
    // would go stale after cudaDeviceReset or a new primary context, and the
    // lookup is a cheap host query once the device code is loaded.
    unsigned char* arena = nullptr;
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_arena);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_msg(err_msg, err_len, NBG_ERR_CUDA, "cudaGetSymbolAddress failed");
        }
        arena = (unsigned char*)p;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    Context ctx;  // carries the SM count for the launch shapes; allocates nothing
    ctx.device = dev;
    ctx.sm_count = sms;
    Tile t;
    t.n = n;
    t.x = const_cast<int32_t*>(x);
    t.y = const_cast<int32_t*>(y);
    t.z = const_cast<int32_t*>(z);
    for (int d = 0; d < 3; ++d) {
        t.tf.scale[d] = scale[d];
        t.tf.offset[d] = offset[d];
    }
    t.bbox = (int32_t*)(arena + kOffBbox);
    t.gp = (GridParams*)(arena + kOffGp);
    t.table_dev = (uint32_t*)(arena + kOffTable);
    t.colinfo = (int4*)(arena + kOffColinfo);
    t.ext = (uint32_t*)(arena + kOffExt);
    t.keys = (uint32_t*)(arena + kOffKeys);
    t.cstart = (uint32_t*)(arena + kOffCstart);
    t.cursor = (uint32_t*)(arena + kOffCursor);
    t.sorted = (float4*)(arena + kOffSorted);
    t.cols_cap = 2 * n + 1024;
    t.table_cap = kTableCap;
    t.fixed_storage = true;
    t.grid_tmp = arena + kOffTmp;
    t.grid_tmp_bytes = kTmpReserve;
    if (grid_temp_bytes(std::max<uint64_t>(kTableCap, t.cols_cap + 1)) > kTmpReserve)
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED, "grid storage exceeds its reserve");
    uint32_t* counters = (uint32_t*)(arena + kOffCounters);
    const int K = (int)(n < (uint64_t)opts->knn + 1 ? n : (uint64_t)opts->knn + 1);

    // counters start at zero on every call (the array keeps the last call's)
    if (cudaMemsetAsync(counters, 0, 256, stream) != cudaSuccess)
        return set_msg(err_msg, err_len, NBG_ERR_CUDA, "counter reset failed");
    int rc = build_grid(&ctx, &t, K, stream);
    if (rc) return set_msg(err_msg, err_len, rc, ctx.err.empty() ? "grid build failed" : ctx.err.c_str());
    GridParams hg;
    cudaError_t e = cudaMemcpyAsync(&hg, t.gp, sizeof(GridParams), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return set_msg(err_msg, err_len, NBG_ERR_CUDA, cudaGetErrorString(e));
    if ((int64_t)hg.maxx - hg.minx >= (1 << 24) || (int64_t)hg.maxy - hg.miny >= (1 << 24) ||
        (int64_t)hg.maxz - hg.minz >= (1 << 24))
        return set_msg(err_msg, err_len, NBG_ERR_UNSUPPORTED, "tile extent must be below 2^24 raw units");

    StageGroup g{};
    g.nstages = 1;
    g.stage_index[0] = 0;
    g.optimal_knn = optimal_knn;
    g.optimal_radius = optimal_radius;
    StageDev& d = g.st[0];
    d.kind = opts->kind;
    d.always_up = opts->always_up;
    d.has_viewpoint = opts->has_viewpoint;
    d.normalize = opts->normalize;
    for (int k = 0; k < 3; ++k) d.viewpoint[k] = opts->viewpoint[k];
    d.feature_mask = opts->feature_mask & NBG_FEAT_ALL;
    d.mode = opts->mode;
    d.ndims = ndims;
    d.base = (char*)out->base;
    d.point_stride = out->point_stride;
    for (int k = 0; k < NBG_MAX_DIMS; ++k) d.offset[k] = out->offset[k];
    g.sign_exact = (opts->kind == NBG_STAGE_NORMAL && !opts->always_up && !opts->has_viewpoint) ||
                   opts->eigen_fp64;
    QueryLaunch ql;
    ql.tile = &t;
    ql.K = K;
    ql.rmax = 8;
    ql.grp = g;
    ql.ex = ExceptionSink{exceptions, counters + 3, exception_capacity};
    ql.exact_rows = unresolved;
    ql.counters = counters;
    rc = launch_query(&ctx, ql, stream);
    if (rc) return set_msg(err_msg, err_len, rc, "query launch failed");
    uint32_t cnt[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return set_msg(err_msg, err_len, NBG_ERR_CUDA, cudaGetErrorString(e));
    *n_unresolved = cnt[0];
    *n_exceptions = cnt[3];
    if (cnt[3] > exception_capacity)
        return set_msg(err_msg, err_len, NBG_ERR_EXCEPTIONS, "row-exception list overflowed");
    return NBG_OK;
}

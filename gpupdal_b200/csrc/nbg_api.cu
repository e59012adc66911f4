// nbg_api.cu — the C ABI declared in include/nbg_b200.h.
//
// Orchestrates one call the way the reference's stage loop does
// (filters/NormalFilter.cpp:288-299 filter(), EigenvaluesFilter.cpp:115,
// CovarianceFeaturesFilter.cpp:175): index the view, then answer every point;
// stages sharing a neighbour count share one fused pass, as later PDAL
// stages reuse the view's KD3 index (pdal/PointView.cpp:276-290).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <new>
#include <string>
#include <vector>

#include "nbg_internal.h"


namespace nbg {

int slots_for_k(int K);

void set_err(Context* c, const std::string& msg) {
    if (!c) return;
    std::lock_guard<std::mutex> lock(c->emu);
    c->err = msg;
}

int fail(Context* c, int code, const std::string& msg) {
    set_err(c, msg);
    return code;
}

static int cuda_fail(Context* c, cudaError_t e, const char* what) {
    return fail(c, NBG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define NBG_TRY(call, what)                               \
    do {                                                  \
        cudaError_t e__ = (call);                         \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, what); \
    } while (0)

std::atomic<uint64_t> g_launches{0};

static size_t round_bytes(size_t bytes) { return bytes == 0 ? 256 : ((bytes + 255) / 256) * 256; }

// Size class of a request: 256-byte granules up to 64 KiB, then eighth-octave
// steps (at most 12.5% over the request).
static size_t size_class(size_t bytes) {
    bytes = round_bytes(bytes);
    if (bytes <= (64u << 10)) return bytes;
    size_t p = (size_t)1 << (63 - __builtin_clzll((unsigned long long)bytes));
    const size_t step = p / 8;
    return ((bytes + step - 1) / step) * step;
}

static void trim_locked(Context* ctx) {
    for (auto& kv : ctx->cache) cudaFree(kv.second);
    ctx->used -= std::min<uint64_t>(ctx->used, ctx->cached);
    ctx->cache.clear();
    ctx->cached = 0;
}

void ctx_trim(Context* ctx) {
    std::lock_guard<std::mutex> lock(ctx->amu);
    trim_locked(ctx);
}

// Device allocation through the context's cache: the smallest cached block
// of at least the request's size class and at most twice it is reused, so
// calls of varying sizes (a request stream) recycle their blocks.
int ctx_alloc(Context* ctx, void** p, size_t bytes) {
    bytes = size_class(bytes);
    std::lock_guard<std::mutex> lock(ctx->amu);
    auto it = ctx->cache.lower_bound(bytes);
    if (it != ctx->cache.end() && it->first <= 2 * bytes) {
        *p = it->second;
        ctx->live[*p] = it->first;
        ctx->cached -= it->first;
        ctx->cache.erase(it);
        return NBG_OK;
    }
    if (ctx->budget && ctx->used + bytes > ctx->budget) trim_locked(ctx);
    if (ctx->budget && ctx->used + bytes > ctx->budget)
        return fail(ctx, NBG_ERR_BUDGET, "HBM budget exceeded");
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        trim_locked(ctx);
        e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return fail(ctx, NBG_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
    }
    ctx->used += bytes;
    ctx->live[*p] = bytes;
    return NBG_OK;
}

void ctx_free(Context* ctx, void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(ctx->amu);
    auto it = ctx->live.find(p);
    if (it != ctx->live.end()) {
        bytes = it->second;
        ctx->live.erase(it);
    } else {
        bytes = size_class(bytes);
    }
    ctx->cache.emplace(bytes, p);
    ctx->cached += bytes;
}

// ---------------------------------------------------------------------------
// host copies
static constexpr size_t kBounce = (size_t)32 << 20;

static bool host_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static int bounce_init(Context* ctx) {
    if (ctx->bounce_ready) return NBG_OK;
    for (int i = 0; i < 2; ++i) {
        if (cudaHostAlloc((void**)&ctx->bounce[i], kBounce, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->bev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, NBG_ERR_OOM, "pinned bounce buffer");
        }
    }
    ctx->bounce_ready = true;
    return NBG_OK;
}

// memcpy with up to 4 host threads for large blocks
static void par_memcpy(void* dst, const void* src, size_t bytes) {
    const size_t per = (size_t)8 << 20;
    const int nt = (int)std::min<size_t>(4, (bytes + per - 1) / per);
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t part = (bytes + nt - 1) / nt;
    for (int i = 1; i < nt; ++i) {
        const size_t off = part * i;
        if (off >= bytes) break;
        th.emplace_back([=] { std::memcpy((char*)dst + off, (const char*)src + off,
                                          std::min(part, bytes - off)); });
    }
    std::memcpy(dst, src, std::min(part, bytes));
    for (auto& t : th) t.join();
}

int host_to_device(Context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    NBG_RANGE("nbg copy in");
    if (!bytes) return NBG_OK;
    if (bytes < ((size_t)1 << 20) || host_pinned(src)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
        return e ? cuda_fail(ctx, e, "host to device copy") : NBG_OK;
    }
    int rc = bounce_init(ctx);
    if (rc) return rc;
    const size_t nch = (bytes + kBounce - 1) / kBounce;
    for (size_t k = 0; k < nch; ++k) {
        const int b = (int)(k & 1);
        const size_t off = k * kBounce, len = std::min(kBounce, bytes - off);
        // the copy that last read this buffer must be done
        if (cudaEventSynchronize(ctx->bev[b]) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "bounce");
        par_memcpy(ctx->bounce[b], (const char*)src + off, len);
        cudaError_t e = cudaMemcpyAsync((char*)dst + off, ctx->bounce[b], len, cudaMemcpyHostToDevice, stream);
        if (!e) e = cudaEventRecord(ctx->bev[b], stream);
        if (e) return cuda_fail(ctx, e, "host to device copy");
    }
    return NBG_OK;
}

int device_to_host(Context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    NBG_RANGE("nbg copy back");
    if (!bytes) return NBG_OK;
    if (bytes < ((size_t)1 << 20) || host_pinned(dst)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        return e ? cuda_fail(ctx, e, "device to host copy") : NBG_OK;
    }
    int rc = bounce_init(ctx);
    if (rc) return rc;
    const size_t nch = (bytes + kBounce - 1) / kBounce;
    auto issue = [&](size_t k) -> cudaError_t {
        const int b = (int)(k & 1);
        const size_t off = k * kBounce, len = std::min(kBounce, bytes - off);
        cudaError_t e = cudaMemcpyAsync(ctx->bounce[b], (const char*)src + off, len,
                                        cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaEventRecord(ctx->bev[b], stream);
        return e;
    };
    // previous users of the buffers (host-to-device chunks) must be done
    for (int b = 0; b < 2; ++b)
        if (cudaEventSynchronize(ctx->bev[b]) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "bounce");
    cudaError_t e = issue(0);
    for (size_t k = 0; k < nch && !e; ++k) {
        if (k + 1 < nch) e = issue(k + 1);
        if (e) break;
        const int b = (int)(k & 1);
        e = cudaEventSynchronize(ctx->bev[b]);
        if (e) break;
        const size_t off = k * kBounce, len = std::min(kBounce, bytes - off);
        par_memcpy((char*)dst + off, ctx->bounce[b], len);
    }
    return e ? cuda_fail(ctx, e, "device to host copy") : NBG_OK;
}

static int dev_alloc(Context* ctx, void** p, size_t bytes, uint64_t* account) {
    int rc = ctx_alloc(ctx, p, bytes);
    if (rc == NBG_OK && account) *account += round_bytes(bytes);
    return rc;
}

static void dev_free(Context* ctx, void* p, size_t bytes) { ctx_free(ctx, p, bytes); }

int ensure_scratch(Context* ctx, uint64_t n, uint64_t ex_cap) {
    if (ctx->sums_cap < n) {
        if (ctx->sums) dev_free(ctx, ctx->sums, ctx->sums_cap * sizeof(RowSums));
        ctx->sums = nullptr;
        ctx->sums_cap = 0;
        int rc = dev_alloc(ctx, (void**)&ctx->sums, std::max<uint64_t>(n, 1024) * sizeof(RowSums), nullptr);
        if (rc) return rc;
        ctx->sums_cap = std::max<uint64_t>(n, 1024);
    }
    if (ctx->tie_cap < n) {
        if (ctx->ties) dev_free(ctx, ctx->ties, ctx->tie_cap * sizeof(uint2));
        ctx->ties = nullptr;
        ctx->tie_cap = 0;
        int rc = dev_alloc(ctx, (void**)&ctx->ties, std::max<uint64_t>(n, 1024) * sizeof(uint2), nullptr);
        if (rc) return rc;
        ctx->tie_cap = std::max<uint64_t>(n, 1024);
    }
    if (ctx->retry_cap < n) {
        if (ctx->retry_rows) dev_free(ctx, ctx->retry_rows, ctx->retry_cap * 4);
        ctx->retry_rows = nullptr;
        ctx->retry_cap = 0;
        int rc = dev_alloc(ctx, (void**)&ctx->retry_rows, std::max<uint64_t>(n, 1024) * 4, nullptr);
        if (rc) return rc;
        ctx->retry_cap = std::max<uint64_t>(n, 1024);
    }
    if (ctx->exact_cap < n) {
        if (ctx->exact_rows) dev_free(ctx, ctx->exact_rows, ctx->exact_cap * 4);
        ctx->exact_rows = nullptr;
        ctx->exact_cap = 0;
        int rc = dev_alloc(ctx, (void**)&ctx->exact_rows, std::max<uint64_t>(n, 1024) * 4, nullptr);
        if (rc) return rc;
        ctx->exact_cap = std::max<uint64_t>(n, 1024);
    }
    if (ctx->ex_cap < ex_cap) {
        if (ctx->ex_rows) dev_free(ctx, ctx->ex_rows, ctx->ex_cap * sizeof(nbg_row_exception));
        ctx->ex_rows = nullptr;
        ctx->ex_cap = 0;
        int rc = dev_alloc(ctx, (void**)&ctx->ex_rows, ex_cap * sizeof(nbg_row_exception), nullptr);
        if (rc) return rc;
        ctx->ex_cap = ex_cap;
    }
    return NBG_OK;
}

static void tile_release(Context* ctx, Tile* t) {
    kd_free(ctx, t);
    const uint64_t n = t->n;
    dev_free(ctx, t->x, n * 4);
    dev_free(ctx, t->y, n * 4);
    dev_free(ctx, t->z, n * 4);
    dev_free(ctx, t->bbox, 64);
    dev_free(ctx, t->gp, sizeof(GridParams));
    dev_free(ctx, t->colinfo, t->cols_cap * 16);
    dev_free(ctx, t->ext, (t->cols_cap + 1) * 4);
    dev_free(ctx, t->table_dev, 16);
    dev_free(ctx, t->keys, n * 4);
    dev_free(ctx, t->cstart, t->table_cap * 4);
    dev_free(ctx, t->cursor, t->table_cap * 4);
    dev_free(ctx, t->sorted, n * 16);
    dev_free(ctx, t->grid_tmp, t->grid_tmp_bytes);
    t->x = t->y = t->z = nullptr;
}

}  // namespace nbg

namespace nbg {
// Grows the cell table (cstart, cursor) and the scan storage to `entries`.
int grid_grow_table(Context* ctx, Tile* t, uint64_t entries) {
    if (t->fixed_storage) {
        set_err(ctx, "cell table exceeds the fixed storage");
        return NBG_ERR_UNSUPPORTED;
    }
    const uint64_t cap = std::max<uint64_t>(entries, 2 * t->table_cap);
    uint32_t *cs = nullptr, *cu = nullptr;
    int rc = dev_alloc(ctx, (void**)&cs, cap * 4, &t->bytes);
    if (!rc) rc = dev_alloc(ctx, (void**)&cu, cap * 4, &t->bytes);
    if (rc) {
        if (cs) dev_free(ctx, cs, cap * 4);
        return rc;
    }
    dev_free(ctx, t->cstart, t->table_cap * 4);
    dev_free(ctx, t->cursor, t->table_cap * 4);
    t->cstart = cs;
    t->cursor = cu;
    t->table_cap = cap;
    const size_t need = grid_temp_bytes(std::max<uint64_t>(cap, t->cols_cap + 1));
    if (need > t->grid_tmp_bytes) {
        void* tmp = nullptr;
        rc = dev_alloc(ctx, &tmp, need, &t->bytes);
        if (rc) return rc;
        dev_free(ctx, t->grid_tmp, t->grid_tmp_bytes);
        t->grid_tmp = tmp;
        t->grid_tmp_bytes = need;
    }
    return NBG_OK;
}

static int ndims_of(const nbg_stage_opts& o) {
    switch (o.kind) {
        case NBG_STAGE_NORMAL: return 4;
        case NBG_STAGE_EIGENVALUES: return 3;
        case NBG_STAGE_COVARIANCEFEATURES: return __builtin_popcount(o.feature_mask & NBG_FEAT_ALL);
        case NBG_STAGE_OPTIMALNEIGHBORHOOD: return 2;
        case NBG_STAGE_LOF: return 3;
        default: return 1;
    }
}

}  // namespace nbg

using namespace nbg;

extern "C" {

const char* nbg_version(void) { return "nbg-b200 0.1 sm_100a"; }

int nbg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int good = 0;
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++good;
    }
    return good;
}

int nbg_create(nbg_context** out, int device, uint64_t hbm_budget_bytes) {
    if (!out) return NBG_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return NBG_ERR_NO_DEVICE;
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess || p.major != 10) return NBG_ERR_NO_DEVICE;
    nbg_context* h = new (std::nothrow) nbg_context();
    if (!h) return NBG_ERR_OOM;
    Context* ctx = &h->c;
    ctx->device = device;
    ctx->sm_count = p.multiProcessorCount;
    ctx->budget = hbm_budget_bytes;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete h;
        return NBG_ERR_CUDA;
    }
    for (int i = 0; i < 10; ++i) cudaEventCreate(&ctx->ev[i]);
    for (int i = 0; i < 2; ++i) cudaEventCreateWithFlags(&ctx->xev[i], cudaEventDisableTiming);
    ctx->events = true;
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    if (cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, hi_prio) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->fork, cudaStreamNonBlocking, lo_prio) != cudaSuccess) {
        if (ctx->side) cudaStreamDestroy(ctx->side);
        delete h;
        return NBG_ERR_CUDA;
    }
    for (int i = 0; i < 4; ++i) cudaEventCreateWithFlags(&ctx->fev[i], cudaEventDisableTiming);
    if (dev_alloc(ctx, (void**)&ctx->counters, 64 * sizeof(uint32_t), nullptr)) {
        delete h;
        return NBG_ERR_OOM;
    }
    *out = h;
    return NBG_OK;
}

int nbg_destroy(nbg_context* h) {
    if (!h) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    cudaSetDevice(ctx->device);
    dev_free(ctx, ctx->exact_rows, ctx->exact_cap * 4);
    if (ctx->retry_rows) dev_free(ctx, ctx->retry_rows, ctx->retry_cap * 4);
    if (ctx->ties) dev_free(ctx, ctx->ties, ctx->tie_cap * sizeof(uint2));
    if (ctx->sums) dev_free(ctx, ctx->sums, ctx->sums_cap * sizeof(RowSums));
    dev_free(ctx, ctx->ex_rows, ctx->ex_cap * sizeof(nbg_row_exception));
    dev_free(ctx, ctx->counters, 64 * sizeof(uint32_t));
    ctx_trim(ctx);
    if (ctx->events) {
        for (int i = 0; i < 10; ++i) cudaEventDestroy(ctx->ev[i]);
        for (int i = 0; i < 2; ++i) cudaEventDestroy(ctx->xev[i]);
    }
    batch_release(ctx);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->fork) {
        cudaStreamDestroy(ctx->fork);
        for (int i = 0; i < 4; ++i) cudaEventDestroy(ctx->fev[i]);
    }
    if (ctx->bounce_ready) {
        for (int i = 0; i < 2; ++i) {
            cudaFreeHost(ctx->bounce[i]);
            cudaEventDestroy(ctx->bev[i]);
        }
    }
    delete h;
    return NBG_OK;
}

const char* nbg_last_error(const nbg_context* h) {
    if (!h) return "no context";
    std::lock_guard<std::mutex> lock(const_cast<nbg_context*>(h)->c.emu);
    return h->c.err.c_str();
}

uint64_t nbg_tile_size(const nbg_tile* t) { return t ? t->t.n : 0; }

int nbg_tile_upload(nbg_context* h, const int32_t* x, const int32_t* y, const int32_t* z,
                    uint64_t n, const double scale[3], const double offset[3], int32_t on_device,
                    void* stream_v, nbg_tile** out) {
    NBG_RANGE("nbg tile upload");
    if (!h || !out) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    *out = nullptr;
    if (n > 0 && (!x || !y || !z)) return fail(ctx, NBG_ERR_INVALID, "null coordinate array");
    nbg_tile* th = nullptr;
    int rc = tile_alloc(ctx, n, scale, offset, &th);
    if (rc) return rc;
    Tile* t = &th->t;
    cudaStream_t stream = (cudaStream_t)stream_v;
    if (n) {
        int urc = NBG_OK;
        if (on_device) {
            cudaError_t e = cudaMemcpyAsync(t->x, x, n * 4, cudaMemcpyDeviceToDevice, stream);
            if (!e) e = cudaMemcpyAsync(t->y, y, n * 4, cudaMemcpyDeviceToDevice, stream);
            if (!e) e = cudaMemcpyAsync(t->z, z, n * 4, cudaMemcpyDeviceToDevice, stream);
            if (e) urc = cuda_fail(ctx, e, "coordinate upload");
        } else {
            urc = host_to_device(ctx, t->x, x, n * 4, stream);
            if (!urc) urc = host_to_device(ctx, t->y, y, n * 4, stream);
            if (!urc) urc = host_to_device(ctx, t->z, z, n * 4, stream);
        }
        if (urc) {
            tile_release(ctx, t);
            delete th;
            return urc;
        }
    }
    *out = th;
    return NBG_OK;
}

}  // extern "C"

namespace nbg {

// A tile of n points with its device storage, coordinates not yet filled.
int tile_alloc(Context* ctx, uint64_t n, const double scale[3], const double offset[3],
               nbg_tile** out) {
    *out = nullptr;
    if (n >= 0x7FFFFFF0ull) return fail(ctx, NBG_ERR_UNSUPPORTED, "tile larger than 2^31 points");
    if (!scale || !offset) return fail(ctx, NBG_ERR_INVALID, "null scale/offset");
    for (int d = 0; d < 3; ++d)
        if (!(scale[d] > 0.0) || !std::isfinite(scale[d]) || !std::isfinite(offset[d]))
            return fail(ctx, NBG_ERR_INVALID, "scale must be positive and finite");
    if (scale[0] != scale[1] || scale[0] != scale[2])
        return fail(ctx, NBG_ERR_UNSUPPORTED,
                    "the integer distance order needs one scale for x, y and z");
    cudaSetDevice(ctx->device);
    nbg_tile* th = new (std::nothrow) nbg_tile();
    if (!th) return NBG_ERR_OOM;
    Tile* t = &th->t;
    t->n = n;
    for (int d = 0; d < 3; ++d) {
        t->tf.scale[d] = scale[d];
        t->tf.offset[d] = offset[d];
    }
    t->cols_cap = std::max<uint64_t>(2 * n + 1024, 1u << 20);
    t->table_cap = 4 * n + 1024;
    int rc = NBG_OK;
#define ALLOC(PTR_, NBYTES_) \
    if (!rc) rc = dev_alloc(ctx, (void**)&(PTR_), (NBYTES_), &t->bytes);
    ALLOC(t->x, n * 4);
    ALLOC(t->y, n * 4);
    ALLOC(t->z, n * 4);
    ALLOC(t->bbox, 64);
    ALLOC(t->gp, sizeof(GridParams));
    ALLOC(t->colinfo, t->cols_cap * 16);
    ALLOC(t->ext, (t->cols_cap + 1) * 4);
    ALLOC(t->table_dev, 16);
    ALLOC(t->keys, n * 4);
    ALLOC(t->cstart, t->table_cap * 4);
    ALLOC(t->cursor, t->table_cap * 4);
    ALLOC(t->sorted, n * 16);
    t->grid_tmp_bytes = grid_temp_bytes(std::max<uint64_t>(t->table_cap, t->cols_cap + 1));
    ALLOC(t->grid_tmp, t->grid_tmp_bytes);
#undef ALLOC
    if (rc) {
        tile_release(ctx, t);
        delete th;
        return rc;
    }
    *out = th;
    return NBG_OK;
}

void tile_destroy(Context* ctx, nbg_tile* th) {
    tile_release(ctx, &th->t);
    delete th;
}

}  // namespace nbg

extern "C" {

int nbg_tile_tune(nbg_context* h, nbg_tile* th, float cell_factor, int32_t fixed_cell) {
    if (!h || !th) return NBG_ERR_INVALID;
    if (!(cell_factor > 0.0f) || cell_factor > 64.0f || fixed_cell < 0)
        return fail(&h->c, NBG_ERR_INVALID, "cell_factor must be in (0, 64], fixed_cell >= 0");
    std::lock_guard<std::mutex> lock(h->c.mu);
    th->t.cell_factor = cell_factor;
    th->t.fixed_cell = fixed_cell;
    th->t.grid_valid = false;
    th->t.tuning_set = true;
    return NBG_OK;
}

static bool valid_select(int32_t k) {
    return k == 0 || k == 1 || k == 2 || k == 8 || k == 16 || k == 32;
}

extern "C" int nbg_tile_set_select(nbg_context* h, nbg_tile* th, int32_t select_kernel,
                                   float first_margin) {
    if (!h || !th) return NBG_ERR_INVALID;
    if (!valid_select(select_kernel))
        return fail(&h->c, NBG_ERR_INVALID, "select kernel must be 0, 1, 2, 8, 16 or 32");
    if (!(first_margin > 0.0f && first_margin <= 16.0f))
        return fail(&h->c, NBG_ERR_INVALID, "first margin must be in (0, 16] cell edges");
    std::lock_guard<std::mutex> lock(h->c.mu);
    th->t.group = select_kernel;
    th->t.margin0 = first_margin;
    th->t.tuning_set = true;
    return NBG_OK;
}

int nbg_tile_free(nbg_context* h, nbg_tile* th) {
    if (!h || !th) return NBG_ERR_INVALID;
    std::lock_guard<std::mutex> lock(h->c.mu);
    cudaSetDevice(h->c.device);
    tile_release(&h->c, &th->t);
    delete th;
    return NBG_OK;
}

}  // extern "C"

namespace nbg {

// Grid for neighbour count k1 (rebuilt when k1 moves far from the build's).
// Grid for neighbour count k1, or with a fixed cell edge `cell` raw units
// (radius stages); rebuilt when k1 moves far from the build's or the edge rule
// changes.
int ensure_grid(Context* ctx, Tile* t, int k1, cudaStream_t stream, int32_t cell) {
    NBG_RANGE("nbg grid build");
    const int32_t fixed = cell ? cell : t->fixed_cell;
    if (t->grid_valid && t->grid_fixed == fixed &&
        (fixed || (k1 <= 2 * t->grid_k1 && 2 * k1 >= t->grid_k1)))
        return NBG_OK;
    const int32_t saved = t->fixed_cell;
    t->fixed_cell = fixed;
    int rc = build_grid(ctx, t, k1, stream);
    t->fixed_cell = saved;
    if (rc) return fail(ctx, rc, "grid build failed");
    NBG_TRY(cudaMemcpyAsync(&t->host_gp, t->gp, sizeof(GridParams), cudaMemcpyDeviceToHost, stream),
            "grid params");
    NBG_TRY(cudaStreamSynchronize(stream), "grid build");
    const GridParams& g = t->host_gp;
    if ((int64_t)g.maxx - g.minx >= (1 << 24) || (int64_t)g.maxy - g.miny >= (1 << 24) ||
        (int64_t)g.maxz - g.minz >= (1 << 24))
        return fail(ctx, NBG_ERR_UNSUPPORTED, "tile extent must be below 2^24 raw units per axis");
    t->grid_valid = true;
    t->grid_k1 = k1;
    t->grid_fixed = fixed;
    return NBG_OK;
}

int validate_stages(Context* ctx, const nbg_stage_opts* stages, int n_stages,
                    const nbg_columns* outputs, bool* need_aux) {
    *need_aux = false;
    for (int s = 0; s < n_stages; ++s) {
        const nbg_stage_opts& o = stages[s];
        if (o.kind < 1 || o.kind > NBG_STAGE_OUTLIER)
            return fail(ctx, NBG_ERR_INVALID, "unknown stage kind");
        if (o.knn < 0 || o.knn > 64)
            return fail(ctx, NBG_ERR_INVALID, "knn must be in [0, 64]");
        if (o.kind > NBG_STAGE_COVARIANCEFEATURES) {
            // the other kNN consumers: their own options only
            if (outputs[s].ndims != ndims_of(o))
                return fail(ctx, NBG_ERR_INVALID, "output ndims does not match the stage");
            if ((o.kind == NBG_STAGE_APPROXIMATECOPLANAR || o.kind == NBG_STAGE_ESTIMATERANK) &&
                o.knn < 1)
                return fail(ctx, NBG_ERR_UNSUPPORTED,
                            "knn 0 reads before the search's result buffer in the reference");
            if (o.kind == NBG_STAGE_OPTIMALNEIGHBORHOOD && (o.min_k < 1 || o.min_k > o.knn))
                return fail(ctx, NBG_ERR_INVALID, "optimalneighborhood needs 1 <= min_k <= max_k");
            if ((o.kind == NBG_STAGE_NNDISTANCE && (o.mode < 0 || o.mode > 1)) ||
                (o.kind == NBG_STAGE_OUTLIER && (o.mode < 0 || o.mode > 2)))
                return fail(ctx, NBG_ERR_INVALID, "invalid mode");
            if (o.kind == NBG_STAGE_OUTLIER && o.mode == 1 && !(std::fabs(o.radius) < 1e300))
                return fail(ctx, NBG_ERR_INVALID, "radius is not a finite number");
            continue;
        }
        // a radius makes the reference ignore knn and stride
        // (EigenvaluesFilter.cpp:96-100, CovarianceFeaturesFilter.cpp:216-225)
        const bool by_radius = o.use_radius && !(o.kind == NBG_STAGE_COVARIANCEFEATURES && o.optimized);
        if (!by_radius && o.kind != NBG_STAGE_NORMAL && o.stride > 1 && !o.optimized &&
            (int64_t)o.stride * (o.knn + 1) > 65)
            return fail(ctx, NBG_ERR_UNSUPPORTED, "stride * (knn + 1) above 65 is not supported");
        if (o.stride < 0) return fail(ctx, NBG_ERR_INVALID, "stride must be positive");
        if (by_radius && !(o.radius == o.radius))
            return fail(ctx, NBG_ERR_INVALID, "radius is not a number");
        if (o.kind != NBG_STAGE_COVARIANCEFEATURES && o.optimized)
            return fail(ctx, NBG_ERR_INVALID, "optimized applies to covariancefeatures only");
        if (o.kind == NBG_STAGE_COVARIANCEFEATURES &&
            (o.mode < NBG_MODE_RAW || o.mode > NBG_MODE_NORMALIZED))
            return fail(ctx, NBG_ERR_INVALID, "invalid mode");
        if (outputs[s].ndims != ndims_of(o))
            return fail(ctx, NBG_ERR_INVALID, "output ndims does not match the stage");
        if (o.kind == NBG_STAGE_COVARIANCEFEATURES &&
            ((o.feature_mask & NBG_FEAT_DENSITY) || o.optimized))
            *need_aux = true;
    }
    return NBG_OK;
}

void fill_stage(StageDev& d, const nbg_stage_opts& o, const nbg_columns& c) {
    d.kind = o.kind;
    d.always_up = o.always_up;
    d.has_viewpoint = o.has_viewpoint;
    d.normalize = o.normalize;
    for (int k = 0; k < 3; ++k) d.viewpoint[k] = o.viewpoint[k];
    d.feature_mask = o.feature_mask & NBG_FEAT_ALL;
    d.mode = o.mode;
    d.ip = o.min_k;
    d.t1 = o.thresh1;
    d.t2 = o.thresh2;
    d.aux = nullptr;
    d.ndims = c.ndims;
    d.base = (char*)c.base;
    d.point_stride = c.point_stride;
    for (int k = 0; k < NBG_MAX_DIMS; ++k) d.offset[k] = c.offset[k];
}

__global__ void optimal_k_max_kernel(const double* k, uint64_t n, unsigned long long* out) {
    double mx = 0.0;
    int bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double v = k[i];
        if (!(v > -0.5) || !(v < 1.8446744073709552e19)) bad = 1;
        else mx = fmax(mx, v);
    }
    // non-negative doubles order as their bit patterns
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(mx));
    if (bad) atomicOr(&out[1], 1ull);
}

// Largest OptimalKNN of a column (host or device); `bad` when a value is
// negative, NaN or beyond uint64 (the reference's numericCast would fail).
int optimal_k_max(Context* ctx, const double* k, uint64_t n, bool on_device, cudaStream_t stream,
                  double* mx, bool* bad) {
    *mx = 0.0;
    *bad = false;
    if (!on_device) {
        for (uint64_t i = 0; i < n; ++i) {
            const double v = k[i];
            if (!(v > -0.5) || !(v < 1.8446744073709552e19)) *bad = true;
            else if (v > *mx) *mx = v;
        }
        return NBG_OK;
    }
    unsigned long long* d = nullptr;
    int rc = ctx_alloc(ctx, (void**)&d, 16);
    if (rc) return rc;
    unsigned long long h[2] = {0, 0};
    cudaMemsetAsync(d, 0, 16, stream);
    optimal_k_max_kernel<<<(unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 1024)), 256, 0,
                           stream>>>(k, n, d);
    NBG_LAUNCHED(1);
    cudaError_t e = cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    ctx_free(ctx, d, 16);
    if (e) return cuda_fail(ctx, e, "OptimalKNN scan");
    *mx = __builtin_bit_cast(double, (long long)h[0]);
    *bad = h[1] != 0;
    return NBG_OK;
}

struct HostOut {
    const nbg_columns* user;
    char* dev = nullptr;  // device staging (host outputs only)
    size_t bytes = 0;
};

// Host records of a plain kNN group copied back while the rows are still
// being answered.  The rows are taken in `C` chunks of the point-id range
// (each chunk's sorted positions in cell order).  Every chunk's select +
// finish is queued on `stream` at once; the KD replica builds on the side
// stream beside them (its build waits on the host, which has nothing else to
// queue), and then, chunk by chunk as each one's queries complete, the side
// stream orders and replays its tie rows and a copy stream copies its
// records -- one contiguous byte range of the caller's pinned buffer -- back
// while the later chunks are still being answered.  Every chunk has its own
// counters, tie list and replay list (disjoint slices of the context's), so
// chunks share no mutable state; the outputs equal the unchunked path's bit
// for bit.
struct PipeStats {
    float query_ms = 0, tree_ms = 0, build_ms = 0;
    uint64_t tie_rows = 0, deferred_rows = 0, replay_rows = 0, retry_rows = 0;
};

static int run_pipelined(Context* ctx, Tile* t, int K, const StageGroup& g, const ExceptionSink& sink,
                         const char* dev_records, char* host_records, size_t record_bytes, int C,
                         cudaStream_t stream, PipeStats& ps) {
    NBG_RANGE("nbg pipelined query");
    const uint64_t n = t->n;
    // chunk c counts in counters[8c .. 8c+4]: at most four chunks stay below
    // the word build_id_chunks writes (counters[48])
    if (C < 1 || C > 4) return fail(ctx, NBG_ERR_INVALID, "pipeline chunk count");
    // four chunks of 30, 30, 25 and 15 % of the id range: the copy of the last
    // chunk is the only one left after the queries end, so it is the smallest
    // (the earlier, larger copies still finish while later chunks run)
    static const uint64_t w4[5] = {0, 300, 600, 850, 1000};
    uint64_t b[9];
    for (int c = 0; c <= C; ++c)
        b[c] = C == 4 ? n * w4[c] / 1000 : n * (uint64_t)c / (uint64_t)C;
    uint32_t* rows = nullptr;
    int rc = ctx_alloc(ctx, (void**)&rows, n * 4);
    if (rc) return rc;
    cudaStream_t cs = nullptr;
    cudaEvent_t sel[8] = {}, t0[8] = {}, t1[8] = {}, done = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int c = 0; c < C && !e; ++c) {
        e = cudaEventCreate(&sel[c]);
        if (!e) e = cudaEventCreate(&t0[c]);
        if (!e) e = cudaEventCreate(&t1[c]);
    }
    if (!e) e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    if (e) rc = fail(ctx, NBG_ERR_CUDA, std::string("pipeline setup: ") + cudaGetErrorString(e));
    if (!rc) rc = build_id_chunks(ctx, t, b, C, rows, ctx->counters + 48, stream);
    const bool speculative = !(t->kd && kd_built(t));
    auto finish_chunk = [&](int c) -> int {
        const uint32_t rows_c = (uint32_t)(b[c + 1] - b[c]);
        uint32_t* cnt_dev = ctx->counters + 8 * c;
        uint32_t cnt[7] = {0, 0, 0, 0, 0, 0, 0};
        cudaError_t e = cudaStreamWaitEvent(ctx->side, sel[c], 0);
        if (!e) e = cudaMemcpyAsync(cnt, cnt_dev, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->side);
        if (!e) e = cudaStreamSynchronize(ctx->side);
        if (e) return fail(ctx, NBG_ERR_CUDA, std::string("query kernel: ") + cudaGetErrorString(e));
        ps.tie_rows += cnt[1];
        ps.deferred_rows += cnt[2];
        ps.retry_rows += cnt[6];
        cudaEventRecord(t0[c], ctx->side);
        const uint32_t nties = std::min(cnt[4], rows_c);
        if (nties) {
            TieLaunch tl;
            tl.tile = t;
            tl.K = K;
            tl.grp = g;
            tl.ex = sink;
            tl.ties = ctx->ties + b[c];
            tl.nties = nties;
            tl.kd = kd_order(t);
            tl.exact_rows = ctx->exact_rows + b[c];
            tl.counters = cnt_dev;
            tl.ids_out = nullptr;
            tl.row_k = nullptr;
            int r = launch_ties(ctx, tl, ctx->side);
            if (r) return fail(ctx, r, "tie-order resolver launch failed");
            e = cudaMemcpyAsync(cnt, cnt_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->side);
            if (!e) e = cudaStreamSynchronize(ctx->side);
            if (e) return fail(ctx, NBG_ERR_CUDA, std::string("tie-order resolver: ") + cudaGetErrorString(e));
        }
        ps.replay_rows += cnt[0];
        int r = kd_run_rows(ctx, t, K, g, sink, ctx->exact_rows + b[c], cnt[0], ctx->side, nullptr);
        if (r) return r;
        cudaEventRecord(t1[c], ctx->side);
        e = cudaStreamWaitEvent(cs, t1[c], 0);
        if (!e) e = cudaMemcpyAsync(host_records + b[c] * record_bytes, dev_records + b[c] * record_bytes,
                                    rows_c * record_bytes, cudaMemcpyDeviceToHost, cs);
        if (e) return fail(ctx, NBG_ERR_CUDA, std::string("output copy: ") + cudaGetErrorString(e));
        return NBG_OK;
    };
    int launched = 0;
    if (!rc && speculative) {
        cudaEventRecord(ctx->xev[0], stream);
        cudaStreamWaitEvent(ctx->side, ctx->xev[0], 0);
    }
    for (int c = 0; c < C && !rc; ++c) {
        QueryLaunch ql;
        ql.tile = t;
        ql.K = K;
        ql.rmax = 8;
        ql.grp = g;
        ql.ex = sink;
        ql.exact_rows = ctx->exact_rows + b[c];
        ql.counters = ctx->counters + 8 * c;
        ql.ties = ctx->ties + b[c];
        ql.tie_cap = (uint32_t)(b[c + 1] - b[c]);
        ql.sums = ctx->sums;
        ql.row_k = nullptr;
        ql.rows = rows + b[c];
        ql.nrows = b[c + 1] - b[c];
        ql.retry_rows = ctx->retry_rows + b[c];
        ql.group = t->group;
        ql.margin0 = t->margin0;
        // sel[c] marks the chunk's rows answered; the next chunk's select may
        // start while this chunk's handed-back rows still run
        ql.done = sel[c];
        rc = launch_query(ctx, ql, stream);
        if (rc) {
            rc = fail(ctx, rc, std::string("query launch failed: ") + cudaGetErrorString(cudaGetLastError()));
            break;
        }
        ++launched;
    }
    if (!rc && speculative) {
        // the KD replica (needed by the tie rows) builds beside the queries
        cudaEventRecord(ctx->ev[8], ctx->side);
        rc = kd_ensure(ctx, t, ctx->side);  // uncapped: the first chunk's tie rows wait for it
        cudaEventRecord(ctx->ev[9], ctx->side);
    }
    for (int c = 0; c < launched && !rc; ++c) rc = finish_chunk(c);
    // every queued kernel and copy completes before the buffers are released
    if (cs && done) {
        cudaEventRecord(done, cs);
        cudaStreamWaitEvent(stream, done, 0);
    }
    e = cudaStreamSynchronize(stream);
    if (cs && !e) e = cudaStreamSynchronize(cs);
    if (ctx->fork && !e) e = cudaStreamSynchronize(ctx->fork);
    cudaError_t e2 = cudaStreamSynchronize(ctx->side);
    if (!rc && (e || e2))
        rc = fail(ctx, NBG_ERR_CUDA, std::string("pipelined query: ") + cudaGetErrorString(e ? e : e2));
    if (!rc) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ctx->ev[2], sel[C - 1]) == cudaSuccess) ps.query_ms += ms;
        for (int c = 0; c < C; ++c)
            if (cudaEventElapsedTime(&ms, t0[c], t1[c]) == cudaSuccess) ps.tree_ms += ms;
        if (speculative && cudaEventElapsedTime(&ms, ctx->ev[8], ctx->ev[9]) == cudaSuccess) ps.build_ms += ms;
    }
    for (int c = 0; c < C; ++c) {
        if (sel[c]) cudaEventDestroy(sel[c]);
        if (t0[c]) cudaEventDestroy(t0[c]);
        if (t1[c]) cudaEventDestroy(t1[c]);
    }
    if (done) cudaEventDestroy(done);
    if (cs) cudaStreamDestroy(cs);
    ctx_free(ctx, rows, n * 4);
    return rc;
}

}  // namespace nbg

extern "C" int nbg_run(nbg_context* h, nbg_tile* th, const nbg_stage_opts* stages,
                       int32_t n_stages, const nbg_columns* outputs, const double* optimal_knn,
                       const double* optimal_radius, int32_t aux_on_device,
                       nbg_row_exception* exceptions, uint32_t exception_capacity,
                       uint32_t* n_exceptions, nbg_run_stats* stats, void* stream_v) {
    NBG_RANGE("nbg_run");
    if (!h || !th) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    Tile* t = &th->t;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t stream = (cudaStream_t)stream_v;
    if (n_exceptions) *n_exceptions = 0;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const uint64_t launches0 = g_launches.load();
    if (n_stages < 0 || n_stages > NBG_MAX_STAGES || (n_stages && (!stages || !outputs)))
        return fail(ctx, NBG_ERR_INVALID, "bad stage array");
    bool need_aux = false;
    int vrc = validate_stages(ctx, stages, n_stages, outputs, &need_aux);
    if (vrc) return vrc;
    bool need_radius = false, any_optimized = false;
    for (int s = 0; s < n_stages; ++s) {
        if (stages[s].kind == NBG_STAGE_COVARIANCEFEATURES && (stages[s].feature_mask & NBG_FEAT_DENSITY))
            need_radius = true;
        if (stages[s].optimized) any_optimized = true;
    }
    if (need_radius && (!optimal_knn || !optimal_radius))
        return fail(ctx, NBG_ERR_INVALID, "Density needs OptimalKNN and OptimalRadius");
    if (any_optimized && !optimal_knn)
        return fail(ctx, NBG_ERR_INVALID, "optimized needs OptimalKNN");
    const uint64_t n = t->n;
    if (n == 0 || n_stages == 0) return NBG_OK;
    int rc = ensure_scratch(ctx, n, std::max<uint64_t>(exception_capacity, 1));
    if (rc) return rc;

    // host-side outputs: device staging in column layout, copied back after
    std::vector<HostOut> hout(n_stages);
    std::vector<nbg_columns> dcols(n_stages);
    double* aux_dev[2] = {nullptr, nullptr};
    char* packed_dev_c = nullptr;
    size_t packed_bytes_c = 0;
    auto cleanup = [&]() {
        // The blocks go back to the context's cache, where the next call may
        // take them: on an error return the fork stream (handed-back rows, tie
        // order) or the side stream (KD replica) can still be writing them.
        cudaStreamSynchronize(stream);
        cudaStreamSynchronize(ctx->fork);
        cudaStreamSynchronize(ctx->side);
        if (packed_dev_c) dev_free(ctx, packed_dev_c, packed_bytes_c);
        for (auto& o : hout)
            if (o.dev) dev_free(ctx, o.dev, o.bytes);
        if (!aux_on_device) {
            if (aux_dev[0]) dev_free(ctx, aux_dev[0], n * 8);
            if (aux_dev[1]) dev_free(ctx, aux_dev[1], n * 8);
        }
    };
    // Host outputs that form one packed record (every stage writes fresh
    // dims into the same base, and the record holds exactly those dims) are
    // staged on the device in the caller's own layout and copied back with a
    // single contiguous transfer.
    char* packed_dev = nullptr;
    size_t packed_bytes = 0;
    bool packed = n_stages > 0;
    {
        int total = 0;
        uint64_t seen = 0;
        for (int s = 0; s < n_stages && packed; ++s) {
            const nbg_columns& u = outputs[s];
            if (u.on_device != 2 || u.base != outputs[0].base ||
                u.point_stride != outputs[0].point_stride)
                packed = false;
            for (int d = 0; packed && d < u.ndims; ++d) {
                const int64_t off = u.offset[d];
                if (off < 0 || off % 8 || off / 8 >= 64 || (seen >> (off / 8) & 1)) packed = false;
                else seen |= 1ull << (off / 8);
            }
            total += u.ndims;
        }
        if (packed && (total == 0 || outputs[0].point_stride != 8 * total)) packed = false;
    }
    if (packed) {
        packed_bytes = n * (size_t)outputs[0].point_stride;
        rc = dev_alloc(ctx, (void**)&packed_dev, packed_bytes, nullptr);
        if (rc) return rc;
        packed_dev_c = packed_dev;
        packed_bytes_c = packed_bytes;
        cudaError_t e = cudaMemsetAsync(packed_dev, 0, packed_bytes, stream);
        if (e) { cleanup(); return cuda_fail(ctx, e, "output staging"); }
        for (int s = 0; s < n_stages; ++s) {
            hout[s].user = &outputs[s];
            dcols[s] = outputs[s];
            dcols[s].base = packed_dev;
            dcols[s].on_device = 1;
        }
    }
    for (int s = 0; s < n_stages && !packed; ++s) {
        hout[s].user = &outputs[s];
        dcols[s] = outputs[s];
        if (outputs[s].on_device != 1 && outputs[s].ndims > 0) {
            hout[s].bytes = n * 8 * outputs[s].ndims;
            rc = dev_alloc(ctx, (void**)&hout[s].dev, hout[s].bytes, nullptr);
            if (rc) { cleanup(); return rc; }
            dcols[s].base = hout[s].dev;
            dcols[s].point_stride = 8;
            dcols[s].on_device = 1;
            for (int d = 0; d < outputs[s].ndims; ++d) dcols[s].offset[d] = (int64_t)d * n * 8;
            if (outputs[s].on_device == 2) {
                // fresh dimensions: skipped rows read 0, as in a new PDAL table
                cudaError_t e = cudaMemsetAsync(hout[s].dev, 0, hout[s].bytes, stream);
                if (e) { cleanup(); return cuda_fail(ctx, e, "output staging"); }
                continue;
            }
            // rows the reference skips keep the caller's values
            for (int d = 0; d < outputs[s].ndims; ++d) {
                const nbg_columns& u = outputs[s];
                if (u.point_stride == 8) {
                    rc = host_to_device(ctx, hout[s].dev + (size_t)d * n * 8,
                                        (char*)u.base + u.offset[d], n * 8, stream);
                    if (rc) { cleanup(); return rc; }
                    continue;
                }
                cudaError_t e = cudaMemcpy2DAsync(hout[s].dev + (size_t)d * n * 8, 8,
                                                  (char*)u.base + u.offset[d], u.point_stride, 8, n,
                                                  cudaMemcpyHostToDevice, stream);
                if (e) { cleanup(); return cuda_fail(ctx, e, "output staging"); }
            }
        }
    }
    const double* kopt = optimal_knn;
    const double* ropt = optimal_radius;
    // largest per-point k of the optimized stages (sizes their launch)
    int opt_k = 0;
    if (any_optimized) {
        double mx = 0.0;
        bool bad = false;
        rc = optimal_k_max(ctx, optimal_knn, n, aux_on_device != 0, stream, &mx, &bad);
        if (rc) { cleanup(); return rc; }
        if (bad) {
            cleanup();
            return fail(ctx, NBG_ERR_INVALID, "OptimalKNN holds a value that is not a neighbour count");
        }
        opt_k = (int)std::min<double>((double)n, std::floor(mx + 0.5));
        if (opt_k > 65) {
            cleanup();
            return fail(ctx, NBG_ERR_UNSUPPORTED, "OptimalKNN above 65 is not supported");
        }
    }
    if (need_aux && !aux_on_device) {
        rc = dev_alloc(ctx, (void**)&aux_dev[0], n * 8, nullptr);
        if (!rc && optimal_radius) rc = dev_alloc(ctx, (void**)&aux_dev[1], n * 8, nullptr);
        if (rc) { cleanup(); return rc; }
        rc = host_to_device(ctx, aux_dev[0], optimal_knn, n * 8, stream);
        if (!rc && optimal_radius) rc = host_to_device(ctx, aux_dev[1], optimal_radius, n * 8, stream);
        if (rc) { cleanup(); return rc; }
        kopt = aux_dev[0];
        ropt = optimal_radius ? aux_dev[1] : nullptr;
    }

    // group stages by neighbour count
    std::vector<int> order(n_stages);
    for (int s = 0; s < n_stages; ++s) order[s] = s;
    // neighbour count of a stage's launch: knn + 1 (capped at n), or the
    // largest OptimalKNN for optimized stages (their rows then use their own)
    auto stage_k = [&](int s) -> int {
        if (stages[s].optimized) return std::max(1, opt_k);
        // approximatecoplanar / estimaterank query knn points, the point included
        const int extra = (stages[s].kind == NBG_STAGE_APPROXIMATECOPLANAR ||
                           stages[s].kind == NBG_STAGE_ESTIMATERANK) ? 0 : 1;
        return (int)std::min<uint64_t>(n, (uint64_t)stages[s].knn + extra);
    };
    auto by_radius = [&](int s) {
        return stages[s].use_radius && stages[s].kind <= NBG_STAGE_COVARIANCEFEATURES &&
               !(stages[s].kind == NBG_STAGE_COVARIANCEFEATURES && stages[s].optimized);
    };
    // strided stages (eigenvalues / covariancefeatures; normal has no stride)
    auto strided = [&](int s) {
        return !by_radius(s) && (stages[s].kind == NBG_STAGE_EIGENVALUES ||
                                 stages[s].kind == NBG_STAGE_COVARIANCEFEATURES) &&
               stages[s].stride > 1 && !stages[s].optimized;
    };
    std::vector<std::vector<int>> groups;
    std::vector<int> consumers;  // list / outlier stages: run_consumer
    for (int s = 0; s < n_stages; ++s) {
        if (is_list_consumer(stages[s].kind)) {
            consumers.push_back(s);
            continue;
        }
        bool placed = false;
        for (auto& gr : groups) {
            // radius and strided stages run alone
            if (by_radius(gr[0]) || by_radius(s) || strided(gr[0]) || strided(s)) continue;
            if (stage_k(gr[0]) == stage_k(s) && !stages[gr[0]].optimized == !stages[s].optimized) {
                gr.push_back(s);
                placed = true;
                break;
            }
        }
        if (!placed) groups.push_back({s});
    }

    // pinned host records of one plain kNN group on a large tile: copied back
    // chunk by chunk while the later chunks are answered (run_pipelined)
    const bool pipelined = packed && host_pinned(outputs[0].base) && groups.size() == 1 &&
                           consumers.empty() && n >= (1ull << 22) && !by_radius(groups[0][0]) &&
                           !strided(groups[0][0]) && !stages[groups[0][0]].optimized;
    const int pipe_chunks = n >= (8ull << 20) ? 4 : 2;
    bool packed_copied = false;
    cudaEventRecord(ctx->ev[0], stream);
    float grid_ms = 0, query_ms = 0, tree_ms = 0;
    uint64_t tie_rows = 0, deferred_rows = 0, replay_rows = 0, retry_rows = 0;
    float build_ms = 0;
    ExceptionSink sink{ctx->ex_rows, ctx->counters + 3, (uint32_t)std::max<uint32_t>(exception_capacity, 1)};
    if (cudaMemsetAsync(ctx->counters, 0, 64 * sizeof(uint32_t), stream)) { cleanup(); return NBG_ERR_CUDA; }
    for (auto& gr : groups) {
        const int K = stage_k(gr[0]);
        const double* row_k = stages[gr[0]].optimized ? kopt : nullptr;
        const bool radius_group = by_radius(gr[0]);
        int32_t radius_cell = 0;
        if (radius_group) {
            // cells one radius wide (plus a margin): the ball fits in one ring
            const double r_raw = std::fabs(stages[gr[0]].radius) / t->tf.scale[0];
            radius_cell = (int32_t)std::min(1.0e9, std::ceil(r_raw * 1.001) + 1.0);
        }
        if (!radius_group) apply_cached_tuning(ctx, t, K);
        cudaEventRecord(ctx->ev[1], stream);
        rc = ensure_grid(ctx, t, K, stream, radius_cell);
        if (rc) { cleanup(); return rc; }
        cudaEventRecord(ctx->ev[2], stream);
        StageGroup g{};
        g.nstages = (int)gr.size();
        g.optimal_knn = kopt;
        g.optimal_radius = ropt;
        for (int i = 0; i < g.nstages; ++i) {
            const int s = gr[i];
            const nbg_stage_opts& o = stages[s];
            g.stage_index[i] = s;
            fill_stage(g.st[i], o, dcols[s]);
            if ((o.kind == NBG_STAGE_NORMAL && !o.always_up && !o.has_viewpoint) || o.eigen_fp64)
                g.sign_exact = 1;
        }
        g.resolve_count = ctx->counters + 5;
        if (cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(uint32_t), stream) ||
            cudaMemsetAsync(ctx->counters + 4, 0, sizeof(uint32_t), stream)) {
            cleanup();
            return NBG_ERR_CUDA;
        }
        if (strided(gr[0])) {
            const int stride = stages[gr[0]].stride;
            const int kpick = K;  // min(n, knn + 1)
            const int K2 = kpick * stride;
            rc = kd_ensure(ctx, t, stream);
            if (rc) { cleanup(); return rc; }
            QueryLaunch ql;
            ql.tile = t;
            ql.K = K2;
            ql.rmax = 8;
            ql.grp = g;
            ql.ex = sink;
            ql.exact_rows = ctx->exact_rows;
            ql.counters = ctx->counters;
            rc = launch_stride(ctx, ql, stride, kpick, kd_order(t), stream);
            if (rc) { cleanup(); return fail(ctx, rc, "stride launch failed"); }
            cudaEventRecord(ctx->ev[3], stream);
            uint32_t cnt[3] = {0, 0, 0};
            cudaError_t e = cudaMemcpyAsync(cnt, ctx->counters, sizeof(cnt), cudaMemcpyDeviceToHost,
                                            stream);
            if (!e) e = cudaStreamSynchronize(stream);
            if (e) { cleanup(); return cuda_fail(ctx, e, "stride kernel"); }
            tie_rows += cnt[1];
            deferred_rows += cnt[2];
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
            grid_ms += ms;
            cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
            query_ms += ms;
            if (cnt[0]) {
                replay_rows += cnt[0];
                rc = kd_run_rows(ctx, t, K2, g, sink, ctx->exact_rows, cnt[0], stream, nullptr,
                                 stride, kpick);
                if (rc) { cleanup(); return rc; }
            }
            continue;
        }
        if (radius_group) {
            RadiusLaunch rl;
            rl.tile = t;
            rl.grp = g;
            rl.ex = sink;
            rl.radius = stages[gr[0]].radius;
            rl.min_k = stages[gr[0]].min_k;
            rc = launch_radius(ctx, rl, stream);
            if (rc) { cleanup(); return fail(ctx, rc, "radius launch failed"); }
            cudaEventRecord(ctx->ev[3], stream);
            cudaError_t e = cudaStreamSynchronize(stream);
            if (e) { cleanup(); return cuda_fail(ctx, e, "radius kernel"); }
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
            grid_ms += ms;
            cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
            query_ms += ms;
            continue;
        }
        if (pipelined) {
            PipeStats ps;
            rc = run_pipelined(ctx, t, K, g, sink, packed_dev, (char*)outputs[0].base,
                               (size_t)outputs[0].point_stride, pipe_chunks, stream, ps);
            if (rc) { cleanup(); return rc; }
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
            grid_ms += ms;
            query_ms += ps.query_ms;
            tree_ms += ps.tree_ms;
            build_ms += ps.build_ms;
            tie_rows += ps.tie_rows;
            deferred_rows += ps.deferred_rows;
            replay_rows += ps.replay_rows;
            retry_rows += ps.retry_rows;
            packed_copied = true;
            continue;
        }
        QueryLaunch ql;
        ql.tile = t;
        ql.K = K;
        ql.rmax = 8;
        ql.grp = g;
        ql.ex = sink;
        ql.exact_rows = ctx->exact_rows;
        ql.counters = ctx->counters;
        ql.ties = ctx->ties;
        ql.tie_cap = (uint32_t)std::min<uint64_t>(ctx->tie_cap, UINT32_MAX);
        ql.sums = ctx->sums;
        ql.row_k = row_k;
        ql.retry_rows = ctx->retry_rows;
        ql.group = t->group;
        ql.margin0 = t->margin0;
        // the KD replica does not depend on the query: build it on the side
        // stream while the query kernel runs (tie rows almost always need it)
        const bool speculative = !(t->kd && kd_built(t)) && n > 100;
        if (speculative) {
            cudaEventRecord(ctx->xev[0], stream);
            cudaStreamWaitEvent(ctx->side, ctx->xev[0], 0);
        }
        rc = launch_query(ctx, ql, stream);
        if (rc) { cleanup(); return fail(ctx, rc, std::string("query launch failed: ") +
                                                 cudaGetErrorString(cudaGetLastError())); }
        cudaEventRecord(ctx->ev[3], stream);
        if (speculative) {
            cudaEventRecord(ctx->ev[8], ctx->side);
            rc = kd_ensure(ctx, t, ctx->side, true);
            if (rc) { cudaStreamSynchronize(stream); cleanup(); return rc; }
            cudaEventRecord(ctx->ev[9], ctx->side);
            cudaEventRecord(ctx->xev[1], ctx->side);
            cudaStreamWaitEvent(stream, ctx->xev[1], 0);
        }
        // With the single-pass select the tie list is complete once its
        // handed-back rows are answered on the fork stream: the tie rows are
        // ordered there (count read on the device) beside the finish pass
        // instead of after it.
        const bool ties_queued = query_forks(ctx, ql) && kd_built(t);
        if (ties_queued) {
            cudaError_t qe = speculative ? cudaStreamWaitEvent(ctx->fork, ctx->xev[1], 0) : cudaSuccess;
            if (!qe) qe = cudaEventRecord(ctx->ev[4], ctx->fork);
            TieLaunch tl;
            tl.tile = t;
            tl.K = K;
            tl.grp = g;
            tl.ex = sink;
            tl.ties = ctx->ties;
            tl.nties = ql.tie_cap;
            tl.kd = kd_order(t);
            tl.exact_rows = ctx->exact_rows;
            tl.counters = ctx->counters;
            tl.ids_out = nullptr;
            tl.row_k = row_k;
            rc = qe ? NBG_ERR_CUDA : launch_ties_counted(ctx, tl, ctx->counters + 4, ctx->fork);
            if (!rc && (cudaEventRecord(ctx->fev[3], ctx->fork) || cudaStreamWaitEvent(stream, ctx->fev[3], 0)))
                rc = NBG_ERR_CUDA;
            if (rc) {
                cudaStreamSynchronize(ctx->fork);
                cudaStreamSynchronize(stream);
                cleanup();
                return fail(ctx, rc, "tie-order resolver launch failed");
            }
        }
        uint32_t cnt[7] = {0, 0, 0, 0, 0, 0, 0};
        cudaError_t e = cudaMemcpyAsync(cnt, ctx->counters, 7 * sizeof(uint32_t),
                                        cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        if (e) { cleanup(); return cuda_fail(ctx, e, "query kernel"); }
        tie_rows += cnt[1];
        deferred_rows += cnt[2];
        retry_rows += cnt[6];
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
        grid_ms += ms;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        query_ms += ms;
        if (speculative) {
            cudaEventElapsedTime(&ms, ctx->ev[8], ctx->ev[9]);
            build_ms += ms;
        }
        const uint32_t nties = (uint32_t)std::min<uint64_t>(cnt[4], ctx->tie_cap);
        if (cnt[0] || nties) {
            if (!ties_queued) cudaEventRecord(ctx->ev[4], stream);
            rc = kd_ensure(ctx, t, stream);
            if (!rc && nties && !ties_queued) {
                TieLaunch tl;
                tl.tile = t;
                tl.K = K;
                tl.grp = g;
                tl.ex = sink;
                tl.ties = ctx->ties;
                tl.nties = nties;
                tl.kd = kd_order(t);
                tl.exact_rows = ctx->exact_rows;
                tl.counters = ctx->counters;
                tl.ids_out = nullptr;
                tl.row_k = row_k;
                rc = launch_ties(ctx, tl, stream);
                if (!rc) {
                    e = cudaMemcpyAsync(cnt, ctx->counters, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        stream);
                    if (!e) e = cudaStreamSynchronize(stream);
                    if (e) { cleanup(); return cuda_fail(ctx, e, "tie-order resolver"); }
                }
            }
            replay_rows += cnt[0];
            if (!rc) rc = kd_run_rows(ctx, t, K, g, sink, ctx->exact_rows, cnt[0], stream, row_k);
            if (rc) { cleanup(); return rc; }
            cudaEventRecord(ctx->ev[5], stream);
            e = cudaStreamSynchronize(stream);
            if (e) { cleanup(); return cuda_fail(ctx, e, "exact KD path"); }
            cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
            tree_ms += ms;
        }
    }
    ConsumerCounts cc;
    for (int s : consumers) {
        cudaEventRecord(ctx->ev[1], stream);
        rc = run_consumer(ctx, t, stages[s], s, dcols[s], sink, stream, &cc);
        if (rc) { cudaStreamSynchronize(stream); cleanup(); return rc; }
        cudaEventRecord(ctx->ev[2], stream);
        cudaStreamSynchronize(stream);
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
        query_ms += ms;
    }
    tie_rows += cc.tie_rows;
    replay_rows += cc.replay_rows;
    // results back to host layouts
    if (packed && !packed_copied) {
        rc = device_to_host(ctx, outputs[0].base, packed_dev, packed_bytes, stream);
        if (rc) { cleanup(); return rc; }
    }
    for (int s = 0; s < n_stages; ++s) {
        if (!hout[s].dev) continue;
        const nbg_columns& u = outputs[s];
        for (int d = 0; d < u.ndims; ++d) {
            if (u.point_stride == 8) {
                rc = device_to_host(ctx, (char*)u.base + u.offset[d], hout[s].dev + (size_t)d * n * 8,
                                    n * 8, stream);
                if (rc) { cleanup(); return rc; }
                continue;
            }
            cudaError_t e = cudaMemcpy2DAsync((char*)u.base + u.offset[d], u.point_stride,
                                              hout[s].dev + (size_t)d * n * 8, 8, 8, n,
                                              cudaMemcpyDeviceToHost, stream);
            if (e) { cleanup(); return cuda_fail(ctx, e, "output copy"); }
        }
    }
    uint32_t nex = 0, nresolve = 0;
    cudaError_t e = cudaMemcpyAsync(&nex, ctx->counters + 3, 4, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaMemcpyAsync(&nresolve, ctx->counters + 5, 4, cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (e) { cleanup(); return cuda_fail(ctx, e, "exception count"); }
    const uint32_t ncopy = std::min(nex, exception_capacity);
    if (ncopy && exceptions) {
        e = cudaMemcpyAsync(exceptions, ctx->ex_rows, ncopy * sizeof(nbg_row_exception),
                            cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        if (e) { cleanup(); return cuda_fail(ctx, e, "exception copy"); }
    }
    cudaEventRecord(ctx->ev[6], stream);
    cudaStreamSynchronize(stream);
    if (n_exceptions) *n_exceptions = nex;
    if (stats) {
        stats->points = n * (groups.size() + consumers.size());
        stats->outliers = cc.outliers;
        stats->inliers = cc.inliers;
        stats->tie_rows = tie_rows;
        stats->deferred_rows = deferred_rows;
        stats->resolved_rows = nresolve;
        stats->replay_rows = replay_rows;
        stats->grid_ms = grid_ms;
        stats->query_ms = query_ms;
        stats->tree_ms = tree_ms;
        stats->kd_build_ms = build_ms;
        stats->output_chunks = packed_copied ? (uint64_t)pipe_chunks : 0;
        stats->retry_rows = retry_rows;
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[6]);
        stats->total_ms = ms;
        stats->kernel_launches = g_launches.load() - launches0;
    }
    cleanup();
    if (nex > exception_capacity)
        return fail(ctx, NBG_ERR_EXCEPTIONS, "row-exception list overflowed");
    return NBG_OK;
}

namespace nbg {

// Tuning class of a tile for a neighbour count K: (floor(log2 points),
// neighbour slots of the select kernel).
static std::pair<int, int> tuning_class(const Tile* t, int K) {
    int lg = 0;
    while ((1ull << (lg + 1)) <= t->n) ++lg;
    return std::make_pair(lg, slots_for_k(K));
}

// A tile the caller did not tune takes the context's cached choice for its
// class (from nbg_tile_autotune or a loaded tuning file), if there is one.
// The batched form tunes its tiles through the autotuner's cache itself.
void apply_cached_tuning(Context* ctx, Tile* t, int K) {
    if (t->tuning_set || t->n == 0) return;
    auto hit = ctx->tuned.find(tuning_class(t, K));
    if (hit == ctx->tuned.end()) return;
    if (t->cell_factor != hit->second.first && !t->fixed_cell) {
        t->cell_factor = hit->second.first;
        t->grid_valid = false;
    }
    t->group = hit->second.second;
}

int tile_autotune(Context* ctx, Tile* t, int32_t knn, const float* candidates, int32_t n_candidates,
                  bool use_cache, float* chosen, cudaStream_t stream, bool per_thread_only) {
    if (knn < 0 || knn > 64) return fail(ctx, NBG_ERR_INVALID, "knn must be in [0, 64]");
    static const float defaults[] = {1.0f, 1.5f, 2.0f, 3.0f, 4.0f, 6.0f};
    if (!candidates || n_candidates <= 0) {
        candidates = defaults;
        n_candidates = (int32_t)(sizeof(defaults) / sizeof(defaults[0]));
    }
    const uint64_t n = t->n;
    if (n == 0) return NBG_OK;
    const int K = (int)std::min<uint64_t>(n, (uint64_t)knn + 1);
    const std::pair<int, int> key = tuning_class(t, K);
    auto hit = ctx->tuned.find(key);
    t->tuning_set = true;
    if (use_cache && hit != ctx->tuned.end()) {
        if (t->cell_factor != hit->second.first) {
            t->cell_factor = hit->second.first;
            t->fixed_cell = 0;
            t->grid_valid = false;
        }
        t->group = hit->second.second;
        if (chosen) *chosen = hit->second.first;
        return NBG_OK;
    }
    int rc = ensure_scratch(ctx, n, 1);
    if (rc) return rc;
    // sample: one contiguous window of rows in the grid's order (the whole
    // tile up to 8M rows), so that neighbouring blocks share cells and the
    // caches behave as in a full launch (runs of blocks scattered over the
    // tile misjudged the 32M-point stress tile: they chose a cell factor and
    // kernel 10 % slower than the default; a 4M-row window, best of two, did
    // not always separate kernels 8 % apart)
    const uint64_t window = std::min<uint64_t>(n, 8ull << 20);
    const uint64_t first_row = (n - window) / 2;
    std::vector<uint32_t> sample(window);
    for (uint64_t r = 0; r < window; ++r) sample[r] = (uint32_t)(first_row + r);
    const double scale = (double)n / (double)std::max<size_t>(sample.size(), 1);
    uint32_t* rows_dev = nullptr;
    rc = ctx_alloc(ctx, (void**)&rows_dev, sample.size() * 4 + 4);
    if (rc) return rc;
    rc = host_to_device(ctx, rows_dev, sample.data(), sample.size() * 4, stream);
    if (rc) {
        ctx_free(ctx, rows_dev, sample.size() * 4 + 4);
        return rc;
    }
    // select kernels tried: the two-pass ring search, the same in Morton
    // order, the single-pass ring search, 32 queries per candidate list (the
    // batched form's queue kernels are the two-pass ring search only)
    static const int kGroups[] = {0, 1, 2, 32};
    const int ngroups = per_thread_only ? 1 : 4;
    uint32_t* cnt_dev = ctx->counters + 32;  // scratch block, not the call counters
    float best = candidates[0];
    int best_group = 0;
    double best_ms = 1e300;
    for (int c = 0; c < n_candidates && !rc; ++c) {
        const float cf = candidates[c];
        if (!(cf > 0.0f) || cf > 64.0f) {
            rc = fail(ctx, NBG_ERR_INVALID, "bad cell factor");
            break;
        }
        t->cell_factor = cf;
        t->fixed_cell = 0;
        t->grid_valid = false;
        cudaEventRecord(ctx->ev[0], stream);
        rc = ensure_grid(ctx, t, K, stream);
        if (rc) break;
        cudaEventRecord(ctx->ev[1], stream);
        for (int gi = 0; gi < ngroups; ++gi) {
            const int G = kGroups[gi];
            QueryLaunch ql;
            ql.tile = t;
            ql.K = K;
            ql.rmax = 8;
            ql.grp = StageGroup{};
            ql.ex = ExceptionSink{ctx->ex_rows, cnt_dev + 3, 1};
            ql.exact_rows = ctx->exact_rows;
            ql.counters = cnt_dev;
            ql.ties = ctx->ties;
            ql.tie_cap = (uint32_t)std::min<uint64_t>(ctx->tie_cap, UINT32_MAX);
            ql.sums = ctx->sums;
            ql.rows = rows_dev;
            ql.nrows = sample.size();
            ql.retry_rows = ctx->retry_rows;
            ql.group = G;
            ql.margin0 = t->margin0;
            // best of three launches of the window
            float build_ms = 0, sample_ms = 1e30f;
            uint32_t cnt[3] = {0, 0, 0};
            for (int rep = 0; rep < 3 && !rc; ++rep) {
                cudaMemsetAsync(cnt_dev, 0, 8 * sizeof(uint32_t), stream);
                cudaEventRecord(ctx->ev[2], stream);
                rc = launch_query(ctx, ql, stream);
                if (rc) {
                    rc = fail(ctx, rc, "autotune sample launch");
                    break;
                }
                cudaEventRecord(ctx->ev[3], stream);
                cudaError_t e = cudaMemcpyAsync(cnt, cnt_dev, sizeof(cnt), cudaMemcpyDeviceToHost, stream);
                if (!e) e = cudaStreamSynchronize(stream);
                if (e) {
                    rc = fail(ctx, NBG_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
                    break;
                }
                float ms = 0;
                cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
                sample_ms = std::min(sample_ms, ms);
            }
            if (rc) break;
            cudaEventElapsedTime(&build_ms, ctx->ev[0], ctx->ev[1]);
            // rows the ring search cannot finish go to the search replay: charge
            // each an estimated 5 us of replay
            const double deferred = (double)cnt[0] * scale;
            const double est = build_ms + sample_ms * scale + deferred * 0.005;
            if (est < best_ms) {
                best_ms = est;
                best = cf;
                best_group = G;
            }
        }
    }
    ctx_free(ctx, rows_dev, sample.size() * 4 + 4);
    if (rc) return rc;
    t->cell_factor = best;
    t->group = best_group;
    t->grid_valid = false;
    ctx->tuned[key] = std::make_pair(best, best_group);
    if (chosen) *chosen = best;
    return NBG_OK;
}

}  // namespace nbg

extern "C" int nbg_tile_autotune(nbg_context* h, nbg_tile* th, int32_t knn, const float* candidates,
                                 int32_t n_candidates, int32_t use_cache, float* chosen,
                                 void* stream_v) {
    if (!h || !th) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    return tile_autotune(ctx, &th->t, knn, candidates, n_candidates, use_cache != 0, chosen,
                         (cudaStream_t)stream_v);
}

extern "C" int nbg_autotune_cache_get(nbg_context* h, nbg_tune_entry* entries, int32_t capacity,
                                      int32_t* count) {
    if (!h || !count || capacity < 0 || (capacity > 0 && !entries)) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    int32_t i = 0;
    for (const auto& kv : ctx->tuned) {
        if (i < capacity) {
            entries[i].size_class = kv.first.first;
            entries[i].slots = kv.first.second;
            entries[i].cell_factor = kv.second.first;
            entries[i].select_kernel = kv.second.second;
        }
        ++i;
    }
    *count = i;
    return NBG_OK;
}

extern "C" int nbg_autotune_cache_set(nbg_context* h, const nbg_tune_entry* entries, int32_t count) {
    if (!h || count < 0 || (count > 0 && !entries)) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    for (int32_t i = 0; i < count; ++i) {
        const nbg_tune_entry& e = entries[i];
        if (e.size_class < 0 || e.size_class > 63 || e.slots < 1 || e.slots > 128 ||
            !std::isfinite(e.cell_factor) || !(e.cell_factor > 0.0f) ||
            !valid_select(e.select_kernel))
            return fail(ctx, NBG_ERR_INVALID, "bad tuning-cache entry");
    }
    for (int32_t i = 0; i < count; ++i)
        ctx->tuned[std::make_pair((int)entries[i].size_class, (int)entries[i].slots)] =
            std::make_pair(entries[i].cell_factor, (int)entries[i].select_kernel);
    return NBG_OK;
}

extern "C" int nbg_neighbor_sets(nbg_context* h, nbg_tile* th, int32_t knn, uint32_t* ids_out,
                                 int32_t ids_on_device, nbg_run_stats* stats, void* stream_v) {
    if (!h || !th || !ids_out) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    Tile* t = &th->t;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t stream = (cudaStream_t)stream_v;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (knn < 0 || knn > 64) return fail(ctx, NBG_ERR_INVALID, "knn must be in [0, 64]");
    const uint64_t n = t->n;
    if (n == 0) return NBG_OK;
    const int K = (int)std::min<uint64_t>(n, (uint64_t)knn + 1);
    int rc = ensure_scratch(ctx, n, 1);
    if (rc) return rc;
    rc = ensure_grid(ctx, t, K, stream);
    if (rc) return rc;
    uint32_t* dev_ids = ids_out;
    const size_t bytes = n * (size_t)K * 4;
    if (!ids_on_device) {
        rc = dev_alloc(ctx, (void**)&dev_ids, bytes, nullptr);
        if (rc) return rc;
    }
    cudaMemsetAsync(ctx->counters, 0, 64 * sizeof(uint32_t), stream);
    rc = launch_neighbor_sets(ctx, t, K, 8, dev_ids, ctx->exact_rows, ctx->counters, ctx->ties,
                              (uint32_t)std::min<uint64_t>(ctx->tie_cap, UINT32_MAX), stream,
                              ctx->retry_rows);
    uint32_t cnt[5] = {0, 0, 0, 0, 0};
    cudaError_t e = cudaSuccess;
    if (!rc) {
        e = cudaMemcpyAsync(cnt, ctx->counters, 20, cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
    }
    const uint32_t nties = (uint32_t)std::min<uint64_t>(cnt[4], ctx->tie_cap);
    if (!rc && !e && (cnt[0] || nties)) {
        rc = kd_ensure(ctx, t, stream);
        if (!rc && nties) {
            TieLaunch tl{};
            tl.tile = t;
            tl.K = K;
            tl.ties = ctx->ties;
            tl.nties = nties;
            tl.kd = kd_order(t);
            tl.exact_rows = ctx->exact_rows;
            tl.counters = ctx->counters;
            tl.ids_out = dev_ids;
            rc = launch_ties(ctx, tl, stream);
            if (!rc) {
                e = cudaMemcpyAsync(cnt, ctx->counters, 4, cudaMemcpyDeviceToHost, stream);
                if (!e) e = cudaStreamSynchronize(stream);
            }
        }
        if (!rc && !e) rc = kd_neighbor_rows(ctx, t, K, ctx->exact_rows, cnt[0], dev_ids, stream);
    }
    if (!rc && !e && !ids_on_device) rc = device_to_host(ctx, ids_out, dev_ids, bytes, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (!ids_on_device) dev_free(ctx, dev_ids, bytes);
    if (stats) {
        stats->points = n;
        stats->tie_rows = cnt[1];
        stats->deferred_rows = cnt[2];
        stats->replay_rows = cnt[0];
    }
    if (rc) return rc;
    if (e) return cuda_fail(ctx, e, "neighbour sets");
    return NBG_OK;
}

extern "C" int nbg_debug_kd_export(nbg_context* h, nbg_tile* th, uint32_t* vind, uint32_t* n_nodes,
                                   int32_t* child1, int32_t* child2, int32_t* divfeat,
                                   double* divlow, double* divhigh, uint32_t* begin,
                                   uint32_t* end, uint32_t node_capacity) {
    if (!h || !th || !vind || !n_nodes) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    Tile* t = &th->t;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if (t->n == 0) {
        *n_nodes = 0;
        return NBG_OK;
    }
    int rc = ensure_grid(ctx, t, (int)std::min<uint64_t>(t->n, 9), 0);
    if (rc) return rc;
    return kd_export(ctx, t, vind, n_nodes, child1, child2, divfeat, divlow, divhigh, begin, end,
                     node_capacity, 0);
}

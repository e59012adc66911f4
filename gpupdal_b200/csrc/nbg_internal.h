// nbg_internal.h — host-side internals shared by the library's .cu files.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <unordered_map>
#include <string>
#include <vector>

#include "nbg_common.cuh"
#include "nbg_consumers.cuh"

struct nbg_tile;

namespace nbg {

struct KdReplica;  // exact nanoflann replica (nbg_kdtree.cu)

// Kernels launched by this library (all contexts), for the per-call count.
extern std::atomic<uint64_t> g_launches;
#define NBG_LAUNCHED(n) ::nbg::g_launches.fetch_add((n), std::memory_order_relaxed)

// NVTX range over a host-side phase (grid build, KD replica build, search
// replay, copies, whole calls), seen by Nsight tools; without a tool attached
// a push/pop is a no-op call.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define NBG_RANGE_CAT2(a, b) a##b
#define NBG_RANGE_CAT(a, b) NBG_RANGE_CAT2(a, b)
#define NBG_RANGE(name) ::nbg::NvtxRange NBG_RANGE_CAT(nbg_range_, __LINE__)(name)

struct Context {
    int device = 0;
    int sm_count = 148;
    uint64_t budget = 0;   // HBM budget in bytes (0 = no limit)
    uint64_t used = 0;     // bytes held by tiles and scratch
    std::string err;
    std::mutex mu;   // held by every entry point that takes the context
    std::mutex amu;  // the block cache below (the batched form's KD helper thread allocates too)
    std::mutex emu;  // err
    // per-call scratch (grown on demand)
    uint32_t* exact_rows = nullptr;
    uint64_t exact_cap = 0;
    uint2* ties = nullptr;          // tie list of the query kernels
    uint64_t tie_cap = 0;
    uint32_t* retry_rows = nullptr; // rows the group select hands to the per-thread select
    uint64_t retry_cap = 0;
    RowSums* sums = nullptr;        // select -> finish hand-over
    uint64_t sums_cap = 0;
    uint32_t* counters = nullptr;   // [0] exact rows, [1] tie rows, [2] deferred, [3] exceptions,
                                    // [4] tie list, [5] eigen re-solves, [6] group select retries
    nbg_row_exception* ex_rows = nullptr;
    uint64_t ex_cap = 0;
    cudaEvent_t ev[10];
    bool events = false;
    // high-priority side stream: the KD replica build runs there while the
    // query kernels run on the caller's stream
    cudaStream_t side = nullptr;
    cudaEvent_t xev[2];
    // normal-priority stream for the single-pass select's handed-back rows,
    // answered beside the finish pass of the other rows (fev: fork and join)
    cudaStream_t fork = nullptr;
    cudaEvent_t fev[4];
    // device blocks released by earlier calls, kept for reuse by size
    std::multimap<size_t, void*> cache;
    uint64_t cached = 0;
    std::unordered_map<void*, size_t> live;  // block sizes of handed-out blocks
    // autotuner: chosen cell factor and select kernel (queries per group)
    // per (log2 points, neighbour slots) class
    std::map<std::pair<int, int>, std::pair<float, int>> tuned;
    // pinned bounce buffers for copies to and from pageable host memory
    char* bounce[2] = {nullptr, nullptr};
    cudaEvent_t bev[2];
    bool bounce_ready = false;
};

// Copies between device memory and host memory.  Pinned (or registered) host
// memory is copied directly; pageable host memory goes through the
// context's pinned bounce buffers in 32 MiB chunks, the device copy of one
// chunk overlapping the host-side memcpy (several threads) of the previous.
// Both return once the host side is complete (d2h) or the source may be
// reused (h2d).
int host_to_device(Context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream);
int device_to_host(Context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Device allocation through the context: reuses a cached block of the
// request's size class (up to twice its size), honours the HBM budget (cached
// blocks are released first when the budget would be exceeded).  Returns
// NBG_OK, NBG_ERR_BUDGET or NBG_ERR_OOM.
int ctx_alloc(Context* ctx, void** p, size_t bytes);
void ctx_free(Context* ctx, void* p, size_t bytes);
void ctx_trim(Context* ctx);

struct Tile {
    uint64_t n = 0;
    int32_t* x = nullptr;
    int32_t* y = nullptr;
    int32_t* z = nullptr;
    Transform tf{};
    // grid
    int32_t* bbox = nullptr;
    GridParams* gp = nullptr;
    int4* colinfo = nullptr;     // cols_cap: {base, zmin, zmax, 0}
    uint32_t* ext = nullptr;     // cols_cap + 1: column extents, then bases
    uint32_t* table_dev = nullptr;
    uint32_t* keys = nullptr;    // n: table entry of each point
    uint32_t* cstart = nullptr;  // table_cap: first point of each entry
    uint32_t* cursor = nullptr;  // table_cap: scatter cursor
    float4* sorted = nullptr;    // n
    void* grid_tmp = nullptr;
    size_t grid_tmp_bytes = 0;
    uint64_t cols_cap = 0;
    uint64_t table_cap = 0;
    uint64_t table_size = 0;
    bool fixed_storage = false;  // storage provided by the caller: never grow
    float cell_factor = 4.0f;
    int32_t fixed_cell = 0;
    // select kernel: 0 the two-pass per-thread ring search (default), 1 the
    // same in block-local Morton order, 2 the single-pass ring search, 8 / 16
    // / 32 queries sharing one candidate list; the group select's first box
    // margin in cell edges
    int group = 0;
    float margin0 = 0.5f;
    // the caller chose the cell factor or select kernel (nbg_tile_tune,
    // nbg_tile_set_select, nbg_tile_autotune): the context's cached tuning of
    // the tile's class is then not applied by nbg_run
    bool tuning_set = false;
    int grid_k1 = 0;
    int32_t grid_fixed = 0;      // fixed cell edge the current grid was built with (0: density)
    bool grid_valid = false;
    GridParams host_gp{};
    // exact replica of the reference's KD tree (built on first need)
    KdReplica* kd = nullptr;
    uint64_t bytes = 0;
};

int build_grid(Context* ctx, Tile* t, int k1, cudaStream_t stream);
// Grid for neighbour count k1 (or a fixed cell edge), rebuilt only when needed.
int ensure_grid(Context* ctx, Tile* t, int k1, cudaStream_t stream, int32_t cell = 0);
int build_grid_async(Context* ctx, Tile* t, int k1, cudaStream_t stream);

int fail(Context* c, int code, const std::string& msg);
// Sets the context's error message (thread-safe).
void set_err(Context* c, const std::string& msg);
int validate_stages(Context* ctx, const nbg_stage_opts* stages, int n_stages,
                    const nbg_columns* outputs, bool* need_aux);
void fill_stage(StageDev& d, const nbg_stage_opts& o, const nbg_columns& c);
int ensure_scratch(Context* ctx, uint64_t n, uint64_t ex_cap);
size_t grid_temp_bytes(uint64_t items);
int grid_grow_table(Context* ctx, Tile* t, uint64_t entries);
GridView grid_view(const Tile* t);

struct QueryLaunch {
    const Tile* tile;
    int K;          // neighbours including the point itself
    int rmax;
    StageGroup grp;
    ExceptionSink ex;
    uint32_t* exact_rows;
    uint32_t* counters;
    uint2* ties = nullptr;  // tie list (null: tie rows join exact_rows)
    uint32_t tie_cap = 0;
    RowSums* sums = nullptr;  // split select/finish kernels (null: one fused kernel)
    const double* row_k = nullptr;  // per-row neighbour count (optimized), device
    const uint32_t* rows = nullptr;  // split form only: sorted positions to answer (null: all)
    uint64_t nrows = 0;
    // group select (split form): rows handed back to the per-thread select
    // (capacity: the rows answered; null: the per-thread select for every row)
    uint32_t* retry_rows = nullptr;
    int group = 0;
    float margin0 = 0.25f;
    // when set, the launch records `done` once every row is answered and
    // leaves `stream` free for the next launch (the single-pass select's
    // handed-back rows may still run on the context's fork stream); when
    // null, every row is answered in `stream` order
    cudaEvent_t done = nullptr;
};
int launch_query(Context* ctx, const QueryLaunch& q, cudaStream_t stream);
// rows + bounds[c] receives, in ascending order, the sorted positions whose
// point id lies in [bounds[c], bounds[c+1]), for c < nchunks (bounds[nchunks]
// = n); `dnum` is one device word the selection writes its count to.
// Returns after the selection completed.
int build_id_chunks(Context* ctx, const Tile* t, const uint64_t* bounds, int nchunks,
                    uint32_t* rows, uint32_t* dnum, cudaStream_t st);
// Select pass over a sample of `blocks` blocks of 128 rows, in runs of `run`
// consecutive blocks whose starts are `stride` rows apart.
int launch_select_sample(Context* ctx, const QueryLaunch& q, uint64_t stride, unsigned blocks,
                         unsigned run, cudaStream_t stream);

// Tie rows ordered on the KD replica's tree (no search replay).
struct TieLaunch {
    const Tile* tile;
    int K;
    StageGroup grp;
    ExceptionSink ex;
    const uint2* ties;
    uint32_t nties;
    KdOrder kd;
    uint32_t* exact_rows;  // rows the resolver hands to the search replay
    uint32_t* counters;
    uint32_t* ids_out;     // neighbour-set export (null in the fused path)
    const double* row_k = nullptr;
};
int launch_ties(Context* ctx, const TieLaunch& tl, cudaStream_t stream);
// The same with the row count read on the device: min(*count, tl.nties) rows
// (tl.nties: the list's capacity), so the launch can be queued before the
// query that fills the list has finished.
int launch_ties_counted(Context* ctx, const TieLaunch& tl, const uint32_t* count, cudaStream_t stream);
// True when launch_query answers `q`'s handed-back rows on the context's fork
// stream (the single-pass select): work queued there after the launch runs
// once the tie list is complete, beside the finish pass.
bool query_forks(const Context* ctx, const QueryLaunch& q);
// The tie rows of several tiles in one launch (returns after it completed).
int launch_ties_many(Context* ctx, const TieLaunch* tls, int count, cudaStream_t stream);

// Radius neighbourhoods of one stage (no tie order: every point within the
// radius belongs to the set).
struct RadiusLaunch {
    const Tile* tile;
    StageGroup grp;   // one stage
    ExceptionSink ex;
    double radius;
    int32_t min_k;    // rows below it are skipped (not for normal)
};
int launch_radius(Context* ctx, const RadiusLaunch& rl, cudaStream_t stream);

// Exact path: nanoflann replica build (lazy) + DFS for the listed rows.
// beside_query: the build shares the SMs with a running query whose results
// do not wait for it early; from 16M points its launches then keep to a few
// blocks per SM (tiles and subtrees walked in strides)
int kd_ensure(Context* ctx, Tile* t, cudaStream_t stream, bool beside_query = false);
// One forest holding the replicas of every listed tile that has none.
int kd_ensure_many(Context* ctx, Tile* const* tiles, int count, cudaStream_t stream,
                   bool beside_query = false);
int kd_run_rows(Context* ctx, Tile* t, int K, const StageGroup& grp, const ExceptionSink& ex,
                const uint32_t* rows, uint32_t nrows, cudaStream_t stream,
                const double* row_k = nullptr, int stride = 1, int kpick = 0);
// Strided neighbourhoods of one stage over every row (K = k * stride);
// needs the tile's KD replica.
// With `list`, the ordered list of K entries goes to that kNN consumer's
// epilogue instead (stride 1, kpick K).
int launch_stride(Context* ctx, const QueryLaunch& q, int stride, int kpick, const KdOrder& kd,
                  cudaStream_t stream, const ListArgs* list = nullptr);
// Search replay of the listed rows for a kNN consumer (the replica's own
// list order is the reference's).
int kd_list_rows(Context* ctx, Tile* t, int K, const ListArgs& L, const ExceptionSink& ex,
                 const uint32_t* rows, uint32_t nrows, cudaStream_t stream);
int kd_neighbor_rows(Context* ctx, Tile* t, int K, const uint32_t* rows, uint32_t nrows,
                     uint32_t* ids_out, cudaStream_t stream);
KdOrder kd_order(const Tile* t);
bool kd_built(const Tile* t);
void kd_free(Context* ctx, Tile* t);
uint64_t kd_bytes(uint64_t n);
int kd_export(Context* ctx, Tile* t, uint32_t* vind, uint32_t* nnodes, int32_t* c1, int32_t* c2,
              int32_t* feat, double* dlo, double* dhi, uint32_t* nb, uint32_t* ne, uint32_t cap,
              cudaStream_t st);

// neighbour-set export of the grid path
int launch_neighbor_sets(Context* ctx, const Tile* t, int K, int rmax, uint32_t* ids_out,
                         uint32_t* exact_rows, uint32_t* counters, uint2* ties, uint32_t tie_cap,
                         cudaStream_t stream, uint32_t* retry_rows = nullptr);

// A tile the caller did not tune (cell factor, select kernel) takes the
// context's cached autotuner choice for its (size, neighbour slots) class.
void apply_cached_tuning(Context* ctx, Tile* t, int K);

// Autotuner (nbg_tile_autotune without the context lock).
int tile_autotune(Context* ctx, Tile* t, int32_t knn, const float* candidates, int32_t n_candidates,
                  bool use_cache, float* chosen, cudaStream_t stream,
                  bool per_thread_only = false);

// A tile of n points with its device storage allocated (coordinates unset),
// and its release (nbg_api.cu).
int tile_alloc(Context* ctx, uint64_t n, const double scale[3], const double offset[3],
               nbg_tile** out);
void tile_destroy(Context* ctx, nbg_tile* th);

// kNN-consumer stages (nndistance, optimalneighborhood, lof, outlier) of one
// nbg_run call (nbg_consumers.cu); outlier counts accumulate into `stats`.
struct ConsumerCounts {
    uint64_t outliers = 0, inliers = 0, tie_rows = 0, replay_rows = 0;
};
int run_consumer(Context* ctx, Tile* t, const nbg_stage_opts& o, int stage_index,
                 const nbg_columns& col, const ExceptionSink& sink, cudaStream_t stream,
                 ConsumerCounts* counts);
bool is_list_consumer(int kind);

// Batched form: the context's batch scratch and cached graph (nbg_batch.cu).
void batch_release(Context* ctx);

}  // namespace nbg

// The C ABI's opaque handles.
struct nbg_context {
    nbg::Context c;
};
struct nbg_tile {
    nbg::Tile t;
};

// nbg_batch.cu — the batched form: many tiles, one graph-captured queue.
//
// 1. grids     every tile's grid, built without host synchronisation, then
//              one synchronisation reads all grid shapes (a tile whose cell
//              table overflowed is rebuilt by the synchronising build)
// 2. queue     per neighbour-count class one persistent select kernel drains
//              the class's (tile, 128-query block) items; one persistent
//              finish kernel then takes every item of every class.  The head
//              resets and the launches are captured in a CUDA graph, replayed
//              while the batch's job arrays and counts are unchanged.
// 3. replicas  the tiles' KD replicas, all as one forest (one level-synchronous
//              build for every tile), once the queue has drained
// 4. exact     per tile: the tie-order resolver, then the search replay for
//              the rows it hands on, as in nbg_run
// Each tile owns disjoint slices of the row-sum, tie and replay lists and
// its own counter block, so a tile's results do not depend on the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "nbg_internal.h"

namespace nbg {

// `reserve`: resident blocks per SM the persistent launch leaves free, so that
// the KD replica build on the side stream runs beside it instead of after it.
int launch_select_queue(Context* ctx, int K, const BatchJob* jobs, int njobs, uint64_t items,
                        unsigned long long* head, cudaStream_t stream, int reserve);
int launch_finish_queue(Context* ctx, const BatchJob* jobs, int njobs, uint64_t items,
                        unsigned long long* head, cudaStream_t stream, int reserve);
int slots_for_k(int K);

static constexpr int kCounters = 64;  // u32 counters per tile

struct BatchScratch {
    uint64_t rows = 0, items = 0, ex = 0;
    RowSums* sums = nullptr;
    uint2* ties = nullptr;
    uint32_t* exact = nullptr;
    uint32_t* counters = nullptr;
    nbg_row_exception* ex_rows = nullptr;
    BatchJob* jobs = nullptr;  // select order (by class), then finish order
    unsigned long long* heads = nullptr;
    uint64_t jobs_cap = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6];
    bool events = false;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key;  // what the captured graph was built for
};

static std::map<Context*, BatchScratch*> g_batch;
static std::mutex g_batch_mu;

static BatchScratch* scratch_of(Context* ctx) {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    BatchScratch*& b = g_batch[ctx];
    if (!b) b = new BatchScratch();
    return b;
}

template <class T>
static int grow(Context* ctx, T** p, uint64_t& cap_now, uint64_t want) {
    if (*p && cap_now >= want) return NBG_OK;
    if (*p) ctx_free(ctx, *p, cap_now * sizeof(T));
    *p = nullptr;
    int rc = ctx_alloc(ctx, (void**)p, std::max<uint64_t>(want, 1) * sizeof(T));
    if (rc) return rc;
    cap_now = std::max<uint64_t>(want, 1);
    return NBG_OK;
}

void batch_release(Context* ctx) {
    BatchScratch* B = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        auto it = g_batch.find(ctx);
        if (it == g_batch.end()) return;
        B = it->second;
        g_batch.erase(it);
    }
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->sums) ctx_free(ctx, B->sums, B->rows * sizeof(RowSums));
    if (B->ties) ctx_free(ctx, B->ties, B->rows * sizeof(uint2));
    if (B->exact) ctx_free(ctx, B->exact, B->rows * 4);
    if (B->counters) ctx_free(ctx, B->counters, B->items * 4);
    if (B->ex_rows) ctx_free(ctx, B->ex_rows, B->ex * sizeof(nbg_row_exception));
    if (B->jobs) ctx_free(ctx, B->jobs, B->jobs_cap * sizeof(BatchJob));
    if (B->heads) ctx_free(ctx, B->heads, (B->jobs_cap + 1) * sizeof(unsigned long long));
    if (B->events) {
        for (int e = 0; e < 6; ++e) cudaEventDestroy(B->ev[e]);
        cudaStreamDestroy(B->stream);
    }
    delete B;
}

}  // namespace nbg

using namespace nbg;

extern "C" int nbg_run_batch(nbg_context* h, const nbg_batch_item* items, int32_t n_items,
                             uint32_t flags, nbg_run_stats* stats, void* stream_v) {
    NBG_RANGE("nbg_run_batch");
    if (!h || n_items < 0 || (n_items && !items)) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t user = (cudaStream_t)stream_v;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const uint64_t launches0 = g_launches.load();
    // ---- validation and per-tile groups
    std::set<const nbg_tile*> seen;
    std::vector<int> live;
    std::vector<int> Ks(n_items, 0);
    std::vector<StageGroup> groups(n_items);
    uint64_t rows = 0, ex_total = 0;
    for (int i = 0; i < n_items; ++i) {
        const nbg_batch_item& it = items[i];
        if (it.n_exceptions) *it.n_exceptions = 0;
        if (!it.tile || it.n_stages < 1 || it.n_stages > NBG_MAX_STAGES || !it.stages || !it.outputs)
            return fail(ctx, NBG_ERR_INVALID, "bad batch item");
        if (!seen.insert(it.tile).second)
            return fail(ctx, NBG_ERR_INVALID, "a tile appears twice in the batch");
        bool need_aux = false;
        int rc = validate_stages(ctx, it.stages, it.n_stages, it.outputs, &need_aux);
        if (rc) return rc;
        if (need_aux && (!it.optimal_knn || !it.optimal_radius))
            return fail(ctx, NBG_ERR_INVALID, "Density needs OptimalKNN and OptimalRadius");
        for (int s = 0; s < it.n_stages; ++s) {
            if (it.stages[s].kind > NBG_STAGE_COVARIANCEFEATURES)
                return fail(ctx, NBG_ERR_UNSUPPORTED,
                            "the other kNN consumers run through nbg_run, not the batch");
            if (it.stages[s].knn != it.stages[0].knn)
                return fail(ctx, NBG_ERR_UNSUPPORTED, "the stages of a batch item share one knn");
            if (it.outputs[s].on_device != 1)
                return fail(ctx, NBG_ERR_UNSUPPORTED, "batch outputs are device-resident");
            if (it.stages[s].use_radius || it.stages[s].optimized ||
                (it.stages[s].kind != NBG_STAGE_NORMAL && it.stages[s].stride > 1))
                return fail(ctx, NBG_ERR_UNSUPPORTED,
                            "radius, optimized and strided stages run through nbg_run, not the batch");
        }
        const Tile* t = &it.tile->t;
        if (t->n == 0) continue;
        Ks[i] = (int)std::min<uint64_t>(t->n, (uint64_t)it.stages[0].knn + 1);
        StageGroup& g = groups[i];
        g = StageGroup{};
        g.nstages = it.n_stages;
        g.optimal_knn = it.optimal_knn;
        g.optimal_radius = it.optimal_radius;
        for (int s = 0; s < it.n_stages; ++s) {
            g.stage_index[s] = s;
            fill_stage(g.st[s], it.stages[s], it.outputs[s]);
            const nbg_stage_opts& o = it.stages[s];
            if ((o.kind == NBG_STAGE_NORMAL && !o.always_up && !o.has_viewpoint) || o.eigen_fp64)
                g.sign_exact = 1;
        }
        live.push_back(i);
        rows += t->n;
        ex_total += std::max<uint32_t>(it.exception_capacity, 1);
    }
    if (live.empty()) return NBG_OK;
    BatchScratch* B = scratch_of(ctx);
    if (!B->events) {
        for (int e = 0; e < 6; ++e) cudaEventCreate(&B->ev[e]);
        cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
        B->events = true;
    }
    cudaStream_t st = B->stream;
    // ---- scratch
    const int nl = (int)live.size();
    int rc = NBG_OK;
    if (B->rows < rows) {
        uint64_t c1 = B->rows, c2 = B->rows, c3 = B->rows;
        rc = grow(ctx, &B->sums, c1, rows);
        if (!rc) rc = grow(ctx, &B->ties, c2, rows);
        if (!rc) rc = grow(ctx, &B->exact, c3, rows);
        if (rc) return rc;
        B->rows = rows;
    }
    if (B->items < (uint64_t)nl * kCounters) {
        uint64_t c = B->items;
        rc = grow(ctx, &B->counters, c, (uint64_t)nl * kCounters);
        if (rc) return rc;
        B->items = (uint64_t)nl * kCounters;
    }
    if (B->ex < ex_total) {
        uint64_t c = B->ex;
        rc = grow(ctx, &B->ex_rows, c, ex_total);
        if (rc) return rc;
        B->ex = ex_total;
    }
    // ---- cell factors from the autotuner (measured once per size/knn class)
    if (flags & NBG_BATCH_AUTOTUNE) {
        for (int i : live) {
            rc = tile_autotune(ctx, &items[i].tile->t, items[i].stages[0].knn, nullptr, 0, true,
                               nullptr, st, true);
            if (rc) return rc;
        }
    }
    // ---- grids (no host synchronisation), then one read of every shape
    cudaEventRecord(B->ev[0], user);
    cudaStreamWaitEvent(st, B->ev[0], 0);
    for (int i : live) {
        Tile* t = &items[i].tile->t;
        if (t->grid_valid && t->grid_fixed == t->fixed_cell &&
            (t->fixed_cell || (Ks[i] <= 2 * t->grid_k1 && 2 * Ks[i] >= t->grid_k1)))
            continue;
        t->grid_valid = false;
        rc = build_grid_async(ctx, t, Ks[i], st);
        if (rc) return fail(ctx, rc, "grid build failed");
    }
    std::vector<GridParams> gps(nl);
    for (int j = 0; j < nl; ++j)
        cudaMemcpyAsync(&gps[j], items[live[j]].tile->t.gp, sizeof(GridParams), cudaMemcpyDeviceToHost, st);
    cudaEventRecord(B->ev[1], st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch grid build");
    for (int j = 0; j < nl; ++j) {
        Tile* t = &items[live[j]].tile->t;
        const GridParams& g = gps[j];
        if ((int64_t)g.maxx - g.minx >= (1 << 24) || (int64_t)g.maxy - g.miny >= (1 << 24) ||
            (int64_t)g.maxz - g.minz >= (1 << 24))
            return fail(ctx, NBG_ERR_UNSUPPORTED, "tile extent must be below 2^24 raw units per axis");
        if (g.cap_hit & 2u) {
            // cell table too small for this grid: the synchronising build grows it
            rc = build_grid(ctx, t, Ks[live[j]], st);
            if (!rc && cudaMemcpyAsync(&t->host_gp, t->gp, sizeof(GridParams), cudaMemcpyDeviceToHost, st))
                rc = NBG_ERR_CUDA;
            if (!rc && cudaStreamSynchronize(st)) rc = NBG_ERR_CUDA;
            if (rc) return fail(ctx, rc, "grid rebuild failed");
        } else {
            t->host_gp = g;
        }
        t->grid_valid = true;
        t->grid_k1 = Ks[live[j]];
        t->grid_fixed = t->fixed_cell;
    }
    // ---- jobs: select order grouped by class, then finish order
    std::vector<int> order(live);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return slots_for_k(Ks[a]) < slots_for_k(Ks[b]); });
    std::vector<BatchJob> jobs(2 * (size_t)nl);
    std::vector<uint64_t> row0(n_items, 0), ex0(n_items, 0), slot(n_items, 0);
    {
        uint64_t r = 0, e = 0;
        for (int j = 0; j < nl; ++j) {
            const int i = live[j];
            row0[i] = r;
            ex0[i] = e;
            slot[i] = (uint64_t)j;
            r += items[i].tile->t.n;
            e += std::max<uint32_t>(items[i].exception_capacity, 1);
        }
    }
    struct Cls {
        int K;
        int begin, count;
        uint64_t items;
    };
    std::vector<Cls> classes;
    uint64_t fin_items = 0;
    for (int j = 0; j < nl; ++j) {
        const int i = order[j];
        const Tile* t = &items[i].tile->t;
        QueryArgs q{};
        q.gv = grid_view(t);
        q.gp = t->gp;
        q.n = t->n;
        q.K = Ks[i];
        q.rmax = 8;
        q.grp = groups[i];
        q.grp.resolve_count = B->counters + slot[i] * kCounters + 5;
        q.tf = t->tf;
        q.ex = ExceptionSink{B->ex_rows + ex0[i], B->counters + slot[i] * kCounters + 3,
                             std::max<uint32_t>(items[i].exception_capacity, 1)};
        q.exact_rows = B->exact + row0[i];
        q.counters = B->counters + slot[i] * kCounters;
        q.ids_out = nullptr;
        q.ties = B->ties + row0[i];
        q.tie_cap = (uint32_t)t->n;
        q.sums = B->sums + row0[i];
        const uint64_t blocks = (t->n + 127) / 128;
        if (classes.empty() || slots_for_k(classes.back().K) != slots_for_k(Ks[i]))
            classes.push_back(Cls{Ks[i], j, 0, 0});
        Cls& c = classes.back();
        jobs[j].q = q;
        jobs[j].first = c.items;
        c.items += blocks;
        c.count += 1;
        jobs[nl + j].q = q;
        jobs[nl + j].first = fin_items;
        fin_items += blocks;
    }
    if (B->jobs_cap < jobs.size()) {
        if (B->jobs) ctx_free(ctx, B->jobs, B->jobs_cap * sizeof(BatchJob));
        if (B->heads) ctx_free(ctx, B->heads, (B->jobs_cap + 1) * sizeof(unsigned long long));
        B->jobs = nullptr;
        B->heads = nullptr;
        rc = ctx_alloc(ctx, (void**)&B->jobs, jobs.size() * sizeof(BatchJob));
        if (!rc) rc = ctx_alloc(ctx, (void**)&B->heads, (jobs.size() + 1) * sizeof(unsigned long long));
        if (rc) return rc;
        B->jobs_cap = jobs.size();
        if (B->exec) {
            cudaGraphExecDestroy(B->exec);
            B->exec = nullptr;
        }
    }
    // per-tile counters restart at zero; the job table is pageable host memory,
    // so its upload completes before this call returns from the copy
    cudaMemsetAsync(B->counters, 0, (size_t)nl * kCounters * sizeof(uint32_t), st);
    rc = host_to_device(ctx, B->jobs, jobs.data(), jobs.size() * sizeof(BatchJob), st);
    if (rc) return rc;
    // tiles whose KD replica is built after the queue
    std::vector<Tile*> kd_tiles;
    for (int i : live)
        if (items[i].tile->t.n > 100 && !kd_built(&items[i].tile->t)) kd_tiles.push_back(&items[i].tile->t);
    // the persistent launches take every resident block slot
    const int reserve = 0;
    // ---- the queue launches, captured once per batch shape
    std::vector<uint64_t> key;
    key.push_back((uint64_t)reserve);
    key.push_back((uint64_t)(uintptr_t)B->jobs);
    key.push_back(fin_items);
    key.push_back((uint64_t)nl);
    for (const Cls& c : classes) {
        key.push_back((uint64_t)slots_for_k(c.K));
        key.push_back((uint64_t)c.begin);
        key.push_back((uint64_t)c.count);
        key.push_back(c.items);
    }
    auto record = [&](cudaStream_t s) -> int {
        cudaMemsetAsync(B->heads, 0, (classes.size() + 1) * sizeof(unsigned long long), s);
        for (size_t k = 0; k < classes.size(); ++k) {
            const Cls& c = classes[k];
            int r = launch_select_queue(ctx, c.K, B->jobs + c.begin, c.count, c.items, B->heads + k, s,
                                        reserve);
            if (r) return r;
        }
        return launch_finish_queue(ctx, B->jobs + nl, nl, fin_items, B->heads + classes.size(), s,
                                   reserve);
    };
    const bool graph = (flags & NBG_BATCH_GRAPH) != 0;
    if (graph && (!B->exec || B->key != key)) {
        if (B->exec) {
            cudaGraphExecDestroy(B->exec);
            B->exec = nullptr;
        }
        cudaGraph_t gr = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(ctx, NBG_ERR_CUDA, "graph capture");
        const int r = record(st);
        cudaError_t ce = cudaStreamEndCapture(st, &gr);
        if (r || ce != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return fail(ctx, NBG_ERR_CUDA, "graph capture of the batch queue failed");
        }
        ce = cudaGraphInstantiate(&B->exec, gr, 0);
        cudaGraphDestroy(gr);
        if (ce != cudaSuccess) {
            B->exec = nullptr;
            return fail(ctx, NBG_ERR_CUDA, "graph instantiation failed");
        }
        B->key = key;
    }
    // ---- the queue on st, then the KD replicas of its tiles as one forest.
    // The forest's level passes are many short launches with host
    // synchronisations between levels: beside the persistent queue kernels,
    // which hold every resident block slot, each waited for free slots (the
    // forest of 256 tiles took longer than the queue itself); after the queue
    // they have the whole GPU.
    cudaEventRecord(B->ev[2], st);
    int qrc = graph ? (cudaGraphLaunch(B->exec, st) == cudaSuccess ? NBG_OK : NBG_ERR_CUDA) : record(st);
    cudaEventRecord(B->ev[3], st);
    cudaError_t qe = cudaStreamSynchronize(st);
    if (qrc || qe != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch queue launch failed");
    float kd_ms = 0;
    if (!kd_tiles.empty()) {
        cudaEventRecord(ctx->ev[8], st);
        rc = kd_ensure_many(ctx, kd_tiles.data(), (int)kd_tiles.size(), st);
        if (rc) return rc;
        cudaEventRecord(ctx->ev[9], st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch KD replicas");
        cudaEventElapsedTime(&kd_ms, ctx->ev[8], ctx->ev[9]);
    }
    // ---- exact rows per tile
    std::vector<uint32_t> cnt((size_t)nl * kCounters);
    cudaMemcpyAsync(cnt.data(), B->counters, cnt.size() * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch counters");
    uint64_t tie_rows = 0, deferred_rows = 0, replay_rows = 0, resolved = 0;
    std::vector<TieLaunch> tls;
    for (int i : live) {
        const uint32_t* c = &cnt[slot[i] * kCounters];
        tie_rows += c[1];
        deferred_rows += c[2];
        const uint32_t nties = std::min<uint32_t>(c[4], (uint32_t)items[i].tile->t.n);
        if (!nties) continue;
        Tile* t = &items[i].tile->t;
        rc = kd_ensure(ctx, t, st);
        if (rc) return rc;
        TieLaunch tl{};
        tl.tile = t;
        tl.K = Ks[i];
        tl.grp = groups[i];
        tl.grp.resolve_count = B->counters + slot[i] * kCounters + 5;
        tl.ex = ExceptionSink{B->ex_rows + ex0[i], B->counters + slot[i] * kCounters + 3,
                              std::max<uint32_t>(items[i].exception_capacity, 1)};
        tl.ties = B->ties + row0[i];
        tl.nties = nties;
        tl.kd = kd_order(t);
        tl.exact_rows = B->exact + row0[i];
        tl.counters = B->counters + slot[i] * kCounters;
        tl.ids_out = nullptr;
        tls.push_back(tl);
    }
    // every tile's tie rows in one launch
    rc = launch_ties_many(ctx, tls.data(), (int)tls.size(), st);
    if (rc) return fail(ctx, rc, "tie-order resolver");
    cudaMemcpyAsync(cnt.data(), B->counters, cnt.size() * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch tie rows");
    for (int i : live) {
        const uint32_t* c = &cnt[slot[i] * kCounters];
        if (!c[0]) continue;
        Tile* t = &items[i].tile->t;
        rc = kd_ensure(ctx, t, st);
        if (!rc) {
            const ExceptionSink sink{B->ex_rows + ex0[i], B->counters + slot[i] * kCounters + 3,
                                     std::max<uint32_t>(items[i].exception_capacity, 1)};
            StageGroup g = groups[i];
            g.resolve_count = B->counters + slot[i] * kCounters + 5;
            rc = kd_run_rows(ctx, t, Ks[i], g, sink, B->exact + row0[i], c[0], st);
        }
        if (rc) return rc;
        replay_rows += c[0];
    }
    cudaEventRecord(B->ev[4], st);
    // ---- exceptions back to each item
    cudaMemcpyAsync(cnt.data(), B->counters, cnt.size() * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch exceptions");
    bool overflow = false;
    for (int i : live) {
        const uint32_t* c = &cnt[slot[i] * kCounters];
        const uint32_t nex = c[3], capi = std::max<uint32_t>(items[i].exception_capacity, 1);
        resolved += c[5];
        if (items[i].n_exceptions) *items[i].n_exceptions = nex;
        if (nex > capi) overflow = true;
        const uint32_t m = std::min(nex, capi);
        if (m && items[i].exceptions)
            cudaMemcpyAsync(items[i].exceptions, B->ex_rows + ex0[i], m * sizeof(nbg_row_exception),
                            cudaMemcpyDeviceToHost, st);
    }
    cudaEventRecord(B->ev[5], st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, "batch exceptions");
    // the caller's stream orders after the batch
    cudaStreamWaitEvent(user, B->ev[5], 0);
    if (stats) {
        stats->points = rows;
        stats->tie_rows = tie_rows;
        stats->deferred_rows = deferred_rows;
        stats->resolved_rows = resolved;
        stats->replay_rows = replay_rows;
        float ms = 0;
        cudaEventElapsedTime(&ms, B->ev[0], B->ev[1]);
        stats->grid_ms = ms;
        cudaEventElapsedTime(&ms, B->ev[2], B->ev[3]);
        stats->query_ms = ms;
        cudaEventElapsedTime(&ms, B->ev[3], B->ev[4]);
        stats->tree_ms = ms;
        stats->kd_build_ms = kd_ms;
        cudaEventElapsedTime(&ms, B->ev[0], B->ev[5]);
        stats->total_ms = ms;
        stats->kernel_launches = g_launches.load() - launches0;
    }
    if (overflow) return fail(ctx, NBG_ERR_EXCEPTIONS, "row-exception list overflowed");
    return NBG_OK;
}

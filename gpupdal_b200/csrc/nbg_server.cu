// nbg_server.cu — the served form: a request loop with HBM-budget admission
// whose admitted requests run as waves through the batched queue.
//
// Requests queue FIFO.  `slots` host workers each own a context (its caching
// allocator, side stream, batch scratch) and a stream.  A free worker takes a
// wave: every queued request, head first, while the bytes charged to running
// requests plus the next estimate fit the budget (an idle server always
// admits its head), the wave stays within kWavePoints / kWaveItems and within
// half of this worker's share of the queued points (split over the free
// workers).  The
// wave's requests are uploaded, their grids, KD replicas and outputs held on
// the device, and all of them answered by ONE nbg_run_batch call: a
// persistent kernel per neighbour-count class drains a device queue of
// (tile, 128-query block) items across every request of the wave.  Each
// request's outputs are copied back into its own buffers and its tile freed
// as the wave ends.  Requests that arrive while a wave runs are admitted into
// the next free worker's wave (continuous batching: they wait for a worker
// and memory, not for a batch boundary), so waves of different workers
// overlap on the device.  A wave of one request, and requests the batch does
// not take (radius, optimized, strided stages, the other kNN consumers,
// stages of different knn), run the plain per-tile call instead.  The batch
// answers each tile exactly as nbg_run does, so results are the same alone
// and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nbg_internal.h"

namespace {

struct Job {
    uint64_t ticket = 0;
    nbg_request req{};
    std::vector<nbg_stage_opts> stages;
    std::vector<nbg_columns> outputs;
    uint64_t est = 0;
    double submit_us = 0;
};

using Clock = std::chrono::steady_clock;

// A wave holds at most this many requests / points (a larger queue is split
// over the free workers, so their waves overlap on the device).
constexpr size_t kWaveItems = 256;
constexpr uint64_t kWavePoints = 48ull << 20;

// The batched queue takes plain k-nearest stages that share one knn.
bool batchable(const Job& j) {
    if (j.req.n == 0 || j.stages.empty()) return false;
    for (const nbg_stage_opts& o : j.stages) {
        if (o.kind < NBG_STAGE_NORMAL || o.kind > NBG_STAGE_COVARIANCEFEATURES) return false;
        if (o.use_radius || o.optimized || (o.kind != NBG_STAGE_NORMAL && o.stride > 1)) return false;
        if (o.knn != j.stages[0].knn) return false;
    }
    return true;
}

}  // namespace

struct nbg_server {
    int device = 0;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable work_cv;  // queue or budget changed
    std::condition_variable done_cv;  // a result was posted
    std::deque<Job> queue;
    std::unordered_map<uint64_t, nbg_request_result> done;
    uint64_t next_ticket = 1;
    uint64_t charged = 0;   // estimates of running requests
    uint64_t queued_points = 0;
    int running = 0;
    int idle = 0;           // workers waiting for a wave
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<nbg_context*> contexts;
    Clock::time_point t0;
    std::string err;

    double now_us() const {
        return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    }
    void worker(int slot);
    void post(const Job& job, const nbg_request_result& res, nbg_context* ctx);
    nbg_request_result run_plain(nbg_context* ctx, const Job& job, cudaStream_t stream);
    void run_wave(nbg_context* ctx, std::vector<Job>& wave, cudaStream_t stream);
};

extern "C" uint64_t nbg_request_bytes(const nbg_request* r) {
    if (!r) return 0;
    // grid (coordinates, sorted copy, keys, cell table and column directory),
    // query scratch (row sums, tie and replay lists), KD replica (point order,
    // inverse, partition scratch, nodes), plus host-output staging per dim
    uint64_t dims = 0, extra = 0;
    if (r->n_stages > 0 && !r->outputs) return 0;
    for (int s = 0; s < r->n_stages; ++s) {
        dims += (uint64_t)r->outputs[s].ndims;
        if (!r->stages) continue;
        const nbg_stage_opts& o = r->stages[s];
        // lof keeps its ordered lists (ids and distances) and two row arrays;
        // the outlier stages a row value and a flag per point
        if (o.kind == NBG_STAGE_LOF) extra = std::max<uint64_t>(extra, 12ull * (o.knn + 1) + 16);
        if (o.kind == NBG_STAGE_OUTLIER) extra = std::max<uint64_t>(extra, 16);
    }
    return r->n * (200 + 8 * dims + extra) + (64ull << 20);
}

void nbg_server::post(const Job& job, const nbg_request_result& res, nbg_context* ctx) {
    {
        std::lock_guard<std::mutex> lk(mu);
        if (res.status != NBG_OK) err = nbg_last_error(ctx);
        charged -= job.est;
        --running;
        done[job.ticket] = res;
    }
    done_cv.notify_all();
    work_cv.notify_all();
}

// One request through the plain per-tile call.
nbg_request_result nbg_server::run_plain(nbg_context* ctx, const Job& job, cudaStream_t stream) {
    nbg_request_result res{};
    res.user_tag = job.req.user_tag;
    res.submit_us = job.submit_us;
    res.start_us = now_us();
    res.est_bytes = job.est;
    const nbg_request& q = job.req;
    nbg_tile* tile = nullptr;
    int rc = nbg_tile_upload(ctx, q.x, q.y, q.z, q.n, q.scale, q.offset, q.on_device, stream, &tile);
    if (rc == NBG_OK) {
        rc = nbg_run(ctx, tile, job.stages.data(), (int32_t)job.stages.size(), job.outputs.data(),
                     q.optimal_knn, q.optimal_radius, q.aux_on_device, q.exceptions,
                     q.exception_capacity, &res.n_exceptions, &res.stats, stream);
        nbg_tile_free(ctx, tile);
    }
    res.status = rc;
    res.end_us = now_us();
    return res;
}

// The batchable requests of a wave in one nbg_run_batch call.
void nbg_server::run_wave(nbg_context* ctx, std::vector<Job>& wave, cudaStream_t stream) {
    nbg::Context* c = &ctx->c;
    const double start = now_us();
    struct Staged {
        nbg_tile* tile = nullptr;
        std::vector<nbg_columns> cols;                      // device columns the batch writes
        std::vector<std::pair<double*, size_t>> temps;      // device blocks of this request
        const double* kopt = nullptr;
        const double* ropt = nullptr;
        uint32_t n_exc = 0;
        int rc = NBG_OK;
    };
    std::vector<Staged> sg(wave.size());
    auto temp = [&](Staged& s, size_t bytes) -> double* {
        void* p = nullptr;
        if (nbg::ctx_alloc(c, &p, bytes) != NBG_OK) return nullptr;
        s.temps.emplace_back((double*)p, bytes);
        return (double*)p;
    };
    // upload the tiles; device columns for host outputs (fresh dims zeroed,
    // others seeded with the caller's values: skipped rows keep them)
    for (size_t i = 0; i < wave.size(); ++i) {
        const Job& j = wave[i];
        const nbg_request& q = j.req;
        Staged& s = sg[i];
        s.rc = nbg_tile_upload(ctx, q.x, q.y, q.z, q.n, q.scale, q.offset, q.on_device, stream,
                               &s.tile);
        s.cols = j.outputs;
        for (size_t k = 0; k < j.outputs.size() && s.rc == NBG_OK; ++k) {
            const nbg_columns& u = j.outputs[k];
            if (u.on_device == 1 || u.ndims <= 0) continue;
            const size_t bytes = (size_t)q.n * 8 * u.ndims;
            double* d = temp(s, bytes);
            if (!d) {
                s.rc = NBG_ERR_OOM;
                break;
            }
            nbg_columns& dc = s.cols[k];
            dc.base = d;
            dc.point_stride = 8;
            dc.on_device = 1;
            for (int e = 0; e < u.ndims; ++e) dc.offset[e] = (int64_t)e * q.n * 8;
            if (u.on_device == 2) {
                if (cudaMemsetAsync(d, 0, bytes, stream)) s.rc = NBG_ERR_CUDA;
                continue;
            }
            for (int e = 0; e < u.ndims && s.rc == NBG_OK; ++e) {
                if (cudaMemcpy2DAsync(d + (size_t)e * q.n, 8, (const char*)u.base + u.offset[e],
                                      u.point_stride, 8, q.n, cudaMemcpyHostToDevice, stream))
                    s.rc = NBG_ERR_CUDA;
            }
        }
        s.kopt = q.optimal_knn;
        s.ropt = q.optimal_radius;
        if (s.rc == NBG_OK && q.optimal_knn && q.optimal_radius && !q.aux_on_device) {
            double* dk = temp(s, (size_t)q.n * 8);
            double* dr = dk ? temp(s, (size_t)q.n * 8) : nullptr;
            if (!dr) s.rc = NBG_ERR_OOM;
            else {
                s.rc = nbg::host_to_device(c, dk, q.optimal_knn, (size_t)q.n * 8, stream);
                if (s.rc == NBG_OK) s.rc = nbg::host_to_device(c, dr, q.optimal_radius, (size_t)q.n * 8, stream);
                s.kopt = dk;
                s.ropt = dr;
            }
        }
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess)
        for (Staged& s : sg) s.rc = s.rc ? s.rc : NBG_ERR_CUDA;
    std::vector<nbg_batch_item> items;
    std::vector<size_t> of;
    for (size_t i = 0; i < wave.size(); ++i) {
        if (sg[i].rc != NBG_OK) continue;
        nbg_batch_item it{};
        it.tile = sg[i].tile;
        it.n_stages = (int32_t)wave[i].stages.size();
        it.exception_capacity = wave[i].req.exception_capacity;
        it.stages = wave[i].stages.data();
        it.outputs = sg[i].cols.data();
        it.optimal_knn = sg[i].kopt;
        it.optimal_radius = sg[i].ropt;
        it.exceptions = wave[i].req.exception_capacity ? wave[i].req.exceptions : nullptr;
        it.n_exceptions = &sg[i].n_exc;
        items.push_back(it);
        of.push_back(i);
    }
    nbg_run_stats bst{};
    int brc = items.empty() ? NBG_OK
                            : nbg_run_batch(ctx, items.data(), (int32_t)items.size(), 0, &bst, stream);
    const bool batched = brc == NBG_OK || brc == NBG_ERR_EXCEPTIONS;
    for (size_t m = 0; m < of.size(); ++m) {
        const size_t i = of[m];
        Job& j = wave[i];
        Staged& s = sg[i];
        if (!batched) {
            // the batch refused the wave (e.g. a tile's extent): each request alone
            nbg_tile_free(ctx, s.tile);
            s.tile = nullptr;
            continue;
        }
        s.rc = s.n_exc > j.req.exception_capacity ? NBG_ERR_EXCEPTIONS : NBG_OK;
        // outputs back into the request's own buffers
        for (size_t k = 0; k < j.outputs.size() && s.rc == NBG_OK; ++k) {
            const nbg_columns& u = j.outputs[k];
            if (u.on_device == 1 || u.ndims <= 0) continue;
            const double* d = (const double*)s.cols[k].base;
            for (int e = 0; e < u.ndims && s.rc == NBG_OK; ++e) {
                if (u.point_stride == 8) {
                    s.rc = nbg::device_to_host(c, (char*)u.base + u.offset[e], d + (size_t)e * j.req.n,
                                               (size_t)j.req.n * 8, stream);
                } else if (cudaMemcpy2DAsync((char*)u.base + u.offset[e], u.point_stride,
                                             d + (size_t)e * j.req.n, 8, 8, j.req.n,
                                             cudaMemcpyDeviceToHost, stream) ||
                           cudaStreamSynchronize(stream)) {
                    s.rc = NBG_ERR_CUDA;
                }
            }
        }
    }
    cudaStreamSynchronize(stream);
    for (size_t i = 0; i < wave.size(); ++i) {
        Staged& s = sg[i];
        for (auto& t : s.temps) nbg::ctx_free(c, t.first, t.second);
        if (s.tile) nbg_tile_free(ctx, s.tile);
        s.tile = nullptr;
    }
    const double end = now_us();
    for (size_t i = 0; i < wave.size(); ++i) {
        const bool in_batch = std::find(of.begin(), of.end(), i) != of.end();
        if (sg[i].rc == NBG_OK && in_batch && !batched) {
            post(wave[i], run_plain(ctx, wave[i], stream), ctx);
            continue;
        }
        nbg_request_result res{};
        res.user_tag = wave[i].req.user_tag;
        res.submit_us = wave[i].submit_us;
        res.start_us = start;
        res.end_us = end;
        res.est_bytes = wave[i].est;
        res.status = sg[i].rc;
        res.n_exceptions = sg[i].n_exc;
        // the call's counters are the wave's (one batched launch)
        res.stats = bst;
        res.stats.points = wave[i].req.n;
        post(wave[i], res, ctx);
    }
}

void nbg_server::worker(int slot) {
    nbg_context* ctx = contexts[slot];
    cudaSetDevice(device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    for (;;) {
        std::vector<Job> wave;
        {
            std::unique_lock<std::mutex> lk(mu);
            ++idle;
            work_cv.wait(lk, [&] {
                if (queue.empty()) return stop;
                // FIFO: the head waits for memory; an idle server always admits
                return running == 0 || !budget || charged + queue.front().est <= budget;
            });
            // half of this worker's share of the queue: the waiting requests
            // are split into twice as many waves as there are free workers, so
            // the waves run side by side and, as each worker comes back for its
            // second, their upload, batch and copy-back phases fall out of step
            // (one wave per free worker ran all uploads, then all batches, then
            // all copies at once: 133-207 Mpts/s over three passes of the 64-
            // request stream against 185-195 with two)
            const uint64_t share =
                std::max<uint64_t>(1, queued_points / (2 * (uint64_t)std::max(idle, 1)));
            --idle;
            if (queue.empty()) break;
            uint64_t pts = 0;
            while (!queue.empty()) {
                const Job& h = queue.front();
                const bool fits = running == 0 || !budget || charged + h.est <= budget;
                if (!fits) break;
                if (!wave.empty() && (wave.size() >= kWaveItems || pts + h.req.n > kWavePoints ||
                                      pts >= share))
                    break;
                charged += h.est;
                ++running;
                pts += h.req.n;
                queued_points -= h.req.n;
                wave.push_back(std::move(queue.front()));
                queue.pop_front();
            }
        }
        // the batch takes the plain k-nearest requests; the rest, and a wave of
        // one, go through the per-tile call
        std::vector<Job> batch;
        for (Job& j : wave) {
            if (batchable(j)) batch.push_back(std::move(j));
            else post(j, run_plain(ctx, j, stream), ctx);
        }
        if (batch.size() == 1) post(batch[0], run_plain(ctx, batch[0], stream), ctx);
        else if (!batch.empty()) run_wave(ctx, batch, stream);
    }
    cudaStreamDestroy(stream);
}

extern "C" int nbg_server_create(nbg_server** out, int32_t device, int32_t slots,
                                 uint64_t hbm_budget_bytes) {
    if (!out || slots < 1 || slots > 64) return NBG_ERR_INVALID;
    *out = nullptr;
    nbg_server* s = new (std::nothrow) nbg_server();
    if (!s) return NBG_ERR_OOM;
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->t0 = Clock::now();
    for (int i = 0; i < slots; ++i) {
        nbg_context* c = nullptr;
        int rc = nbg_create(&c, device, 0);
        if (rc != NBG_OK) {
            for (nbg_context* d : s->contexts) nbg_destroy(d);
            delete s;
            return rc;
        }
        s->contexts.push_back(c);
    }
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(&nbg_server::worker, s, i);
    *out = s;
    return NBG_OK;
}

extern "C" int nbg_server_submit(nbg_server* s, const nbg_request* r, uint64_t* ticket) {
    if (!s || !r || !ticket || !r->x || !r->y || !r->z || r->n_stages < 1 || r->n_stages > 4 ||
        !r->stages || !r->outputs)
        return NBG_ERR_INVALID;
    Job job;
    job.req = *r;
    job.stages.assign(r->stages, r->stages + r->n_stages);
    job.outputs.assign(r->outputs, r->outputs + r->n_stages);
    job.est = nbg_request_bytes(r);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return NBG_ERR_INVALID;
    if (s->budget && job.est > s->budget) {
        s->err = "request footprint exceeds the server's HBM budget";
        return NBG_ERR_BUDGET;
    }
    job.ticket = s->next_ticket++;
    job.submit_us = s->now_us();
    *ticket = job.ticket;
    s->queued_points += job.req.n;
    s->queue.push_back(std::move(job));
    s->work_cv.notify_all();
    return NBG_OK;
}

extern "C" int nbg_server_wait(nbg_server* s, uint64_t ticket, int32_t timeout_ms,
                               nbg_request_result* out) {
    if (!s || !out) return NBG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket == 0 || ticket >= s->next_ticket) return NBG_ERR_INVALID;
    auto ready = [&] { return s->done.count(ticket) != 0; };
    if (timeout_ms < 0) s->done_cv.wait(lk, ready);
    else if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return NBG_ERR_TIMEOUT;
    auto it = s->done.find(ticket);
    *out = it->second;
    s->done.erase(it);
    return NBG_OK;
}

extern "C" const char* nbg_server_last_error(const nbg_server* s) {
    return s ? s->err.c_str() : "null server";
}

extern "C" int nbg_server_destroy(nbg_server* s) {
    if (!s) return NBG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    for (auto& w : s->workers) w.join();
    for (nbg_context* c : s->contexts) nbg_destroy(c);
    delete s;
    return NBG_OK;
}

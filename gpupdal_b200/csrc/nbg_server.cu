// nbg_server.cu — the served form: a request loop with HBM-budget admission.
//
// Requests queue FIFO.  `slots` host workers each own a context (its caching
// allocator, side stream and events) and a stream; a worker takes the head
// request when the bytes charged to running requests plus this request's
// estimate fit the budget, runs upload + nbg_run + free on its stream, and
// posts the result.  Requests on different slots overlap on the device; a new
// arrival starts as soon as a slot and memory are free (continuous batching),
// never waiting for a batch boundary.  Every request runs the same code path
// as the plain per-tile call, so its results do not depend on the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/nbg_b200.h"

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
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<nbg_context*> contexts;
    Clock::time_point t0;
    std::string err;

    double now_us() const {
        return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    }
    void worker(int slot);
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

void nbg_server::worker(int slot) {
    nbg_context* ctx = contexts[slot];
    cudaSetDevice(device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(mu);
            work_cv.wait(lk, [&] {
                if (queue.empty()) return stop;
                // FIFO: the head waits for memory; an idle server always admits
                return running == 0 || !budget || charged + queue.front().est <= budget;
            });
            if (queue.empty()) break;
            job = std::move(queue.front());
            queue.pop_front();
            charged += job.est;
            ++running;
        }
        nbg_request_result res{};
        res.user_tag = job.req.user_tag;
        res.submit_us = job.submit_us;
        res.start_us = now_us();
        res.est_bytes = job.est;
        const nbg_request& q = job.req;
        nbg_tile* tile = nullptr;
        int rc = nbg_tile_upload(ctx, q.x, q.y, q.z, q.n, q.scale, q.offset, q.on_device, stream,
                                 &tile);
        if (rc == NBG_OK) {
            rc = nbg_run(ctx, tile, job.stages.data(), (int32_t)job.stages.size(), job.outputs.data(),
                         q.optimal_knn, q.optimal_radius, q.aux_on_device, q.exceptions,
                         q.exception_capacity, &res.n_exceptions, &res.stats, stream);
            nbg_tile_free(ctx, tile);
        }
        res.status = rc;
        res.end_us = now_us();
        {
            std::lock_guard<std::mutex> lk(mu);
            if (rc != NBG_OK) err = nbg_last_error(ctx);
            charged -= job.est;
            --running;
            done[job.ticket] = res;
        }
        done_cv.notify_all();
        work_cv.notify_all();
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

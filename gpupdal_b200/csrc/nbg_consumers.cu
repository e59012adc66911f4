// nbg_consumers.cu — the other consumers of the same kNN index: the passes
// of filters.nndistance, filters.optimalneighborhood, filters.lof and
// filters.outlier after (or instead of) the per-row list epilogue.
//
//   nndistance, optimalneighborhood: one ordered-list pass (nbg_consumers.cuh)
//   lof: list pass (k-distance and the list), then local reachability density
//        and the outlier factor, each a pass over all rows
//        (LOFFilter.cpp:98-138)
//   outlier statistical: list pass (mean neighbour distance per row), the
//        cloud's mean and standard deviation, the threshold, the labels
//        (OutlierFilter.cpp:99-168, 171-229)
//   outlier radius: the radius kernel's count per row (OutlierFilter.cpp:80-96)
//
// The cloud's mean and variance are exact-sum reductions (double-double
// partial sums in a fixed order, so the result does not change from run to
// run); the reference's serial running moments differ from them by rounding
// only, which moves the threshold by a few ulps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "nbg_internal.h"

namespace nbg {

namespace {

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs; fixed, so the summation order is too

// Local reachability density: the inverse of the running mean of
// max(k-distance of the neighbour, distance to it) over the list.
__global__ void lof_lrd_kernel(uint64_t n, int kref, const uint32_t* __restrict__ ids,
                               const double* __restrict__ dist, const double* __restrict__ kdist,
                               double* __restrict__ lrd, StageDev st) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m1 = 0.0;
    for (int j = 0; j < kref; ++j) {
        const double k = __ldg(&kdist[__ldg(&ids[i * kref + j])]);
        const double v = __ldg(&dist[i * kref + j]);
        const double reach = k < v ? v : k;
        m1 = __dadd_rn(m1, __ddiv_rn(__dsub_rn(reach, m1), (double)(j + 1)));
    }
    const double r = __ddiv_rn(1.0, m1);
    lrd[i] = r;
    nbg_store(st, (uint32_t)i, 1, r);
}

// Local outlier factor: the running mean of lrd(neighbour) / lrd(point).
__global__ void lof_factor_kernel(uint64_t n, int kref, const uint32_t* __restrict__ ids,
                                  const double* __restrict__ lrd, StageDev st) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double lp = __ldg(&lrd[i]);
    double m1 = 0.0;
    for (int j = 0; j < kref; ++j) {
        const double ratio = __ddiv_rn(__ldg(&lrd[__ldg(&ids[i * kref + j])]), lp);
        m1 = __dadd_rn(m1, __ddiv_rn(__dsub_rn(ratio, m1), (double)(j + 1)));
    }
    nbg_store(st, (uint32_t)i, 2, m1);
}

// Double-double accumulation (Knuth's two-sum): hi + lo holds the running
// sum to about 2^-105 relative.
__device__ __forceinline__ void dd_add(double& hi, double& lo, double x) {
    const double s = __dadd_rn(hi, x);
    const double bb = __dsub_rn(s, hi);
    const double e = __dadd_rn(__dsub_rn(hi, __dsub_rn(s, bb)), __dsub_rn(x, bb));
    lo = __dadd_rn(lo, e);
    hi = __dadd_rn(s, lo);
    lo = __dsub_rn(lo, __dsub_rn(hi, s));
}

// Sum of v (center null) or of (v - *center)^2, as per-block double-double
// partials in a fixed order.
__global__ void __launch_bounds__(RED_THREADS) moment_kernel(const double* __restrict__ v, uint64_t n,
                                                             const double* center, double2* partial) {
    __shared__ double sh[RED_THREADS], sl[RED_THREADS];
    double hi = 0.0, lo = 0.0;
    const double c = center ? *center : 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)RED_THREADS + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * RED_THREADS) {
        double x = __ldg(&v[i]);
        if (center) {
            const double d = __dsub_rn(x, c);
            x = __dmul_rn(d, d);
        }
        dd_add(hi, lo, x);
    }
    sh[threadIdx.x] = hi;
    sl[threadIdx.x] = lo;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            double h = sh[threadIdx.x], l = sl[threadIdx.x];
            dd_add(h, l, sh[threadIdx.x + w]);
            dd_add(h, l, sl[threadIdx.x + w]);
            sh[threadIdx.x] = h;
            sl[threadIdx.x] = l;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(sh[0], sl[0]);
}

// stats[0] = mean (first call), or stats[1] = threshold (second call):
// mean + multiplier * sqrt(sum sq / (n - 1)).
__global__ void moment_final_kernel(const double2* partial, int blocks, uint64_t n, double* stats,
                                    int second, double multiplier) {
    if (threadIdx.x || blockIdx.x) return;
    double hi = 0.0, lo = 0.0;
    for (int b = 0; b < blocks; ++b) {
        dd_add(hi, lo, partial[b].x);
        dd_add(hi, lo, partial[b].y);
    }
    const double sum = __dadd_rn(hi, lo);
    if (!second) {
        stats[0] = __ddiv_rn(sum, (double)n);
    } else {
        const double var = __ddiv_rn(sum, __dsub_rn((double)n, 1.0));
        stats[1] = __dadd_rn(stats[0], __dmul_rn(multiplier, __dsqrt_rn(var)));
    }
}

// flag[i] = 1 when the row's mean distance is not below the threshold.
__global__ void outlier_flag_kernel(const double* __restrict__ v, uint64_t n,
                                    const double* __restrict__ stats, double* __restrict__ flag) {
    const double thr = stats[1];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = v[i] < thr ? 0.0 : 1.0;
}

__global__ void outlier_count_kernel(const double* __restrict__ flag, uint64_t n,
                                     unsigned long long* count) {
    unsigned long long c = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        c += flag[i] != 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void outlier_apply_kernel(const double* __restrict__ flag, uint64_t n, StageDev st,
                                     double label) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i] != 0.0) nbg_store(st, (uint32_t)i, 0, label);
}

unsigned grid_for(const Context* ctx, uint64_t n) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * 8));
}

// Device scratch of one consumer call, released on every path.
struct Scratch {
    Context* ctx;
    void* p[6] = {};
    size_t b[6] = {};
    int k = 0;
    explicit Scratch(Context* c) : ctx(c) {}
    template <class T>
    int get(T** out, size_t bytes) {
        int rc = ctx_alloc(ctx, (void**)out, std::max<size_t>(bytes, 16));
        if (!rc) {
            p[k] = *out;
            b[k++] = std::max<size_t>(bytes, 16);
        }
        return rc;
    }
    ~Scratch() {
        for (int i = 0; i < k; ++i) ctx_free(ctx, p[i], b[i]);
    }
};

#define CHECK_LAUNCH(what)                                                            \
    do {                                                                              \
        NBG_LAUNCHED(1);                                                              \
        cudaError_t e_ = cudaGetLastError();                                          \
        if (e_ != cudaSuccess) return fail(ctx, NBG_ERR_CUDA, std::string(what) + ": " + \
                                                              cudaGetErrorString(e_)); \
    } while (0)

// The list pass of one consumer over every row: ordered-list kernel on the
// grid, the search replay for the rows it hands over.
int list_pass(Context* ctx, Tile* t, int K, const ListArgs& L, const ExceptionSink& sink,
              cudaStream_t stream, ConsumerCounts* counts) {
    int rc = ensure_grid(ctx, t, K, stream);
    if (rc) return rc;
    rc = kd_ensure(ctx, t, stream);
    if (rc) return rc;
    if (cudaMemsetAsync(ctx->counters, 0, 5 * sizeof(uint32_t), stream))
        return fail(ctx, NBG_ERR_CUDA, "consumer counters");
    QueryLaunch ql{};
    ql.tile = t;
    ql.K = K;
    ql.rmax = 8;
    ql.ex = sink;
    ql.exact_rows = ctx->exact_rows;
    ql.counters = ctx->counters;
    rc = launch_stride(ctx, ql, 1, K, kd_order(t), stream, &L);
    if (rc) return fail(ctx, rc, "consumer list launch failed");
    uint32_t cnt[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(cnt, ctx->counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream);
    if (!e) e = cudaStreamSynchronize(stream);
    if (e) return fail(ctx, NBG_ERR_CUDA, std::string("consumer list: ") + cudaGetErrorString(e));
    counts->tie_rows += cnt[1];
    counts->replay_rows += cnt[0];
    return kd_list_rows(ctx, t, K, L, sink, ctx->exact_rows, cnt[0], stream);
}

}  // namespace

bool is_list_consumer(int kind) {
    return kind == NBG_STAGE_NNDISTANCE || kind == NBG_STAGE_OPTIMALNEIGHBORHOOD ||
           kind == NBG_STAGE_LOF || kind == NBG_STAGE_OUTLIER;
}

int run_consumer(Context* ctx, Tile* t, const nbg_stage_opts& o, int stage_index,
                 const nbg_columns& col, const ExceptionSink& sink, cudaStream_t stream,
                 ConsumerCounts* counts) {
    const uint64_t n = t->n;
    if (!n || (o.kind == NBG_STAGE_OUTLIER && o.mode == 2)) return NBG_OK;
    Scratch S(ctx);
    StageDev st{};
    fill_stage(st, o, col);
    double* flag = nullptr;  // outlier: 1 = outlier
    if (o.kind == NBG_STAGE_OUTLIER && o.mode == 1) {
        // radius method: points (the row included) with squared FP64 distance
        // below radius^2, through the radius kernel (KDImpl.hpp:398-415)
        int rc = S.get(&flag, n * 8);
        if (rc) return rc;
        const double r_raw = std::fabs(o.radius) / t->tf.scale[0];
        const int32_t cell = (int32_t)std::min(1.0e9, std::ceil(r_raw * 1.001) + 1.0);
        rc = ensure_grid(ctx, t, 8, stream, cell);
        if (rc) return rc;
        StageGroup g{};
        g.nstages = 1;
        g.stage_index[0] = stage_index;
        g.st[0] = st;
        g.st[0].aux = flag;
        g.st[0].ip = o.min_k;
        g.no_eigen = 1;
        RadiusLaunch rl;
        rl.tile = t;
        rl.grp = g;
        rl.ex = sink;
        rl.radius = o.radius;
        rl.min_k = 0;
        rc = launch_radius(ctx, rl, stream);
        if (rc) return fail(ctx, rc, "outlier radius launch failed");
    } else {
        const int kref = o.knn + (o.kind == NBG_STAGE_OPTIMALNEIGHBORHOOD ? 0 : 1);
        const int K = (int)std::min<uint64_t>(n, (uint64_t)kref);
        ListArgs L{};
        L.kind = o.kind;
        L.kref = kref;
        L.mode = o.mode;
        L.kmin = o.min_k;
        L.stage = stage_index;
        L.st = st;
        int rc = cudaMemcpyAsync(L.raw0, t->x, 4, cudaMemcpyDeviceToHost, stream) ||
                 cudaMemcpyAsync(L.raw0 + 1, t->y, 4, cudaMemcpyDeviceToHost, stream) ||
                 cudaMemcpyAsync(L.raw0 + 2, t->z, 4, cudaMemcpyDeviceToHost, stream) ||
                 cudaStreamSynchronize(stream);
        if (rc) return fail(ctx, NBG_ERR_CUDA, "point 0");
        if (o.kind == NBG_STAGE_OUTLIER || o.kind == NBG_STAGE_LOF) rc = S.get(&L.rowval, n * 8);
        if (!rc && o.kind == NBG_STAGE_LOF) rc = S.get(&L.list_ids, n * (size_t)kref * 4);
        if (!rc && o.kind == NBG_STAGE_LOF) rc = S.get(&L.list_d, n * (size_t)kref * 8);
        if (rc) return rc;
        rc = list_pass(ctx, t, K, L, sink, stream, counts);
        if (rc) return rc;
        if (o.kind == NBG_STAGE_LOF) {
            double* lrd = nullptr;
            rc = S.get(&lrd, n * 8);
            if (rc) return rc;
            const unsigned blocks = (unsigned)((n + 127) / 128);
            lof_lrd_kernel<<<blocks, 128, 0, stream>>>(n, kref, L.list_ids, L.list_d, L.rowval, lrd, st);
            CHECK_LAUNCH("lof lrd");
            lof_factor_kernel<<<blocks, 128, 0, stream>>>(n, kref, L.list_ids, lrd, st);
            CHECK_LAUNCH("lof factor");
        } else if (o.kind == NBG_STAGE_OUTLIER) {
            double2* partial = nullptr;
            double* stats = nullptr;
            rc = S.get(&flag, n * 8);
            if (!rc) rc = S.get(&partial, RED_BLOCKS * sizeof(double2));
            if (!rc) rc = S.get(&stats, 2 * sizeof(double));
            if (rc) return rc;
            moment_kernel<<<RED_BLOCKS, RED_THREADS, 0, stream>>>(L.rowval, n, nullptr, partial);
            CHECK_LAUNCH("outlier mean");
            moment_final_kernel<<<1, 32, 0, stream>>>(partial, RED_BLOCKS, n, stats, 0, o.thresh1);
            CHECK_LAUNCH("outlier mean");
            moment_kernel<<<RED_BLOCKS, RED_THREADS, 0, stream>>>(L.rowval, n, stats, partial);
            CHECK_LAUNCH("outlier variance");
            moment_final_kernel<<<1, 32, 0, stream>>>(partial, RED_BLOCKS, n, stats, 1, o.thresh1);
            CHECK_LAUNCH("outlier threshold");
            outlier_flag_kernel<<<grid_for(ctx, n), 256, 0, stream>>>(L.rowval, n, stats, flag);
            CHECK_LAUNCH("outlier flags");
        }
    }
    if (flag) {
        // OutlierFilter.cpp:171-229: labels only when inliers remain and
        // outliers exist
        unsigned long long* cnt = nullptr;
        int rc = S.get(&cnt, 8);
        if (rc) return rc;
        unsigned long long h = 0;
        cudaMemsetAsync(cnt, 0, 8, stream);
        outlier_count_kernel<<<grid_for(ctx, n), 256, 0, stream>>>(flag, n, cnt);
        CHECK_LAUNCH("outlier count");
        cudaError_t e = cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        if (e) return fail(ctx, NBG_ERR_CUDA, std::string("outlier count: ") + cudaGetErrorString(e));
        counts->outliers += h;
        counts->inliers += n - h;
        if (h && h < n) {
            outlier_apply_kernel<<<grid_for(ctx, n), 256, 0, stream>>>(flag, n, st, (double)o.label);
            CHECK_LAUNCH("outlier labels");
        }
    }
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e) return fail(ctx, NBG_ERR_CUDA, std::string("consumer stage: ") + cudaGetErrorString(e));
    return NBG_OK;
}

}  // namespace nbg

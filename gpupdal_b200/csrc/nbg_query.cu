// nbg_query.cu — fused kNN + covariance + eigensolve + stage projection.
//
// Replaces the reference's per-point loop (KD3Index::neighbors ->
// computeCovariance -> SelfAdjointEigenSolver -> projection:
// filters/NormalFilter.cpp:140-182, filters/EigenvaluesFilter.cpp:115-172,
// filters/CovarianceFeaturesFilter.cpp:204-367) and the fork's
// knnGatherKernel + eigenSystemsKernel + projection kernels
// (src/index/SpatialIndexKernels.cu:716-1086,1716-1769,
// src/stages/NeighborhoodKernels.cu:67-119,421-498).
//
// One thread per query, queries in cell order (neighbouring lanes share
// cells, so candidate loads hit L1).  The neighbour list never reaches HBM:
//   pass 1  ring expansion over cells; register top-(K+1) of exact integer
//           squared distances (FP32 FMA with a 2^23 bias yields the integer
//           in the mantissa: exact below 2^23 raw units^2)
//   check   complete iff the K-th distance is below the squared gap to the
//           unscanned cells; a row whose K-th and (K+1)-th distances are equal
//           (or whose search is incomplete within rmax rings) goes to the
//           exact KD path, which reproduces nanoflann's tie order
//   pass 2  exact int32 sums of the neighbours' offsets and outer products
//   finish  cov = (n*S2 - S1*S1^T) s^2/(n(n-1)), eigensolve, projections
// Distinct integer distances order points exactly as the reference's FP64
// distances do (the FP64 rounding error is far below one raw unit^2), so a
// row with no boundary tie has exactly the reference's neighbour set.
#include <algorithm>

#include <cub/block/block_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>

#include "nbg_common.cuh"
#include "nbg_internal.h"
#include "nbg_query.cuh"

namespace nbg {

struct Pass1 {
    float qx, qy, qz;
};

template <int KS>
struct Pass1Fn {
    float qx, qy, qz;
    TopK<KS>* top;
    // squared raw distance of the current (K+1)-th candidate: points beyond
    // it can neither enter the set nor tie with its K-th element
    __device__ __forceinline__ unsigned long long limit() const {
        const uint32_t k = top->k[KS - 1];
        return k < KEY_EXACT_END ? (unsigned long long)(k - KEY_BASE) : ~0ull;
    }
    __device__ __forceinline__ void operator()(const float4 p) {
        const uint32_t key = dist_key(p.x - qx, p.y - qy, p.z - qz);
        if (key < top->k[KS - 1]) top->insert(key);
    }
};

struct Pass2Fn {
    float qx, qy, qz;
    uint32_t kk;
    int s1x, s1y, s1z, sxx, syx, syy, szx, szy, szz, cnt;
    __device__ __forceinline__ unsigned long long limit() const {
        return (unsigned long long)(kk - KEY_BASE);
    }
    __device__ __forceinline__ void operator()(const float4 p) {
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const uint32_t key = dist_key(dx, dy, dz);
        if (key <= kk) {
            const int ix = small_int(dx), iy = small_int(dy), iz = small_int(dz);
            s1x += ix;
            s1y += iy;
            s1z += iz;
            sxx += ix * ix;
            syx += iy * ix;
            syy += iy * iy;
            szx += iz * ix;
            szy += iz * iy;
            szz += iz * iz;
            ++cnt;
        }
    }
};

struct CollectFn {
    float qx, qy, qz;
    uint32_t kk;
    uint32_t* row;
    int cnt, cap;
    __device__ __forceinline__ unsigned long long limit() const {
        return (unsigned long long)(kk - KEY_BASE);
    }
    __device__ __forceinline__ void operator()(const float4 p) {
        const uint32_t key = dist_key(p.x - qx, p.y - qy, p.z - qz);
        if (key <= kk) {
            if (cnt < cap) row[cnt] = __float_as_uint(p.w);
            ++cnt;
        }
    }
};



// Pass 1 + completeness/tie decision.  Returns true when the row is exact on
// the grid path; `R` is the final ring and `kk` the K-th key.
template <int KS>
__device__ __forceinline__ bool select_kth(const QueryArgs& a, const GridParams& g,
                                           const QueryCell& qc, const float4 q, int K, int& R,
                                           uint32_t& kk, bool& tie) {
    tie = false;
    const int off = KS - (K + 1);
    TopK<KS> top;
    top.init(off);
    Pass1Fn<KS> f1{q.x, q.y, q.z, &top};
    bool complete = false;
    const int rmax = a.rmax;
    for (R = 0; R <= rmax; ++R) {
        scan_shell(a.gv, g, qc, R, f1);
        const uint32_t kth = top.at(off + K - 1);
        const unsigned long long gap2 = outside_gap2(g, qc, R);
        if (gap2 == ~0ull) {
            complete = kth != 0xFFFFFFFFu;
            break;
        }
        if (kth < KEY_EXACT_END && (unsigned long long)(kth - KEY_BASE) < gap2) {
            complete = true;
            break;
        }
    }
    if (R > rmax) R = rmax;
    kk = top.at(off + K - 1);
    const uint32_t kk1 = top.at(off + K);
    if (!complete || kk >= KEY_EXACT_END) {
        atomicAdd(&a.counters[2], 1u);
        return false;
    }
    if (kk1 == kk) {
        atomicAdd(&a.counters[1], 1u);
        tie = true;
        return false;
    }
    return true;
}

template <int KS>
__global__ void __launch_bounds__(128) knn_fused_kernel(const QueryArgs a) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    const int K = a.K;
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    int R;
    uint32_t kk;
    bool tie;
    if (!select_kth<KS>(a, g, qc, q, K, R, kk, tie)) {
        defer_row(a, id, tie, kk, R);
        return;
    }
    Pass2Fn f2{q.x, q.y, q.z, kk, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int r = 0; r <= R; ++r) scan_shell(a.gv, g, qc, r, f2);
    if (f2.cnt != a.K) {  // cannot happen for a complete, tie-free row; stay exact
        const uint32_t slot = atomicAdd(&a.counters[0], 1u);
        a.exact_rows[slot] = id;
        return;
    }
    const long long n = f2.cnt;
    long long M[6];
    M[0] = n * f2.sxx - (long long)f2.s1x * f2.s1x;
    M[1] = n * f2.syx - (long long)f2.s1y * f2.s1x;
    M[2] = n * f2.syy - (long long)f2.s1y * f2.s1y;
    M[3] = n * f2.szx - (long long)f2.s1z * f2.s1x;
    M[4] = n * f2.szy - (long long)f2.s1z * f2.s1y;
    M[5] = n * f2.szz - (long long)f2.s1z * f2.s1z;
    const int32_t qraw[3] = {qc.qx + g.minx, qc.qy + g.miny, qc.qz + g.minz};
    nbg_finish_row(a.grp, a.tf, a.ex, id, (int)n, M, qraw);
}

// Split form, pass 1 + pass 2: the row's exact neighbourhood sums, in sorted
// order (cnt = 0 marks a row handed to the exact path).  With FINISH the row
// is finished in place instead and its sums are not written (the handed-back
// rows of the single-pass select, whose sums slot already holds cnt = 0).
template <int KS, bool FINISH = false>
__device__ __forceinline__ void select_row(const QueryArgs& a, const uint64_t i) {
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    const int K = row_neighbours(a.row_k, a.K, a.n, id);
    if (K <= 0) {
        // no neighbours: the reference's covariance of an empty set is zero
        const long long M[6] = {0, 0, 0, 0, 0, 0};
        const int32_t qraw[3] = {__float2int_rz(q.x) + g.minx, __float2int_rz(q.y) + g.miny,
                                 __float2int_rz(q.z) + g.minz};
        nbg_finish_row(a.grp, a.tf, a.ex, id, 0, M, qraw);
        if (!FINISH) {
            RowSums z;
            z.cnt = 0;
            a.sums[i] = z;
        }
        return;
    }
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    int R;
    uint32_t kk;
    bool tie;
    RowSums out;
    out.cnt = 0;
    if (!select_kth<KS>(a, g, qc, q, K, R, kk, tie)) {
        defer_row(a, id, tie, kk, R);
        if (!FINISH) a.sums[i] = out;
        return;
    }
    Pass2Fn f2{q.x, q.y, q.z, kk, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int r = 0; r <= R; ++r) scan_shell(a.gv, g, qc, r, f2);
    if (f2.cnt != K) {
        defer_row(a, id, false, kk, R);
        if (!FINISH) a.sums[i] = out;
        return;
    }
    if (FINISH) {
        const long long n = f2.cnt;
        long long M[6];
        M[0] = n * f2.sxx - (long long)f2.s1x * f2.s1x;
        M[1] = n * f2.syx - (long long)f2.s1y * f2.s1x;
        M[2] = n * f2.syy - (long long)f2.s1y * f2.s1y;
        M[3] = n * f2.szx - (long long)f2.s1z * f2.s1x;
        M[4] = n * f2.szy - (long long)f2.s1z * f2.s1y;
        M[5] = n * f2.szz - (long long)f2.s1z * f2.s1z;
        const int32_t qraw[3] = {qc.qx + g.minx, qc.qy + g.miny, qc.qz + g.minz};
        nbg_finish_row(a.grp, a.tf, a.ex, id, (int)n, M, qraw);
        return;
    }
    out.s[0] = f2.s1x;
    out.s[1] = f2.s1y;
    out.s[2] = f2.s1z;
    out.s[3] = f2.sxx;
    out.s[4] = f2.syx;
    out.s[5] = f2.syy;
    out.s[6] = f2.szx;
    out.s[7] = f2.szy;
    out.s[8] = f2.szz;
    out.cnt = f2.cnt;
    a.sums[i] = out;
}

template <int KS>
__global__ void __launch_bounds__(128) knn_select_kernel(const QueryArgs a) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= (a.rows ? a.nq : a.n)) return;
    if (a.rows) i = __ldg(&a.rows[i]);
    select_row<KS>(a, i);
}

// ---------------------------------------------------------------------------
// Single-pass select: the ring search of select_kth with keys that say where
// the candidate lies, so the row's K nearest are read back directly instead
// of re-scanning the rings for their sums (the second pass is about 40 % of
// the two-pass kernel).  A key is
//     d2 << (ob + 5) | slot << ob | offset
// with d2 the exact integer squared distance (saturated at the field's top),
// slot = (dx + 2) * 5 + (dy + 2) the candidate's column among the 5 x 5
// around the query's, and offset its position in that column's run of cells
// (from the column's first point).  Keys order as squared distances (the low
// fields only separate equal distances, which the tie test compares without
// them).  ob is chosen per tile so that d2 holds (2.2 c)^2 for cell edge c.
// Rows this form cannot answer exactly -- a search past ring 2, an offset or
// a K-th distance beyond its field, no neighbours at all -- go to the retry
// list, which the two-pass kernel answers.
struct LocFn {
    float qx, qy, qz;
    uint32_t ob;        // offset bits
    uint32_t ib;        // index bits: ob + 5
    uint32_t d2max;     // saturated squared distance
    uint32_t colkey;    // the current column's slot << ob
    uint32_t colbase;   // the current column's first point
    bool bad;           // an inserted candidate's offset did not fit
};

template <int KS>
__device__ __forceinline__ unsigned long long loc_limit(const TopK<KS>& top, const LocFn& f) {
    const uint32_t d2 = top.k[KS - 1] >> f.ib;
    return d2 >= f.d2max ? ~0ull : (unsigned long long)d2;
}

template <int KS>
__device__ __forceinline__ void loc_candidate(TopK<KS>& top, LocFn& f, const float4 p, uint32_t j) {
    const uint32_t key = dist_key(p.x - f.qx, p.y - f.qy, p.z - f.qz);
    const uint32_t d2 = key < KEY_EXACT_END ? min(key - KEY_BASE, f.d2max) : f.d2max;
    const uint32_t cand = d2 << f.ib;
    if (cand < (top.k[KS - 1] & ~((1u << f.ib) - 1u))) {
        const uint32_t off = j - f.colbase;
        if (off >> f.ob) f.bad = true;
        top.insert(cand | f.colkey | (off & ((1u << f.ob) - 1u)));
    }
}

// Ring R of the located search (R <= 2): scan_shell's columns and z-reach,
// with each column's slot and first point set before its points are keyed.
template <int KS>
__device__ __forceinline__ void loc_shell(const GridView& gv, const GridParams& g, const QueryCell& qc,
                                          int R, TopK<KS>& top, LocFn& f) {
    const int zlo = qc.cz - R, zhi = qc.cz + R;
    const int c = g.cell;
    for (int dy = -R; dy <= R; ++dy) {
        const int y = qc.cy + dy;
        if (y < 0 || y >= g.gy) continue;
        const int ady = dy < 0 ? -dy : dy;
        const int gy_ = slab_gap(qc.qy, y, c);
        for (int dx = -R; dx <= R; ++dx) {
            const int x = qc.cx + dx;
            if (x < 0 || x >= g.gx) continue;
            const int gx_ = slab_gap(qc.qx, x, c);
            const long long h2 = (long long)gx_ * gx_ + (long long)gy_ * gy_;
            const unsigned long long lim = loc_limit(top, f);
            if ((unsigned long long)h2 > lim) continue;
            const int4 ci = __ldg(&gv.colinfo[(uint32_t)y * (uint32_t)g.gx + (uint32_t)x]);
            if (ci.z < ci.y) continue;
            int zr0 = zlo, zr1 = zhi;
            if (lim < (1ull << 46)) {
                const float s = sqrtf((float)(lim - (unsigned long long)h2)) + 1.0f;
                zr0 = max(zr0, (int)floorf(((float)qc.qz - s) / (float)c));
                zr1 = min(zr1, (int)floorf(((float)qc.qz + s) / (float)c));
            }
            f.colkey = (uint32_t)((dx + 2) * 5 + (dy + 2)) << f.ob;
            f.colbase = __ldg(&gv.cstart[(uint32_t)ci.x]);
            const int adx = dx < 0 ? -dx : dx;
            auto run = [&](int zl, int zh) {
                zl = max(zl, ci.y);
                zh = min(zh, ci.z);
                if (zl > zh) return;
                const uint32_t e0 = (uint32_t)ci.x + (uint32_t)(zl - ci.y);
                const uint32_t e1 = (uint32_t)ci.x + (uint32_t)(zh - ci.y) + 1;
                const uint32_t pe = __ldg(&gv.cstart[e1]);
                for (uint32_t j = __ldg(&gv.cstart[e0]); j < pe; ++j)
                    loc_candidate(top, f, __ldg(&gv.sorted[j]), j);
            };
            if (max(ady, adx) == R) {
                run(zr0, zr1);
            } else {
                if (zlo >= zr0 && zlo <= zr1) run(zlo, zlo);
                if (zhi >= zr0 && zhi <= zr1) run(zhi, zhi);
            }
        }
    }
}

template <int KS>
__device__ __forceinline__ void select_row_loc(const QueryArgs& a, const uint64_t i, uint32_t ob) {
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    const int K = row_neighbours(a.row_k, a.K, a.n, id);
    auto retry = [&]() {
        const uint32_t slot = atomicAdd(&a.counters[6], 1u);
        a.retry_rows[slot] = (uint32_t)i;
        a.sums[i].cnt = 0;  // the finish pass leaves the row to the retry launch
    };
    if (K <= 0) {
        retry();
        return;
    }
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    const int off = KS - (K + 1);
    TopK<KS> top;
    top.init(off);
    LocFn f;
    f.qx = q.x;
    f.qy = q.y;
    f.qz = q.z;
    f.ob = ob;
    f.ib = ob + 5;
    f.d2max = (1u << (27 - ob)) - 1u;
    f.bad = false;
    bool complete = false;
    int R;
    for (R = 0; R <= 2; ++R) {
        loc_shell(a.gv, g, qc, R, top, f);
        const uint32_t kd = top.at(off + K - 1) >> f.ib;
        const unsigned long long gap2 = outside_gap2(g, qc, R);
        if (gap2 == ~0ull) {
            complete = kd < f.d2max;
            break;
        }
        if (kd < f.d2max && (unsigned long long)kd < gap2) {
            complete = true;
            break;
        }
    }
    const uint32_t kk = top.at(off + K - 1) >> f.ib;
    const uint32_t kk1 = top.at(off + K) >> f.ib;
    if (!complete || f.bad || kk >= f.d2max || kk >= (1u << 23)) {
        retry();
        return;
    }
    if (kk1 == kk) {
        atomicAdd(&a.counters[1], 1u);
        defer_row(a, id, true, KEY_BASE + kk, R);
        RowSums z;
        z.cnt = 0;
        a.sums[i] = z;
        return;
    }
    int s1x = 0, s1y = 0, s1z = 0, sxx = 0, syx = 0, syy = 0, szx = 0, szy = 0, szz = 0;
    const uint32_t omask = (1u << f.ob) - 1u;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        if (s >= off && s < off + K) {
            const uint32_t idx = top.k[s];
            const uint32_t slot = (idx >> f.ob) & 31u;
            const int dx = (int)(slot / 5) - 2, dy = (int)(slot % 5) - 2;
            const int4 ci = __ldg(&a.gv.colinfo[(uint32_t)(qc.cy + dy) * (uint32_t)g.gx +
                                                (uint32_t)(qc.cx + dx)]);
            const float4 p = __ldg(&a.gv.sorted[__ldg(&a.gv.cstart[(uint32_t)ci.x]) + (idx & omask)]);
            const int ix = small_int(p.x - q.x), iy = small_int(p.y - q.y), iz = small_int(p.z - q.z);
            s1x += ix;
            s1y += iy;
            s1z += iz;
            sxx += ix * ix;
            syx += iy * ix;
            syy += iy * iy;
            szx += iz * ix;
            szy += iz * iy;
            szz += iz * iz;
        }
    }
    RowSums out;
    out.s[0] = s1x;
    out.s[1] = s1y;
    out.s[2] = s1z;
    out.s[3] = sxx;
    out.s[4] = syx;
    out.s[5] = syy;
    out.s[6] = szx;
    out.s[7] = szy;
    out.s[8] = szz;
    out.cnt = K;
    a.sums[i] = out;
}

template <int KS>
__global__ void __launch_bounds__(128) knn_select_loc_kernel(const QueryArgs a, const uint32_t ob) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= (a.rows ? a.nq : a.n)) return;
    if (a.rows) i = __ldg(&a.rows[i]);
    select_row_loc<KS>(a, i, ob);
}

// The per-thread select with the queries of each block of 256 rows re-sorted
// by a Morton key of their coordinates (block-local radix sort): a warp's 32
// lanes are then spatially compact, so their ring searches visit nearly the
// same cells (rows in cell order are random points of a cell that spans
// several warps).
template <int KS>
__global__ void __launch_bounds__(256) knn_select_morton_kernel(const QueryArgs a) {
    using Sort = cub::BlockRadixSort<uint32_t, 256, 1, uint32_t>;
    __shared__ typename Sort::TempStorage sort_tmp;
    __shared__ int s_box[6];
    const uint64_t nrows = a.rows ? a.nq : a.n;
    const uint64_t r0 = (uint64_t)blockIdx.x * 256u;
    if (r0 >= nrows) return;
    const int tid = threadIdx.x;
    const uint32_t nvalid = (uint32_t)min((uint64_t)256, nrows - r0);
    uint32_t key[1], val[1];
    block_morton_order<256>(a, r0, nvalid, s_box, key, val);
    Sort(sort_tmp).Sort(key, val, 0, 31);  // rows past the end sort last
    if (tid < (int)nvalid) select_row<KS>(a, val[0]);
}

// Split form, finish: covariance, eigensolve and stage projections of the
// rows the select kernel completed.  Uniform work per thread.
__device__ __forceinline__ void finish_row(const QueryArgs& a, const uint64_t i) {
    const RowSums r = a.sums[i];
    if (r.cnt == 0) return;
    const GridParams* gp = a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    const long long n = r.cnt;
    long long M[6];
    M[0] = n * r.s[3] - (long long)r.s[0] * r.s[0];
    M[1] = n * r.s[4] - (long long)r.s[1] * r.s[0];
    M[2] = n * r.s[5] - (long long)r.s[1] * r.s[1];
    M[3] = n * r.s[6] - (long long)r.s[2] * r.s[0];
    M[4] = n * r.s[7] - (long long)r.s[2] * r.s[1];
    M[5] = n * r.s[8] - (long long)r.s[2] * r.s[2];
    const int32_t qraw[3] = {__float2int_rz(q.x) + __ldg(&gp->minx), __float2int_rz(q.y) + __ldg(&gp->miny),
                             __float2int_rz(q.z) + __ldg(&gp->minz)};
    nbg_finish_row(a.grp, a.tf, a.ex, id, (int)n, M, qraw);
}

// Autotuning sample: runs of `run` consecutive blocks of 128 rows, run g
// starting at row g*stride (neighbouring blocks share cells, as in a full
// launch, so the sample sees the full launch's cache behaviour).
template <int KS>
__global__ void __launch_bounds__(128) knn_select_sample_kernel(const QueryArgs a, uint64_t stride,
                                                                unsigned run) {
    const uint64_t i = (blockIdx.x / run) * stride + (blockIdx.x % run) * 128ull + threadIdx.x;
    if (i < a.n) select_row<KS>(a, i);
}

__global__ void __launch_bounds__(128) knn_finish_kernel(const QueryArgs a) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= (a.rows ? a.nq : a.n)) return;
    if (a.rows) i = __ldg(&a.rows[i]);
    finish_row(a, i);
}

// ---------------------------------------------------------------------------
// Batched form: persistent kernels draining one device work queue of
// (tile, block of 128 queries) items, tiles of any size in one launch.  A
// block takes the next item with one atomic, finds its tile by binary search
// over the jobs' first items, and answers the item's queries exactly as the
// per-tile kernels do.
__device__ __forceinline__ bool next_item(const BatchJob* __restrict__ jobs, int njobs,
                                          uint64_t items, unsigned long long* head,
                                          uint64_t& item, int& job) {
    __shared__ unsigned long long s_item;
    __shared__ int s_job;
    if (threadIdx.x == 0) {
        const unsigned long long it = atomicAdd(head, 1ull);
        int lo = 0, hi = njobs;
        if (it < items) {
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (jobs[mid].first <= it) lo = mid;
                else hi = mid;
            }
        }
        s_item = it;
        s_job = lo;
    }
    __syncthreads();
    item = s_item;
    job = s_job;
    __syncthreads();
    return item < items;
}

template <int KS>
__global__ void __launch_bounds__(128) knn_select_queue_kernel(const BatchJob* __restrict__ jobs,
                                                               int njobs, uint64_t items,
                                                               unsigned long long* head) {
    uint64_t item;
    int j;
    while (next_item(jobs, njobs, items, head, item, j)) {
        const QueryArgs& a = jobs[j].q;
        const uint64_t i = (item - jobs[j].first) * 128u + threadIdx.x;
        if (i < a.n) select_row<KS>(a, i);
    }
}

__global__ void __launch_bounds__(128) knn_finish_queue_kernel(const BatchJob* __restrict__ jobs,
                                                               int njobs, uint64_t items,
                                                               unsigned long long* head) {
    uint64_t item;
    int j;
    while (next_item(jobs, njobs, items, head, item, j)) {
        const QueryArgs& a = jobs[j].q;
        const uint64_t i = (item - jobs[j].first) * 128u + threadIdx.x;
        if (i < a.n) finish_row(a, i);
    }
}

struct QueueArgs {
    const BatchJob* jobs;
    int njobs;
    uint64_t items;
    unsigned long long* head;
    int sms;
    cudaStream_t stream;
    int reserve;  // resident blocks per SM left to kernels of other streams
};

template <int KS>
struct QueueLauncher {
    using Args = QueueArgs;
    static int run(const QueueArgs& q) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, knn_select_queue_kernel<KS>, 128, 0);
        const uint64_t grid =
            std::min<uint64_t>(q.items, (uint64_t)q.sms * std::max(per_sm - q.reserve, 1));
        if (!grid) return NBG_OK;
        knn_select_queue_kernel<KS><<<(unsigned)grid, 128, 0, q.stream>>>(q.jobs, q.njobs, q.items,
                                                                           q.head);
        NBG_LAUNCHED(1);
        return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
    }
};

template <int KS>
__device__ __forceinline__ void ids_row(const QueryArgs& a, const uint64_t i) {
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    const int K = a.K;
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    int R;
    uint32_t kk;
    bool tie;
    if (!select_kth<KS>(a, g, qc, q, K, R, kk, tie)) {
        defer_row(a, id, tie, kk, R);
        return;
    }
    uint32_t* row = a.ids_out + (uint64_t)id * a.K;
    CollectFn f{q.x, q.y, q.z, kk, row, 0, a.K};
    for (int r = 0; r <= R; ++r) scan_shell(a.gv, g, qc, r, f);
    // ascending ids (insertion sort of at most 66 entries)
    for (int s = 1; s < a.K; ++s) {
        uint32_t v = row[s];
        int t = s - 1;
        while (t >= 0 && row[t] > v) {
            row[t + 1] = row[t];
            --t;
        }
        row[t + 1] = v;
    }
}

template <int KS>
__global__ void __launch_bounds__(128) knn_ids_kernel(const QueryArgs a) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < a.n) ids_row<KS>(a, i);
}

// Rows the group select handed back (a.rows, a.nq_dev entries), answered by
// the per-thread ring search: neighbour sums, or the neighbour-set export.
template <int KS>
__global__ void __launch_bounds__(128) knn_retry_kernel(const QueryArgs a) {
    const uint32_t nr = *a.nq_dev;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += gridDim.x * blockDim.x) {
        const uint32_t i = __ldg(&a.rows[r]);
        if (a.ids_out) ids_row<KS>(a, i);
        else select_row<KS>(a, i);
    }
}

// Rows the single-pass select handed back, answered by the per-thread ring
// search and finished in place (their sums slots hold cnt = 0, so the finish
// pass over the other rows, which may run at the same time, skips them).  A
// few of these rows search far and set the launch's length, so it runs beside
// that finish pass rather than before it.
template <int KS>
__global__ void __launch_bounds__(128) knn_retry_finish_kernel(const QueryArgs a) {
    const uint32_t nr = *a.nq_dev;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += gridDim.x * blockDim.x)
        select_row<KS, true>(a, __ldg(&a.rows[r]));
}

// ---------------------------------------------------------------------------
// Tie-order resolver.
//
// In a tie row the points strictly inside the K-th distance D_K are the
// reference's, and the remaining m = K - less slots go to points at integer
// distance D_K.  Among those the reference keeps the smallest FP64 distances
// and, at equal FP64 distance, the ones its depth-first search meets first
// (nanoflann.hpp:178-205, :1191-1197): while fewer than m of them have been
// admitted the result set holds fewer than K points within D_K, so its worst
// distance exceeds D_K and no subtree holding one of them is pruned.  The
// search meets points of one leaf in the tree's point order and, for points in
// different leaves, first the side of their lowest common node that the query
// visits first (nanoflann.hpp:1226-1236: child1 iff (q-divlow)+(q-divhigh) < 0).
// Ordering that group therefore needs the replica's tree but not its search.
static constexpr int TIE_CAP = 32;

// True when the reference's search meets replica position pa before pb.
__device__ __forceinline__ bool kd_meets_first(const KdOrder& kd, const double q[3], uint32_t pa,
                                               uint32_t pb) {
    int node = kd.root;
    for (int depth = 0; depth < 64; ++depth) {
        const int a = __ldg(&kd.c1[node]);
        if (a < 0) break;
        const uint32_t split = __ldg(&kd.ne[a]);
        const bool la = pa < split, lb = pb < split;
        if (la == lb) {
            node = la ? a : __ldg(&kd.c2[node]);
            continue;
        }
        const double val = q[__ldg(&kd.feat[node])];
        const bool left_first =
            __dadd_rn(__dsub_rn(val, __ldg(&kd.dlo[node])), __dsub_rn(val, __ldg(&kd.dhi[node]))) < 0;
        return la == left_first;
    }
    return pa < pb;
}

struct TieFn {
    float qx, qy, qz;
    uint32_t kk;
    int s1x, s1y, s1z, sxx, syx, syy, szx, szy, szz, less;
    int gcnt;
    uint32_t gid[TIE_CAP];
    int gd[TIE_CAP][3];
    uint32_t* row;  // neighbour-set export: ids of the strictly closer points
    int K;
    __device__ __forceinline__ unsigned long long limit() const {
        return (unsigned long long)(kk - KEY_BASE);
    }
    __device__ __forceinline__ void add(int ix, int iy, int iz) {
        s1x += ix;
        s1y += iy;
        s1z += iz;
        sxx += ix * ix;
        syx += iy * ix;
        syy += iy * iy;
        szx += iz * ix;
        szy += iz * iy;
        szz += iz * iz;
    }
    __device__ __forceinline__ void operator()(const float4 p) {
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const uint32_t key = dist_key(dx, dy, dz);
        if (key < kk) {
            add(small_int(dx), small_int(dy), small_int(dz));
            if (row && less < K) row[less] = __float_as_uint(p.w);
            ++less;
        } else if (key == kk) {
            if (gcnt < TIE_CAP) {
                gid[gcnt] = __float_as_uint(p.w);
                gd[gcnt][0] = small_int(dx);
                gd[gcnt][1] = small_int(dy);
                gd[gcnt][2] = small_int(dz);
            }
            ++gcnt;
        }
    }
};

struct TieArgs {
    GridView gv;
    const GridParams* gp;
    uint64_t n;
    const double* row_k;
    const int32_t* x;  // raw coordinates in caller order
    const int32_t* y;
    const int32_t* z;
    int K;
    StageGroup grp;
    Transform tf;
    ExceptionSink ex;
    const uint2* ties;
    uint32_t nties;
    KdOrder kd;
    uint32_t* exact_rows;
    uint32_t* counters;
    uint32_t* ids_out;
};

// One tie row r of a.ties.
__device__ __forceinline__ void tie_row(const TieArgs& a, uint32_t r) {
    const uint2 e = a.ties[r];
    const uint32_t id = e.x;
    const uint32_t kk = KEY_BASE + (e.y & 0xFFFFFFu);
    const int R = (int)(e.y >> 24);
    const GridParams g = *a.gp;
    const int K = row_neighbours(a.row_k, a.K, a.n, id);
    const int32_t qraw[3] = {__ldg(&a.x[id]), __ldg(&a.y[id]), __ldg(&a.z[id])};
    QueryCell qc;
    qc.qx = qraw[0] - g.minx;
    qc.qy = qraw[1] - g.miny;
    qc.qz = qraw[2] - g.minz;
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    TieFn f;
    f.qx = (float)qc.qx;
    f.qy = (float)qc.qy;
    f.qz = (float)qc.qz;
    f.kk = kk;
    f.s1x = f.s1y = f.s1z = f.sxx = f.syx = f.syy = f.szx = f.szy = f.szz = 0;
    f.less = 0;
    f.gcnt = 0;
    f.row = a.ids_out ? a.ids_out + (uint64_t)id * a.K : nullptr;
    f.K = K;
    for (int ring = 0; ring <= R; ++ring) scan_shell(a.gv, g, qc, ring, f);
    const int m = K - f.less;
    if (f.gcnt > TIE_CAP || m <= 0 || m > f.gcnt) {
        const uint32_t slot = atomicAdd(&a.counters[0], 1u);
        a.exact_rows[slot] = id;
        return;
    }
    // the reference's FP64 distances of the group (nanoflann's L2 adaptor
    // sums the squared differences left to right)
    const double q64[3] = {ref_coord(qraw[0], a.tf.scale[0], a.tf.offset[0]),
                           ref_coord(qraw[1], a.tf.scale[1], a.tf.offset[1]),
                           ref_coord(qraw[2], a.tf.scale[2], a.tf.offset[2])};
    double d64[TIE_CAP];
    for (int t = 0; t < f.gcnt; ++t) {
        double acc = 0.0;
        for (int d = 0; d < 3; ++d) {
            const double pc = ref_coord(qraw[d] + f.gd[t][d], a.tf.scale[d], a.tf.offset[d]);
            const double df = __dsub_rn(q64[d], pc);
            acc = __dadd_rn(acc, __dmul_rn(df, df));
        }
        d64[t] = acc;
    }
    // Members at equal FP64 distance are taken in the search's visiting order.
    // Without a neighbour-id export only their offsets reach the sums: when every
    // member at the m-th smallest FP64 distance has the same offsets (duplicate
    // points, most of a lidar tile's tie groups), any of them gives the same
    // sums, and the row needs no walk down the tree.  (The test is per row: a
    // member skipped as "equivalent" in a pairwise walk would stand in for its
    // twin in later comparisons with the other members and break the order.)
    bool any_order = f.row == nullptr;
    if (any_order) {
        double v = 0.0;  // the m-th smallest FP64 distance
        for (int t = 0; t < f.gcnt; ++t) {
            int less = 0, le = 0;
            for (int u = 0; u < f.gcnt; ++u) {
                less += d64[u] < d64[t];
                le += d64[u] <= d64[t];
            }
            if (less < m && m <= le) v = d64[t];
        }
        int ref = -1;
        for (int t = 0; t < f.gcnt && any_order; ++t) {
            if (d64[t] != v) continue;
            if (ref < 0) ref = t;
            else if (f.gd[t][0] != f.gd[ref][0] || f.gd[t][1] != f.gd[ref][1] ||
                     f.gd[t][2] != f.gd[ref][2])
                any_order = false;
        }
    }
    uint32_t taken = 0;
    for (int j = 0; j < m; ++j) {
        int best = -1;
        for (int t = 0; t < f.gcnt; ++t) {
            if ((taken >> t) & 1u) continue;
            if (best < 0 || d64[t] < d64[best] ||
                (d64[t] == d64[best] && !any_order &&
                 kd_meets_first(a.kd, q64, __ldg(&a.kd.kpos[a.kd.base + f.gid[t]]),
                                __ldg(&a.kd.kpos[a.kd.base + f.gid[best]]))))
                best = t;
        }
        taken |= 1u << best;
        f.add(f.gd[best][0], f.gd[best][1], f.gd[best][2]);
        if (f.row) f.row[f.less + j] = f.gid[best];
    }
    if (f.row) {
        uint32_t* row = f.row;
        for (int s = 1; s < K; ++s) {
            const uint32_t v = row[s];
            int t = s - 1;
            while (t >= 0 && row[t] > v) {
                row[t + 1] = row[t];
                --t;
            }
            row[t + 1] = v;
        }
        return;
    }
    const long long n = K;
    long long M[6];
    M[0] = n * f.sxx - (long long)f.s1x * f.s1x;
    M[1] = n * f.syx - (long long)f.s1y * f.s1x;
    M[2] = n * f.syy - (long long)f.s1y * f.s1y;
    M[3] = n * f.szx - (long long)f.s1z * f.s1x;
    M[4] = n * f.szy - (long long)f.s1z * f.s1y;
    M[5] = n * f.szz - (long long)f.s1z * f.s1z;
    nbg_finish_row(a.grp, a.tf, a.ex, id, (int)n, M, qraw);
}

__global__ void __launch_bounds__(128) knn_tie_kernel(const TieArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < a.nties) tie_row(a, r);
}

// Tie rows counted on the device (a.nties: the list's capacity).
__global__ void __launch_bounds__(128) knn_tie_counted_kernel(const TieArgs a, const uint32_t* count) {
    const uint32_t nt = min(*count, a.nties);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nt; r += gridDim.x * blockDim.x)
        tie_row(a, r);
}

// The tie rows of many tiles in one launch: jobs[j] is tile j's arguments,
// its rows are entries first[j] .. first[j+1]-1 of the launch.
__global__ void __launch_bounds__(128) knn_tie_batch_kernel(const TieArgs* __restrict__ jobs,
                                                            const uint64_t* __restrict__ first,
                                                            int njobs) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= first[njobs]) return;
    int lo = 0, hi = njobs;  // the job whose range holds t
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= t) lo = mid;
        else hi = mid;
    }
    tie_row(jobs[lo], (uint32_t)(t - first[lo]));
}

static TieArgs tie_args(const TieLaunch& tl) {
    TieArgs a;
    a.gv = grid_view(tl.tile);
    a.gp = tl.tile->gp;
    a.n = tl.tile->n;
    a.row_k = tl.row_k;
    a.x = tl.tile->x;
    a.y = tl.tile->y;
    a.z = tl.tile->z;
    a.K = tl.K;
    a.grp = tl.grp;
    a.tf = tl.tile->tf;
    a.ex = tl.ex;
    a.ties = tl.ties;
    a.nties = tl.nties;
    a.kd = tl.kd;
    a.exact_rows = tl.exact_rows;
    a.counters = tl.counters;
    a.ids_out = tl.ids_out;
    return a;
}

int launch_ties(Context* ctx, const TieLaunch& tl, cudaStream_t stream) {
    (void)ctx;
    if (!tl.nties) return NBG_OK;
    knn_tie_kernel<<<(tl.nties + 127) / 128, 128, 0, stream>>>(tie_args(tl));
    NBG_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

// The grid covers a few per cent of a tile at one row per thread (tie rows
// are 3 % of the 32M-point stress tile); a longer list is walked in strides.
static constexpr uint64_t kTieBlocksPerSm = 16;

int launch_ties_counted(Context* ctx, const TieLaunch& tl, const uint32_t* count, cudaStream_t stream) {
    if (!tl.nties) return NBG_OK;
    const uint64_t sms = ctx ? (uint64_t)ctx->sm_count : 148;
    const unsigned blocks = (unsigned)std::min<uint64_t>(((uint64_t)tl.nties + 127) / 128, sms * kTieBlocksPerSm);
    knn_tie_counted_kernel<<<blocks, 128, 0, stream>>>(tie_args(tl), count);
    NBG_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

int launch_ties_many(Context* ctx, const TieLaunch* tls, int count, cudaStream_t stream) {
    std::vector<TieArgs> jobs;
    std::vector<uint64_t> first(1, 0);
    for (int i = 0; i < count; ++i) {
        if (!tls[i].nties) continue;
        jobs.push_back(tie_args(tls[i]));
        first.push_back(first.back() + tls[i].nties);
    }
    if (jobs.empty()) return NBG_OK;
    TieArgs* djobs = nullptr;
    uint64_t* dfirst = nullptr;
    const size_t jb = jobs.size() * sizeof(TieArgs), fb = first.size() * sizeof(uint64_t);
    int rc = ctx_alloc(ctx, (void**)&djobs, jb);
    if (!rc) rc = ctx_alloc(ctx, (void**)&dfirst, fb);
    // pageable sources: both copies complete before they return
    if (!rc) rc = host_to_device(ctx, djobs, jobs.data(), jb, stream);
    if (!rc) rc = host_to_device(ctx, dfirst, first.data(), fb, stream);
    if (!rc) {
        const uint64_t total = first.back();
        knn_tie_batch_kernel<<<(unsigned)((total + 127) / 128), 128, 0, stream>>>(djobs, dfirst,
                                                                               (int)jobs.size());
        NBG_LAUNCHED(1);
        if (cudaGetLastError() != cudaSuccess) rc = NBG_ERR_CUDA;
    }
    // the job table is read by the kernel: return it to the cache only after
    if (cudaStreamSynchronize(stream) != cudaSuccess && !rc) rc = NBG_ERR_CUDA;
    if (djobs) ctx_free(ctx, djobs, jb);
    if (dfirst) ctx_free(ctx, dfirst, fb);
    return rc;
}

// ---------------------------------------------------------------------------
// Strided neighbourhoods (eigenvalues / covariancefeatures stride > 1;
// KD3ImplT::neighbors, KDImpl.hpp:351-381): the reference takes its k*stride
// nearest in its own order and keeps every stride-th, so the order inside the
// list matters, not only the set.  Per row: the ring search finds the
// (k*stride)-th distance D; the points strictly closer and the group at D are
// collected; m members of the group are chosen, and the whole list ordered,
// by (FP64 distance as the reference forms it, then the order the reference's
// search meets them on the KD replica's tree); positions 0, stride, 2*stride,
// ... give the neighbourhood.  Rows the ring search cannot finish, or whose
// group exceeds the collection, go to the search replay.
// The list holds K <= KS - 1 entries (fewer than K points are strictly
// closer than D), so its arrays are sized by the launch's slot count.
template <int KS>
struct StrideFn {
    float qx, qy, qz;
    uint32_t kk;
    int less, gcnt;
    uint32_t id[KS];  // [0, less): closer than D; then the group's chosen members
    int off[KS][3];
    uint32_t gid[TIE_CAP];
    int goff[TIE_CAP][3];
    __device__ __forceinline__ unsigned long long limit() const {
        return (unsigned long long)(kk - KEY_BASE);
    }
    __device__ __forceinline__ void operator()(const float4 p) {
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const uint32_t key = dist_key(dx, dy, dz);
        if (key < kk) {
            if (less < KS) {
                id[less] = __float_as_uint(p.w);
                off[less][0] = small_int(dx);
                off[less][1] = small_int(dy);
                off[less][2] = small_int(dz);
            }
            ++less;
        } else if (key == kk) {
            if (gcnt < TIE_CAP) {
                gid[gcnt] = __float_as_uint(p.w);
                goff[gcnt][0] = small_int(dx);
                goff[gcnt][1] = small_int(dy);
                goff[gcnt][2] = small_int(dz);
            }
            ++gcnt;
        }
    }
};

struct StrideArgs {
    QueryArgs q;       // K = k * stride (list length), ties null
    int32_t stride;
    int32_t kpick;     // k: entries kept
    KdOrder kd;
    int32_t consumer;  // 1: the ordered list goes to a kNN consumer (L), not a covariance
    ListArgs L;
};

template <int KS>
__global__ void __launch_bounds__(128) knn_stride_kernel(const StrideArgs sa) {
    const QueryArgs& a = sa.q;
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t rid = __float_as_uint(q.w);
    const int K = a.K;
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    int R;
    uint32_t kk;
    bool tie;
    if (!select_kth<KS>(a, g, qc, q, K, R, kk, tie) && !tie) {
        const uint32_t slot = atomicAdd(&a.counters[0], 1u);
        a.exact_rows[slot] = rid;
        return;
    }
    StrideFn<KS> f;
    f.qx = q.x;
    f.qy = q.y;
    f.qz = q.z;
    f.kk = kk;
    f.less = 0;
    f.gcnt = 0;
    for (int r = 0; r <= R; ++r) scan_shell(a.gv, g, qc, r, f);
    const int m = K - f.less;
    if (f.gcnt > TIE_CAP || f.less >= KS || m <= 0 || m > f.gcnt) {
        const uint32_t slot = atomicAdd(&a.counters[0], 1u);
        a.exact_rows[slot] = rid;
        return;
    }
    const int32_t qraw[3] = {qc.qx + g.minx, qc.qy + g.miny, qc.qz + g.minz};
    const double q64[3] = {ref_coord(qraw[0], a.tf.scale[0], a.tf.offset[0]),
                           ref_coord(qraw[1], a.tf.scale[1], a.tf.offset[1]),
                           ref_coord(qraw[2], a.tf.scale[2], a.tf.offset[2])};
    // the group's m members the reference admits (as the tie-order resolver)
    double gd[TIE_CAP];
    for (int t = 0; t < f.gcnt; ++t) gd[t] = ref_dist2(q64, qraw, f.goff[t], a.tf);
    uint32_t taken = 0;
    for (int j = 0; j < m; ++j) {
        int best = -1;
        for (int t = 0; t < f.gcnt; ++t) {
            if ((taken >> t) & 1u) continue;
            if (best < 0 || gd[t] < gd[best] ||
                (gd[t] == gd[best] &&
                 kd_meets_first(sa.kd, q64, __ldg(&sa.kd.kpos[sa.kd.base + f.gid[t]]),
                                __ldg(&sa.kd.kpos[sa.kd.base + f.gid[best]]))))
                best = t;
        }
        taken |= 1u << best;
        f.id[f.less + j] = f.gid[best];
        f.off[f.less + j][0] = f.goff[best][0];
        f.off[f.less + j][1] = f.goff[best][1];
        f.off[f.less + j][2] = f.goff[best][2];
    }
    // the list in the reference's order: FP64 distance, then visiting order
    double d[KS];
    for (int t = 0; t < K; ++t) d[t] = ref_dist2(q64, qraw, f.off[t], a.tf);
    for (int t = 1; t < K; ++t) {
        const double dv = d[t];
        const uint32_t iv = f.id[t];
        const int o0 = f.off[t][0], o1 = f.off[t][1], o2 = f.off[t][2];
        int u = t - 1;
        while (u >= 0 &&
               (d[u] > dv || (d[u] == dv && kd_meets_first(sa.kd, q64, __ldg(&sa.kd.kpos[sa.kd.base + iv]),
                                                           __ldg(&sa.kd.kpos[sa.kd.base + f.id[u]]))))) {
            d[u + 1] = d[u];
            f.id[u + 1] = f.id[u];
            f.off[u + 1][0] = f.off[u][0];
            f.off[u + 1][1] = f.off[u][1];
            f.off[u + 1][2] = f.off[u][2];
            --u;
        }
        d[u + 1] = dv;
        f.id[u + 1] = iv;
        f.off[u + 1][0] = o0;
        f.off[u + 1][1] = o1;
        f.off[u + 1][2] = o2;
    }
    if (sa.consumer) {
        list_consume(sa.L, a.tf, a.ex, rid, qraw, K, f.id, f.off, d);
        return;
    }
    long long s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 0; j < sa.kpick; ++j) {
        const int t = j * sa.stride;  // < K by construction (K = kpick * stride)
        const long long d0 = f.off[t][0], d1 = f.off[t][1], d2 = f.off[t][2];
        s1[0] += d0;
        s1[1] += d1;
        s1[2] += d2;
        s2[0] += d0 * d0;
        s2[1] += d1 * d0;
        s2[2] += d1 * d1;
        s2[3] += d2 * d0;
        s2[4] += d2 * d1;
        s2[5] += d2 * d2;
    }
    const long long n = sa.kpick;
    long long M[6];
    M[0] = n * s2[0] - s1[0] * s1[0];
    M[1] = n * s2[1] - s1[1] * s1[0];
    M[2] = n * s2[2] - s1[1] * s1[1];
    M[3] = n * s2[3] - s1[2] * s1[0];
    M[4] = n * s2[4] - s1[2] * s1[1];
    M[5] = n * s2[5] - s1[2] * s1[2];
    nbg_finish_row(a.grp, a.tf, a.ex, rid, (int)n, M, qraw);
}

// ---------------------------------------------------------------------------
// Radius neighbourhoods (NormalFilter.cpp:149-150, EigenvaluesFilter.cpp:
// 121-134, CovarianceFeaturesFilter.cpp:216-225 through KD3Index::radius,
// KDImpl.hpp:398-415): the points whose squared FP64 distance, formed as the
// reference forms it, is below fl(r*r).  nanoflann's RadiusResultSet keeps
// every such point, so there is no tie order.  A candidate whose exact integer
// distance is clearly beyond the radius (relative 1e-5, far above the FP64
// rounding of the coordinates) is dropped; every other candidate is tested
// with the reference's FP64 distance.  Sums are int64 (exact while the
// neighbourhood's sum of squared offsets stays below 2^63 raw units^2).
struct RadiusFn {
    float qx, qy, qz;
    int32_t qraw[3];
    double q64[3];
    double rr;
    unsigned long long dout;
    Transform tf;
    long long s1x, s1y, s1z, sxx, syx, syy, szx, szy, szz;
    uint32_t cnt;
    __device__ __forceinline__ unsigned long long limit() const { return dout; }
    __device__ __forceinline__ void operator()(const float4 p) {
        const int ix = (int)(p.x - qx), iy = (int)(p.y - qy), iz = (int)(p.z - qz);
        const unsigned long long D = (unsigned long long)((long long)ix * ix + (long long)iy * iy +
                                                          (long long)iz * iz);
        if (D > dout) return;
        const int off[3] = {ix, iy, iz};
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double pc = ref_coord(qraw[d] + off[d], tf.scale[d], tf.offset[d]);
            const double df = __dsub_rn(q64[d], pc);
            acc = __dadd_rn(acc, __dmul_rn(df, df));
        }
        if (!(acc < rr)) return;
        s1x += ix;
        s1y += iy;
        s1z += iz;
        sxx += (long long)ix * ix;
        syx += (long long)iy * ix;
        syy += (long long)iy * iy;
        szx += (long long)iz * ix;
        szy += (long long)iz * iy;
        szz += (long long)iz * iz;
        ++cnt;
    }
};

struct RadiusArgs {
    GridView gv;
    const GridParams* gp;
    uint64_t n;
    StageGroup grp;
    Transform tf;
    ExceptionSink ex;
    double rr;                 // fl(r * r)
    unsigned long long dout;   // integer squared distances above it are outside
    double r_raw;              // radius in raw units (for the ring count)
    int32_t min_k;
};

__device__ __forceinline__ double m_entry(long long n, long long sab, long long sa, long long sb) {
    return (double)((__int128)n * sab - (__int128)sa * sb);
}

__global__ void __launch_bounds__(128) knn_radius_kernel(const RadiusArgs a) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const GridParams g = *a.gp;
    const float4 q = __ldg(&a.gv.sorted[i]);
    const uint32_t id = __float_as_uint(q.w);
    QueryCell qc;
    qc.qx = __float2int_rz(q.x);
    qc.qy = __float2int_rz(q.y);
    qc.qz = __float2int_rz(q.z);
    qc.cx = qc.qx / g.cell;
    qc.cy = qc.qy / g.cell;
    qc.cz = qc.qz / g.cell;
    RadiusFn f;
    f.qx = q.x;
    f.qy = q.y;
    f.qz = q.z;
    f.qraw[0] = qc.qx + g.minx;
    f.qraw[1] = qc.qy + g.miny;
    f.qraw[2] = qc.qz + g.minz;
    for (int d = 0; d < 3; ++d) f.q64[d] = ref_coord(f.qraw[d], a.tf.scale[d], a.tf.offset[d]);
    f.rr = a.rr;
    f.dout = a.dout;
    f.tf = a.tf;
    f.s1x = f.s1y = f.s1z = f.sxx = f.syx = f.syy = f.szx = f.szy = f.szz = 0;
    f.cnt = 0;
    const int R = (int)ceil(a.r_raw / (double)g.cell);
    for (int r = 0; r <= R; ++r) scan_shell(a.gv, g, qc, r, f);
    const StageDev& st = a.grp.st[0];
    if (st.kind != NBG_STAGE_NORMAL && (long long)f.cnt < (long long)a.min_k) {
        nbg_append_exception(a.ex, id, a.grp.stage_index[0], NBG_ROW_RADIUS_FEW,
                             (uint16_t)min(f.cnt, 65535u));
        return;
    }
    const long long n = f.cnt;
    const double Md[6] = {m_entry(n, f.sxx, f.s1x, f.s1x), m_entry(n, f.syx, f.s1y, f.s1x),
                          m_entry(n, f.syy, f.s1y, f.s1y), m_entry(n, f.szx, f.s1z, f.s1x),
                          m_entry(n, f.szy, f.s1z, f.s1y), m_entry(n, f.szz, f.s1z, f.s1z)};
    nbg_finish_row_d(a.grp, a.tf, a.ex, id, (int)min(f.cnt, 0x7FFFFFFFu), Md, f.qraw);
}

int launch_radius(Context* ctx, const RadiusLaunch& rl, cudaStream_t stream) {
    (void)ctx;
    const Tile* t = rl.tile;
    if (!t->n) return NBG_OK;
    RadiusArgs a;
    a.gv = grid_view(t);
    a.gp = t->gp;
    a.n = t->n;
    a.grp = rl.grp;
    a.tf = t->tf;
    a.ex = rl.ex;
    a.rr = rl.radius * rl.radius;
    const double s = t->tf.scale[0];
    const double rr_raw = a.rr / (s * s);
    a.dout = rr_raw > 0.0 ? (unsigned long long)ceil(rr_raw * (1.0 + 1e-5)) + 2ull : 0ull;
    a.r_raw = sqrt((double)a.dout);
    a.min_k = rl.min_k;
    knn_radius_kernel<<<(unsigned)((t->n + 127) / 128), 128, 0, stream>>>(a);
    NBG_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

static int slots_for(int K) {
    const int need = K + 1;
    if (need <= 10) return 10;
    if (need <= 12) return 12;
    if (need <= 14) return 14;
    if (need <= 18) return 18;
    if (need <= 26) return 26;
    if (need <= 34) return 34;
    if (need <= 50) return 50;
    if (need <= 66) return 66;
    return -1;
}

template <template <int> class Launcher>
static int dispatch_slots(int K, typename Launcher<10>::Args args) {
    switch (slots_for(K)) {
        case 10: return Launcher<10>::run(args);
        case 12: return Launcher<12>::run(args);
        case 14: return Launcher<14>::run(args);
        case 18: return Launcher<18>::run(args);
        case 26: return Launcher<26>::run(args);
        case 34: return Launcher<34>::run(args);
        case 50: return Launcher<50>::run(args);
        case 66: return Launcher<66>::run(args);
    }
    return NBG_ERR_INVALID;
}

// Offset bits of the single-pass select's keys for cell edge c: the squared
// distance field (27 - ob bits) holds (2.2 c)^2, the search's reach at ring 2.
static uint32_t loc_offset_bits(int32_t c) {
    const double need = 4.84 * (double)std::max(c, 1) * (double)std::max(c, 1);
    int bits = 1;
    while (bits < 27 && (double)(1u << bits) < need) ++bits;
    return (uint32_t)std::min(16, std::max(6, 27 - bits));
}

struct LaunchArgs {
    QueryArgs q;
    cudaStream_t stream;
    cudaStream_t fork = nullptr;   // second stream for the handed-back rows (null: `stream`)
    cudaEvent_t fev[3] = {};       // fork, handed-back rows done, finish done
    cudaEvent_t done = nullptr;    // QueryLaunch::done
    bool ids;
    int group = 0;        // select kernel (nbg_tile_set_select; 0: two-pass per-thread)
    float margin0 = 0.25f;
    int sms = 148;
    uint32_t ob = 11;     // single-pass select: offset bits of a key
};

int launch_group_select(const QueryArgs& q, int slots, int group, float margin0,
                        cudaStream_t stream);

// Handed-back rows are the sparse-region and hard rows: long ring searches
// that need many resident warps to hide their latency.  The row count is read
// on the device, so the grid is sized for the largest expected share (a few
// per cent of the tile) at one row per thread; blocks past it exit at once.
static constexpr uint64_t kRetryBlocksPerSm = 16;

template <int KS>
struct KnnLauncher {
    using Args = LaunchArgs;
    static int run(const LaunchArgs& la) {
        const int threads = 128;
        const uint64_t rows = la.q.rows ? la.q.nq : la.q.n;
        const uint64_t blocks = (rows + threads - 1) / threads;
        if (blocks == 0) return NBG_OK;
        if (la.group == 2 && la.q.sums && !la.ids) {
            // single pass with located keys; rows it hands back through the
            // two-pass kernel (count read on the device); then the finish pass
            if (cudaMemsetAsync(la.q.counters + 6, 0, sizeof(uint32_t), la.stream))
                return NBG_ERR_CUDA;
            knn_select_loc_kernel<KS><<<(unsigned)blocks, threads, 0, la.stream>>>(la.q, la.ob);
            QueryArgs r = la.q;
            r.rows = la.q.retry_rows;
            r.nq_dev = la.q.counters + 6;
            const unsigned rb = (unsigned)std::min<uint64_t>(blocks, (uint64_t)la.sms * kRetryBlocksPerSm);
            if (!la.fork) {
                knn_retry_kernel<KS><<<rb, threads, 0, la.stream>>>(r);
                knn_finish_kernel<<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
                NBG_LAUNCHED(3);
                return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
            }
            // the handed-back rows on the fork stream, queued first so their
            // long searches start first; the finish pass of the other rows on
            // `stream` fills the SMs around them
            cudaError_t e = cudaEventRecord(la.fev[0], la.stream);
            if (!e) e = cudaStreamWaitEvent(la.fork, la.fev[0], 0);
            if (e) return NBG_ERR_CUDA;
            knn_retry_finish_kernel<KS><<<rb, threads, 0, la.fork>>>(r);
            knn_finish_kernel<<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            NBG_LAUNCHED(3);
            if (la.done) {
                // join on the fork stream: `stream` may go on to the next launch
                e = cudaEventRecord(la.fev[2], la.stream);
                if (!e) e = cudaStreamWaitEvent(la.fork, la.fev[2], 0);
                if (!e) e = cudaEventRecord(la.done, la.fork);
            } else {
                e = cudaEventRecord(la.fev[1], la.fork);
                if (!e) e = cudaStreamWaitEvent(la.stream, la.fev[1], 0);
            }
            if (e) return NBG_ERR_CUDA;
            return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
        }
        if (la.group == 1 && la.q.sums && !la.ids) {
            const uint64_t b256 = (rows + 255) / 256;
            knn_select_morton_kernel<KS><<<(unsigned)b256, 256, 0, la.stream>>>(la.q);
            knn_finish_kernel<<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            NBG_LAUNCHED(2);
            return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
        }
        if (la.group >= 8 && (la.ids || la.q.sums)) {
            // group select, then the rows it handed back through the per-thread
            // select (count read on the device), then the finish pass
            if (cudaMemsetAsync(la.q.counters + 6, 0, sizeof(uint32_t), la.stream))
                return NBG_ERR_CUDA;
            int rc = launch_group_select(la.q, KS, la.group, la.margin0, la.stream);
            if (rc) return rc;
            QueryArgs r = la.q;
            r.rows = la.q.retry_rows;
            r.nq_dev = la.q.counters + 6;
            knn_retry_kernel<KS><<<(unsigned)std::min<uint64_t>(blocks, (uint64_t)la.sms * kRetryBlocksPerSm), threads,
                                   0, la.stream>>>(r);
            NBG_LAUNCHED(1);
            if (!la.ids) {
                knn_finish_kernel<<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
                NBG_LAUNCHED(1);
            }
            return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
        }
        if (la.ids) {
            knn_ids_kernel<KS><<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            NBG_LAUNCHED(1);
        } else if (la.q.sums) {
            knn_select_kernel<KS><<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            knn_finish_kernel<<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            NBG_LAUNCHED(2);
        } else {
            knn_fused_kernel<KS><<<(unsigned)blocks, threads, 0, la.stream>>>(la.q);
            NBG_LAUNCHED(1);
        }
        return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
    }
};

GridView grid_view(const Tile* t) {
    GridView v;
    v.sorted = t->sorted;
    v.colinfo = t->colinfo;
    v.cstart = t->cstart;
    return v;
}

int launch_query(Context* ctx, const QueryLaunch& ql, cudaStream_t stream) {
    (void)ctx;
    LaunchArgs la;
    la.q.gv = grid_view(ql.tile);
    la.q.gp = ql.tile->gp;
    la.q.n = ql.tile->n;
    la.q.K = ql.K;
    la.q.rmax = ql.rmax;
    la.q.grp = ql.grp;
    la.q.tf = ql.tile->tf;
    la.q.ex = ql.ex;
    la.q.exact_rows = ql.exact_rows;
    la.q.counters = ql.counters;
    la.q.ids_out = nullptr;
    la.q.ties = ql.ties;
    la.q.tie_cap = ql.tie_cap;
    la.q.sums = ql.sums;
    la.q.row_k = ql.row_k;
    la.q.rows = ql.sums ? ql.rows : nullptr;  // the fused kernel answers every row
    la.q.nq = ql.sums ? ql.nrows : 0;
    la.q.retry_rows = ql.retry_rows;
    la.stream = stream;
    if (ctx && ctx->fork) {
        la.fork = ctx->fork;
        for (int i = 0; i < 3; ++i) la.fev[i] = ctx->fev[i];
    }
    la.done = ql.done;
    la.ids = false;
    la.group = ql.retry_rows ? ql.group : 0;
    la.margin0 = ql.margin0;
    la.sms = ctx ? ctx->sm_count : 148;
    la.ob = loc_offset_bits(ql.tile->host_gp.cell);
    const int rc = dispatch_slots<KnnLauncher>(ql.K, la);
    // the forked single-pass launch records `done` itself, on the fork stream
    if (!rc && ql.done && !query_forks(ctx, ql) && cudaEventRecord(ql.done, stream) != cudaSuccess)
        return NBG_ERR_CUDA;
    return rc;
}

bool query_forks(const Context* ctx, const QueryLaunch& ql) {
    const uint64_t rows = ql.rows ? ql.nrows : ql.tile->n;
    return ctx && ctx->fork && ql.retry_rows && ql.group == 2 && ql.sums && rows > 0;
}

int launch_neighbor_sets(Context* ctx, const Tile* t, int K, int rmax, uint32_t* ids_out,
                         uint32_t* exact_rows, uint32_t* counters, uint2* ties, uint32_t tie_cap,
                         cudaStream_t stream, uint32_t* retry_rows) {
    LaunchArgs la{};
    la.group = retry_rows ? t->group : 0;
    la.margin0 = t->margin0;
    la.sms = ctx ? ctx->sm_count : 148;
    la.q.retry_rows = retry_rows;
    la.q.gv = grid_view(t);
    la.q.gp = t->gp;
    la.q.n = t->n;
    la.q.K = K;
    la.q.rmax = rmax;
    la.q.tf = t->tf;
    la.q.exact_rows = exact_rows;
    la.q.counters = counters;
    la.q.ids_out = ids_out;
    la.q.ties = ties;
    la.q.tie_cap = tie_cap;
    la.q.sums = nullptr;
    la.q.row_k = nullptr;
    la.stream = stream;
    la.ids = true;
    return dispatch_slots<KnnLauncher>(K, la);
}

int slots_for_k(int K) { return slots_for(K); }

// Sorted positions whose point id lies in [lo, hi).
struct InIdRange {
    const float4* sorted;
    uint32_t lo, hi;
    __device__ __forceinline__ bool operator()(const uint32_t i) const {
        const uint32_t id = __float_as_uint(__ldg(&sorted[i]).w);
        return id >= lo && id < hi;
    }
};

int build_id_chunks(Context* ctx, const Tile* t, const uint64_t* bounds, int nchunks,
                    uint32_t* rows, uint32_t* dnum, cudaStream_t st) {
    const uint64_t n = t->n;
    cub::CountingInputIterator<uint32_t> first(0);
    size_t tmp_bytes = 0;
    cudaError_t e = cub::DeviceSelect::If(nullptr, tmp_bytes, first, rows, dnum, (int64_t)n,
                                          InIdRange{t->sorted, 0, 0}, st);
    if (e) return fail(ctx, NBG_ERR_CUDA, std::string("row chunks: ") + cudaGetErrorString(e));
    void* tmp = nullptr;
    int rc = ctx_alloc(ctx, &tmp, std::max<size_t>(tmp_bytes, 16));
    if (rc) return rc;
    for (int c = 0; c < nchunks && !e; ++c) {
        e = cub::DeviceSelect::If(tmp, tmp_bytes, first, rows + bounds[c], dnum, (int64_t)n,
                                  InIdRange{t->sorted, (uint32_t)bounds[c], (uint32_t)bounds[c + 1]},
                                  st);
        NBG_LAUNCHED(1);
    }
    // the temporary storage goes back to the cache only after the selects ran
    if (!e) e = cudaStreamSynchronize(st);
    ctx_free(ctx, tmp, std::max<size_t>(tmp_bytes, 16));
    return e ? fail(ctx, NBG_ERR_CUDA, std::string("row chunks: ") + cudaGetErrorString(e)) : NBG_OK;
}

struct SampleArgs {
    QueryArgs q;
    uint64_t stride;
    unsigned blocks;
    unsigned run;
    cudaStream_t stream;
};

template <int KS>
struct SampleLauncher {
    using Args = SampleArgs;
    static int run(const SampleArgs& s) {
        if (!s.blocks) return NBG_OK;
        knn_select_sample_kernel<KS><<<s.blocks, 128, 0, s.stream>>>(s.q, s.stride, s.run);
        NBG_LAUNCHED(1);
        return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
    }
};

int launch_select_sample(Context* ctx, const QueryLaunch& ql, uint64_t stride, unsigned blocks,
                         unsigned run, cudaStream_t stream) {
    (void)ctx;
    SampleArgs s{};
    s.q.gv = grid_view(ql.tile);
    s.q.gp = ql.tile->gp;
    s.q.n = ql.tile->n;
    s.q.K = ql.K;
    s.q.rmax = ql.rmax;
    s.q.grp = ql.grp;
    s.q.tf = ql.tile->tf;
    s.q.ex = ql.ex;
    s.q.exact_rows = ql.exact_rows;
    s.q.counters = ql.counters;
    s.q.ties = ql.ties;
    s.q.tie_cap = ql.tie_cap;
    s.q.sums = ql.sums;
    s.q.row_k = ql.row_k;
    s.stride = stride;
    s.blocks = blocks;
    s.run = std::max(1u, run);
    s.stream = stream;
    return dispatch_slots<SampleLauncher>(ql.K, s);
}

int launch_select_queue(Context* ctx, int K, const BatchJob* jobs, int njobs, uint64_t items,
                        unsigned long long* head, cudaStream_t stream, int reserve) {
    return dispatch_slots<QueueLauncher>(
        K, QueueArgs{jobs, njobs, items, head, ctx->sm_count, stream, reserve});
}

int launch_finish_queue(Context* ctx, const BatchJob* jobs, int njobs, uint64_t items,
                        unsigned long long* head, cudaStream_t stream, int reserve) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, knn_finish_queue_kernel, 128, 0);
    const uint64_t grid =
        std::min<uint64_t>(items, (uint64_t)ctx->sm_count * std::max(per_sm - reserve, 1));
    if (!grid) return NBG_OK;
    knn_finish_queue_kernel<<<(unsigned)grid, 128, 0, stream>>>(jobs, njobs, items, head);
    NBG_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

struct StrideLaunchArgs {
    StrideArgs s;
    unsigned blocks;
    cudaStream_t stream;
};

template <int KS>
struct StrideLauncher {
    using Args = StrideLaunchArgs;
    static int run(const StrideLaunchArgs& l) {
        if (!l.blocks) return NBG_OK;
        knn_stride_kernel<KS><<<l.blocks, 128, 0, l.stream>>>(l.s);
        NBG_LAUNCHED(1);
        return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
    }
};

int launch_stride(Context* ctx, const QueryLaunch& ql, int stride, int kpick, const KdOrder& kd,
                  cudaStream_t stream, const ListArgs* list) {
    (void)ctx;
    StrideLaunchArgs l{};
    if (list) {
        l.s.consumer = 1;
        l.s.L = *list;
    }
    QueryArgs& q = l.s.q;
    q.gv = grid_view(ql.tile);
    q.gp = ql.tile->gp;
    q.n = ql.tile->n;
    q.K = ql.K;
    q.rmax = ql.rmax;
    q.grp = ql.grp;
    q.tf = ql.tile->tf;
    q.ex = ql.ex;
    q.exact_rows = ql.exact_rows;
    q.counters = ql.counters;
    q.ids_out = nullptr;
    q.ties = nullptr;
    q.tie_cap = 0;
    q.sums = nullptr;
    q.row_k = nullptr;
    l.s.stride = stride;
    l.s.kpick = kpick;
    l.s.kd = kd;
    l.blocks = (unsigned)((ql.tile->n + 127) / 128);
    l.stream = stream;
    return dispatch_slots<StrideLauncher>(ql.K, l);
}

}  // namespace nbg

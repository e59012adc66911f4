// nbg_query.cuh — device helpers shared by the kNN query kernels (grid ring
// search, exact integer distance keys, register top list, row hand-off).
#pragma once

#include <climits>

#include "nbg_common.cuh"

namespace nbg {

static constexpr uint32_t KEY_BASE = 0x4B000000u;    // bits of 2^23f
static constexpr uint32_t KEY_EXACT_END = 0x4B800000u;  // bits of 2^24f

__device__ __forceinline__ uint32_t dist_key(float dx, float dy, float dz) {
    return __float_as_uint(fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 8388608.0f))));
}

// integer value of an exact small float (|v| < 2^22)
__device__ __forceinline__ int small_int(float v) {
    return __float_as_int(v + 12582912.0f) - 0x4B400000;
}

struct QueryCell {
    int qx, qy, qz;     // raw, relative to tile min
    int cx, cy, cz;     // cell coords
};

// Calls f(float4) for the points of cells zl..zh of a column (inclusive).
template <class F>
__device__ __forceinline__ void scan_cells(const GridView& gv, const int4 ci, int zl, int zh, F& f) {
    zl = max(zl, ci.y);
    zh = min(zh, ci.z);
    if (zl > zh) return;
    const uint32_t e0 = (uint32_t)ci.x + (uint32_t)(zl - ci.y);
    const uint32_t e1 = (uint32_t)ci.x + (uint32_t)(zh - ci.y) + 1;
    const uint32_t pe = __ldg(&gv.cstart[e1]);
    for (uint32_t j = __ldg(&gv.cstart[e0]); j < pe; ++j) f(__ldg(&gv.sorted[j]));
}

// Distance (raw units) from coordinate q to the cell slab [k*c, (k+1)*c - 1].
__device__ __forceinline__ int slab_gap(int q, int k, int c) {
    const int lo = k * c, hi = lo + c - 1;
    return q < lo ? lo - q : (q > hi ? q - hi : 0);
}

// Calls f(float4) for every point of the cells at Chebyshev distance R that
// can hold a point within the functor's current squared-distance limit
// f.limit(): boundary columns contribute their cells with z in [cz-R, cz+R],
// interior columns only the two cells at z = cz-R and z = cz+R; a column whose
// horizontal gap already exceeds the limit, and cells beyond the ball's
// z-reach, are skipped (they cannot hold a point at or below the limit).
template <class F>
__device__ __forceinline__ void scan_shell(const GridView& gv, const GridParams& g,
                                           const QueryCell& qc, int R, F& f) {
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
            const unsigned long long lim = f.limit();
            if ((unsigned long long)h2 > lim) continue;
            const int4 ci = __ldg(&gv.colinfo[(uint32_t)y * (uint32_t)g.gx + (uint32_t)x]);
            if (ci.z < ci.y) continue;
            // z-cells within reach of the ball of squared radius lim
            int zr0 = zlo, zr1 = zhi;
            if (lim < (1ull << 46)) {
                const float s = sqrtf((float)(lim - (unsigned long long)h2)) + 1.0f;
                zr0 = max(zr0, (int)floorf(((float)qc.qz - s) / (float)c));
                zr1 = min(zr1, (int)floorf(((float)qc.qz + s) / (float)c));
            }
            const int adx = dx < 0 ? -dx : dx;
            if (max(ady, adx) == R) {
                scan_cells(gv, ci, zr0, zr1, f);
            } else {
                if (zlo >= zr0 && zlo <= zr1) scan_cells(gv, ci, zlo, zlo, f);
                if (zhi >= zr0 && zhi <= zr1) scan_cells(gv, ci, zhi, zhi, f);
            }
        }
    }
}

// Squared raw gap from the query to any point outside the scanned cube of
// radius R; UINT64_MAX when the cube covers the whole grid.
__device__ __forceinline__ unsigned long long outside_gap2(const GridParams& g,
                                                           const QueryCell& qc, int R) {
    long long gap = LLONG_MAX;
    const int c = g.cell;
    if (qc.cx - R > 0) gap = min(gap, (long long)qc.qx - (long long)(qc.cx - R) * c + 1);
    if (qc.cx + R < g.gx - 1) gap = min(gap, (long long)(qc.cx + R + 1) * c - qc.qx);
    if (qc.cy - R > 0) gap = min(gap, (long long)qc.qy - (long long)(qc.cy - R) * c + 1);
    if (qc.cy + R < g.gy - 1) gap = min(gap, (long long)(qc.cy + R + 1) * c - qc.qy);
    if (qc.cz - R > 0) gap = min(gap, (long long)qc.qz - (long long)(qc.cz - R) * c + 1);
    if (qc.cz + R < g.gz - 1) gap = min(gap, (long long)(qc.cz + R + 1) * c - qc.qz);
    if (gap == LLONG_MAX) return ~0ull;
    return (unsigned long long)gap * (unsigned long long)gap;
}

template <int KS>
struct TopK {
    uint32_t k[KS];
    __device__ __forceinline__ void init(int off) {
#pragma unroll
        for (int s = 0; s < KS; ++s) k[s] = s < off ? 0u : 0xFFFFFFFFu;
    }
    __device__ __forceinline__ void insert(uint32_t key) {
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const uint32_t lo = min(k[s], key);
            key = max(k[s], key);
            k[s] = lo;
        }
    }
    __device__ __forceinline__ uint32_t at(int i) const {
        uint32_t v = 0xFFFFFFFFu;
#pragma unroll
        for (int s = 0; s < KS; ++s)
            if (s == i) v = k[s];
        return v;
    }
};

// A row that cannot finish on the grid: a boundary tie goes to the tie list
// (its K-th distance and final ring kept for the order resolver), everything
// else, and ties beyond the list's capacity, to the full search replay.
__device__ __forceinline__ void defer_row(const QueryArgs& a, uint32_t id, bool tie, uint32_t kk,
                                          int R) {
    if (tie && a.ties) {
        const uint32_t slot = atomicAdd(&a.counters[4], 1u);
        if (slot < a.tie_cap) {
            a.ties[slot] = make_uint2(id, (kk - KEY_BASE) | ((uint32_t)R << 24));
            return;
        }
    }
    const uint32_t slot = atomicAdd(&a.counters[0], 1u);
    a.exact_rows[slot] = id;
}

// 10-bit Morton interleave of three coordinates.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Sort keys of a block's rows r0 .. r0 + nvalid - 1 (threads past nvalid get
// a key above every row's): a Morton key of the row's coordinates relative to
// the block's bounding box, at the resolution that fits the box in 10 bits
// per axis; val = the row's sorted position.  s_box: 6 ints of shared memory.
template <int THREADS>
__device__ __forceinline__ void block_morton_order(const QueryArgs& a, uint64_t r0, uint32_t nvalid,
                                                   int* s_box, uint32_t (&key)[1],
                                                   uint32_t (&val)[1]) {
    const int tid = threadIdx.x;
    const bool v = tid < (int)nvalid;
    uint32_t pos = 0;
    int q0 = 0, q1 = 0, q2 = 0;
    if (v) {
        pos = a.rows ? __ldg(&a.rows[r0 + tid]) : (uint32_t)(r0 + tid);
        const float4 q = __ldg(&a.gv.sorted[pos]);
        q0 = __float2int_rz(q.x);
        q1 = __float2int_rz(q.y);
        q2 = __float2int_rz(q.z);
    }
    if (tid < 6) s_box[tid] = tid < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
    const int lo0 = __reduce_min_sync(0xffffffffu, v ? q0 : INT_MAX);
    const int lo1 = __reduce_min_sync(0xffffffffu, v ? q1 : INT_MAX);
    const int lo2 = __reduce_min_sync(0xffffffffu, v ? q2 : INT_MAX);
    const int hi0 = __reduce_max_sync(0xffffffffu, v ? q0 : INT_MIN);
    const int hi1 = __reduce_max_sync(0xffffffffu, v ? q1 : INT_MIN);
    const int hi2 = __reduce_max_sync(0xffffffffu, v ? q2 : INT_MIN);
    if ((tid & 31) == 0) {
        atomicMin(&s_box[0], lo0);
        atomicMin(&s_box[1], lo1);
        atomicMin(&s_box[2], lo2);
        atomicMax(&s_box[3], hi0);
        atomicMax(&s_box[4], hi1);
        atomicMax(&s_box[5], hi2);
    }
    __syncthreads();
    const int ext = max(s_box[3] - s_box[0], max(s_box[4] - s_box[1], s_box[5] - s_box[2]));
    const int sh = max(0, 32 - __clz(max(ext, 1)) - 10);  // (ext >> sh) < 1024
    key[0] = 0x7FFFFFFFu;
    val[0] = pos;
    if (v)
        key[0] = spread3((uint32_t)(q0 - s_box[0]) >> sh) |
                 (spread3((uint32_t)(q1 - s_box[1]) >> sh) << 1) |
                 (spread3((uint32_t)(q2 - s_box[2]) >> sh) << 2);
}

}  // namespace nbg

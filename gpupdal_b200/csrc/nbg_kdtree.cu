// nbg_kdtree.cu — exact replica of the reference's KD3 tree, and its search,
// for the rows whose neighbour set depends on nanoflann's tie order.
//
// The reference keeps, among points at equal FP64 distance, the ones its
// depth-first search meets first (vendor/nanoflann/nanoflann.hpp:178-205
// shifts only on strict >, :1191-1197 admits only dist < worst).  That order
// is a function of the tree, so rows whose k-th distance ties (and rows the
// ring search could not finish) are answered by replaying the reference's
// search over an identical tree built on the device.
//
// Tree build (nanoflann.hpp:640-690 divideTree, :779-828 middleSplit_,
// :837-873 planeSplit), level-synchronous over all segments of a level:
//   minmax    per-segment min/max of the raw coordinates (monotone in the
//             double coordinate raw*scale+offset)
//   split     cut feature among dims whose top-down span > (1-1e-5)*max span,
//             largest actual spread first; cut value = top-down midpoint
//             clamped to the segment's extent
//   pass 1/2  the two Hoare passes.  Their effect is exactly: with L the
//             count of elements satisfying the predicate, the t-th element
//             from the left failing it inside [0, L) swaps with the t-th
//             element from the right satisfying it inside [L, n).  Ranks
//             come from per-tile counts and block scans.
//   children  split index lim1 / lim2 / count/2 rule; segments of at most
//             100 points become leaves
// divlow/divhigh (child extents) are filled bottom-up afterwards.
//
// Search (nanoflann.hpp:875-893, 1059-1079, 1184-1250) is replayed per row
// in FP64 with every operation rounded as the reference rounds it.
#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "nbg_common.cuh"
#include "nbg_internal.h"

namespace nbg {

static constexpr int KD_LEAF = 100;
// Level passes: tiles of KD_TILE elements, KD_THREADS threads of KD_ITEMS
// elements each (segments on the level passes hold more than 4096 points).
static constexpr int KD_TILE = 1024;
static constexpr int KD_THREADS = 256;
static constexpr int KD_ITEMS = KD_TILE / KD_THREADS;
// Segments of at most this many points are finished, subtree and all, by
// one warp (kd_warp_build_kernel) instead of level by level.
static constexpr uint32_t KD_WARP_MAX = 4096;
static constexpr int KD_WSTACK = 64;
static constexpr int KD_WARPS = 4;
// A build beside a running query (the plain call's speculative replica) keeps
// its level passes to 2 blocks of 256 threads per SM and the warp subtree
// builder to 2 blocks of 128, walking tiles and subtrees in strides, so the
// query keeps most of every SM while the build still streams its passes.
// Uncapped, its one-block-per-tile launches take every slot a query block
// frees.  Below 16M points the capped build outlasts the query, which then
// waits for it; the cap applies from there up.
static constexpr int kKdBesideBlocksPerSm = 2;
static constexpr int kKdBesideWarpBlocksPerSm = 2;
static constexpr uint64_t kKdBesideMinPoints = 16000000;
static constexpr int KD_RETRY = -100;  // kd_build: redo without warp subtrees
static constexpr int KD_STACK = 96;
static constexpr int KD_CAP = 66;

struct KdSeg {
    uint32_t begin, end;
    int32_t node;
    int32_t pad;
    double lo[3], hi[3];
};

struct KdSplit {
    int32_t f;
    uint32_t eq;  // points equal to the cut value (pass 2 has work only when > 0)
    double cutval;
    uint32_t L, m;    // pass 1: count below, misplaced pairs
    uint32_t L2, m2;  // pass 2 on [L, n)
    int32_t mn[3], mx[3];
};

struct KdDev {
    const int32_t* rx;
    const int32_t* ry;
    const int32_t* rz;
    const uint32_t* rid;
    const int32_t* c1;
    const int32_t* c2;
    const int32_t* feat;
    const uint32_t* nb;
    const uint32_t* ne;
    const double* dlo;
    const double* dhi;
    int32_t root;  // the tree's root node
    double root_lo[3], root_hi[3];
};

// Storage of one or more replicas built together (a forest): the trees'
// points are concatenated (tree k owns positions [base[k], base[k] + npts[k])),
// their nodes share the node arrays, and tree k's root is node k.  Segments
// carry their tree in KdSeg::pad, nodes in ntree[].
struct KdForest {
    uint64_t n = 0;
    uint32_t grid_cap = 0;   // blocks of a level-pass launch (0: one per tile)
    uint32_t wgrid_cap = 0;  // blocks of the warp subtree builder (0: one warp per subtree)
    int ntrees = 0;
    std::vector<uint64_t> base, npts;
    std::vector<Transform> tfh;
    std::vector<double> rootbox;  // 6 per tree: lo[3], hi[3]
    Transform* tfs = nullptr;     // device, per tree
    int32_t* ntree = nullptr;     // device, per node
    int refs = 0;
    int32_t* rx = nullptr;
    int32_t* ry = nullptr;
    int32_t* rz = nullptr;
    uint32_t* rid = nullptr;
    uint32_t* kpos = nullptr;  // base + point id -> position (inverse of rid per tree)
    uint32_t* mlpos = nullptr;
    uint32_t* mrpos = nullptr;
    // nodes
    uint32_t node_cap = 0, node_count = 0;
    int32_t* c1 = nullptr;
    int32_t* c2 = nullptr;
    int32_t* feat = nullptr;
    uint32_t* nb = nullptr;
    uint32_t* ne = nullptr;
    double* dlo = nullptr;
    double* dhi = nullptr;
    int32_t* bmin = nullptr;  // 3 per node
    int32_t* bmax = nullptr;
    // segments of the current and next level, pass-2 views
    KdSeg* seg[2] = {nullptr, nullptr};
    KdSeg* seg2 = nullptr;
    KdSplit* split = nullptr;
    KdSplit* split2 = nullptr;     // pass-2 segments' split records
    uint32_t* seg2_from = nullptr; // pass-2 segment -> its level segment
    uint32_t seg_cap = 0;
    KdSeg* small = nullptr;      // segments left for the warp builder
    uint32_t* leaves = nullptr;  // leaves made by the level passes (bbox pending)
    uint32_t leaf_cap = 0;
    // tiles
    uint32_t* nt = nullptr;        // per segment tile count, then prefix (seg_cap+1)
    uint32_t* tile_seg = nullptr;
    unsigned long long* tile_cnt = nullptr;  // per tile counts (lt | eq << 32), then prefix
    uint32_t tile_cap = 0;
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    uint32_t* counters = nullptr;  // [0] next segments, [1] nodes, [2] errors, [3] small
                                   // segments, [4] leaves, [5] pass-2 segments
    uint32_t dl_cap = 0;
    uint64_t bytes = 0;
    std::vector<std::pair<void*, size_t>> blocks;  // device blocks owned
};

// A tile's view of its replica: the forest and the tile's tree in it.
struct KdReplica {
    KdForest* f = nullptr;
    int tree = 0;
    bool built = false;
};

// ---------------------------------------------------------------------------
// build kernels
// ---------------------------------------------------------------------------
__global__ void kd_init_kernel(const int32_t* x, const int32_t* y, const int32_t* z, uint64_t n,
                               int32_t* rx, int32_t* ry, int32_t* rz, uint32_t* rid) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        rx[i] = x[i];
        ry[i] = y[i];
        rz[i] = z[i];
        rid[i] = (uint32_t)i;
    }
}

__global__ void kd_seg_tiles_kernel(const KdSeg* segs, uint32_t S, uint32_t* nt) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) nt[s] = (segs[s].end - segs[s].begin + KD_TILE - 1) / KD_TILE;
    if (s == S) nt[s] = 0;
}

__global__ void kd_fill_tiles_kernel(const uint32_t* tile_first, uint32_t S, uint32_t ntiles,
                                     uint32_t* tile_seg) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    // last segment whose first tile <= t
    uint32_t lo = 0, hi = S;  // answer in [lo, hi)
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (tile_first[mid] <= t) lo = mid;
        else hi = mid;
    }
    tile_seg[t] = lo;
}

__global__ void kd_minmax_init_kernel(KdSplit* sp, uint32_t S) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    for (int d = 0; d < 3; ++d) {
        sp[s].mn[d] = INT32_MAX;
        sp[s].mx[d] = INT32_MIN;
    }
}

// Segment extents: each tile's block reduction folded into its segment's
// split record with integer atomics (mn/mx start at INT32_MAX/INT32_MIN).
__global__ void __launch_bounds__(KD_THREADS) kd_minmax_kernel(const KdSeg* segs, const uint32_t* tile_first,
                                                               const uint32_t* tile_seg,
                                                               const int32_t* rx, const int32_t* ry,
                                                               const int32_t* rz, KdSplit* sp,
                                                               uint32_t ntiles) {
    __shared__ int32_t red[KD_THREADS / 32][6];
    // tiles in strides of the grid (capped beside a query: see kd_grid)
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t s = tile_seg[t];
        const KdSeg sg = segs[s];
        const uint32_t i0 = sg.begin + (t - tile_first[s]) * KD_TILE + threadIdx.x;
        int32_t v[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, w[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            const uint32_t i = i0 + k * KD_THREADS;
            if (i < sg.end) {
                const int32_t c[3] = {rx[i], ry[i], rz[i]};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    v[d] = min(v[d], c[d]);
                    w[d] = max(w[d], c[d]);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = __reduce_min_sync(0xffffffffu, v[d]);
            w[d] = __reduce_max_sync(0xffffffffu, w[d]);
        }
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) {
            for (int d = 0; d < 3; ++d) {
                red[warp][d] = v[d];
                red[warp][3 + d] = w[d];
            }
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            int32_t r = red[0][threadIdx.x];
            for (int k = 1; k < KD_THREADS / 32; ++k)
                r = threadIdx.x < 3 ? min(r, red[k][threadIdx.x]) : max(r, red[k][threadIdx.x]);
            if (threadIdx.x < 3) atomicMin(&sp[s].mn[threadIdx.x], r);
            else atomicMax(&sp[s].mx[threadIdx.x - 3], r);
        }
        __syncthreads();
    }
}

// Cut feature and value of a segment from its top-down box (lo, hi) and its
// points' extents (mn, mx): nanoflann.hpp:779-828 middleSplit_.
__device__ __forceinline__ void kd_choose_cut(const double lo[3], const double hi[3],
                                              const int32_t mn_[3], const int32_t mx_[3],
                                              const Transform& tf, int& cutfeat, double& cutval) {
    const double EPS = 0.00001;
    double max_span = __dsub_rn(hi[0], lo[0]);
    for (int i = 1; i < 3; ++i) {
        double span = __dsub_rn(hi[i], lo[i]);
        if (span > max_span) max_span = span;
    }
    double max_spread = -1;
    cutfeat = 0;
    for (int i = 0; i < 3; ++i) {
        double span = __dsub_rn(hi[i], lo[i]);
        if (span > __dmul_rn(__dsub_rn(1.0, EPS), max_span)) {
            double mn = ref_coord(mn_[i], tf.scale[i], tf.offset[i]);
            double mx = ref_coord(mx_[i], tf.scale[i], tf.offset[i]);
            double spread = __dsub_rn(mx, mn);
            if (spread > max_spread) {
                cutfeat = i;
                max_spread = spread;
            }
        }
    }
    double split_val = __ddiv_rn(__dadd_rn(lo[cutfeat], hi[cutfeat]), 2.0);
    double mn = ref_coord(mn_[cutfeat], tf.scale[cutfeat], tf.offset[cutfeat]);
    double mx = ref_coord(mx_[cutfeat], tf.scale[cutfeat], tf.offset[cutfeat]);
    if (split_val < mn) cutval = mn;
    else if (split_val > mx) cutval = mx;
    else cutval = split_val;
}

__global__ void kd_split_kernel(const KdSeg* segs, uint32_t S, KdSplit* sp, const Transform* tfs,
                                int32_t* bmin, int32_t* bmax) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const KdSeg sg = segs[s];
    const Transform tf = tfs[sg.pad];
    KdSplit p = sp[s];
    // the node's extents are its points' extents
    for (int d = 0; d < 3; ++d) {
        bmin[3 * sg.node + d] = p.mn[d];
        bmax[3 * sg.node + d] = p.mx[d];
    }
    int cutfeat;
    double cutval;
    kd_choose_cut(sg.lo, sg.hi, p.mn, p.mx, tf, cutfeat, cutval);
    sp[s].f = cutfeat;
    sp[s].cutval = cutval;
}

__device__ __forceinline__ int32_t kd_coord(const int32_t* rx, const int32_t* ry,
                                            const int32_t* rz, int f, uint32_t i) {
    return f == 0 ? rx[i] : (f == 1 ? ry[i] : rz[i]);
}

// pass 1: x < cutval; pass 2: x <= cutval
template <int PASS>
__device__ __forceinline__ bool kd_pred(double v, double cut) {
    return PASS == 1 ? (v < cut) : (v <= cut);
}

// Per tile: predicate count in the low 32 bits and, on pass 1, the count of
// points equal to the cut value in the high 32 bits.
template <int PASS>
__global__ void __launch_bounds__(KD_THREADS) kd_count_kernel(const KdSeg* segs, const uint32_t* tile_first,
                                                              const uint32_t* tile_seg,
                                                              const KdSplit* sp, const int32_t* rx,
                                                              const int32_t* ry, const int32_t* rz,
                                                              const Transform* tfs,
                                                              unsigned long long* tile_cnt,
                                                              uint32_t ntiles) {
    __shared__ unsigned long long red[KD_THREADS / 32];
    // tiles in strides of the grid (capped beside a query: see kd_grid)
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t s = tile_seg[t];
        const KdSeg sg = segs[s];
        const Transform& tf = tfs[sg.pad];
        const int f = sp[s].f;
        const double cut = sp[s].cutval;
        const int32_t* rc = f == 0 ? rx : (f == 1 ? ry : rz);
        const uint32_t i0 = sg.begin + (t - tile_first[s]) * KD_TILE + threadIdx.x;
        unsigned long long c = 0;
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            const uint32_t i = i0 + k * KD_THREADS;
            if (i < sg.end) {
                const double v = ref_coord(rc[i], tf.scale[f], tf.offset[f]);
                c += kd_pred<PASS>(v, cut) ? 1ull : 0ull;
                if (PASS == 1 && v == cut) c += 1ull << 32;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long r = 0;
            for (int k = 0; k < KD_THREADS / 32; ++k) r += red[k];
            tile_cnt[t] = r;
        }
        __syncthreads();
    }
}

// L and the number of misplaced pairs m for each segment (one warp each: the
// count before L inside L's tile is recounted by the warp).
template <int PASS>
__global__ void kd_seg_count_kernel(const KdSeg* segs, uint32_t S, const uint32_t* tile_first,
                                    const unsigned long long* tile_pref, KdSplit* sp, const int32_t* rx,
                                    const int32_t* ry, const int32_t* rz, const Transform* tfs) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= S) return;
    const KdSeg sg = segs[s];
    const Transform& tf = tfs[sg.pad];
    const uint32_t first = tile_first[s], nt = tile_first[s + 1] - first;
    const uint32_t len = sg.end - sg.begin;
    const int f = sp[s].f;
    const double cut = sp[s].cutval;
    const int32_t* rc = f == 0 ? rx : (f == 1 ? ry : rz);
    const unsigned long long tot = tile_pref[first + nt] - tile_pref[first];
    const uint32_t L = (uint32_t)tot, eq = (uint32_t)(tot >> 32);
    const uint32_t tl = L / KD_TILE;
    uint32_t pleft = 0;
    if (len) {
        pleft = (uint32_t)(tile_pref[first + tl] - tile_pref[first]);
        for (uint32_t base = sg.begin + tl * KD_TILE; base < sg.begin + L; base += 32) {
            const uint32_t i = base + lane;
            const bool p = i < sg.begin + L &&
                           kd_pred<PASS>(ref_coord(rc[i], tf.scale[f], tf.offset[f]), cut);
            pleft += __popc(__ballot_sync(0xffffffffu, p));
        }
    }
    if (lane) return;
    const uint32_t m = L - pleft;
    if (PASS == 1) {
        sp[s].L = L;
        sp[s].m = m;
        sp[s].eq = eq;
    } else {
        sp[s].L2 = L;
        sp[s].m2 = m;
    }
}

template <int PASS>
__global__ void __launch_bounds__(KD_THREADS) kd_classify_kernel(const KdSeg* segs, const uint32_t* tile_first,
                                                                 const uint32_t* tile_seg,
                                                                 const unsigned long long* tile_pref,
                                                                 const KdSplit* sp, const int32_t* rx,
                                                                 const int32_t* ry, const int32_t* rz,
                                                                 const Transform* tfs, uint32_t* mlpos,
                                                                 uint32_t* mrpos,
                                                                 uint32_t ntiles) {
    typedef cub::BlockScan<uint32_t, KD_THREADS> Scan;
    __shared__ typename Scan::TempStorage tmp;
    // tiles in strides of the grid (capped beside a query: see kd_grid)
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t s = tile_seg[t];
        const KdSeg sg = segs[s];
        const Transform& tf = tfs[sg.pad];
        const int f = sp[s].f;
        const double cut = sp[s].cutval;
        const int32_t* rc = f == 0 ? rx : (f == 1 ? ry : rz);
        const uint32_t L = PASS == 1 ? sp[s].L : sp[s].L2;
        const uint32_t m = PASS == 1 ? sp[s].m : sp[s].m2;
        // blocked arrangement: thread j owns elements j*KD_ITEMS .. j*KD_ITEMS+KD_ITEMS-1
        const uint32_t i0 = sg.begin + (t - tile_first[s]) * KD_TILE + threadIdx.x * KD_ITEMS;
        uint32_t p[KD_ITEMS], rank[KD_ITEMS];
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            const uint32_t i = i0 + k;
            p[k] = i < sg.end && kd_pred<PASS>(ref_coord(rc[i], tf.scale[f], tf.offset[f]), cut);
        }
        Scan(tmp).ExclusiveSum(p, rank);
        const uint32_t before = (uint32_t)(tile_pref[t] - tile_pref[tile_first[s]]);
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            const uint32_t i = i0 + k;
            if (i >= sg.end) break;
            const uint32_t prank = before + rank[k];  // predicate holders before i in the segment
            const uint32_t li = i - sg.begin;
            if (li < L) {
                if (!p[k]) mlpos[sg.begin + (li - prank)] = i;
            } else if (p[k]) {
                const uint32_t rml = prank - (L - m);
                mrpos[sg.begin + (m - 1 - rml)] = i;
            }
        }
        __syncthreads();
    }
}

// The misplaced pairs of a tile: every load of the thread's pairs is issued
// before any store (each position belongs to exactly one pair of the level, so
// the loads never read what a store of this launch writes), which keeps the
// dependent position -> coordinate loads of all the thread's items in flight
// together instead of one item at a time.
template <int PASS>
__global__ void __launch_bounds__(KD_THREADS) kd_swap_kernel(const KdSeg* __restrict__ segs,
                                                             const uint32_t* __restrict__ tile_first,
                                                             const uint32_t* __restrict__ tile_seg,
                                                             const KdSplit* __restrict__ sp,
                                                             const uint32_t* __restrict__ mlpos,
                                                             const uint32_t* __restrict__ mrpos,
                                                             int32_t* __restrict__ rx,
                                                             int32_t* __restrict__ ry,
                                                             int32_t* __restrict__ rz,
                                                             uint32_t* __restrict__ rid,
                                                             uint32_t ntiles) {
    // tiles in strides of the grid (capped beside a query: see kd_grid)
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t s = tile_seg[t];
        const KdSeg sg = segs[s];
        const uint32_t m = PASS == 1 ? sp[s].m : sp[s].m2;
        const uint32_t l0 = (t - tile_first[s]) * KD_TILE + threadIdx.x;
        if (l0 >= m) continue;
        uint32_t a[KD_ITEMS], b[KD_ITEMS];
        int32_t ax[KD_ITEMS], ay[KD_ITEMS], az[KD_ITEMS], bx[KD_ITEMS], by[KD_ITEMS], bz[KD_ITEMS];
        uint32_t ai[KD_ITEMS], bi[KD_ITEMS];
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            const uint32_t li = l0 + k * KD_THREADS;
            if (li < m) {
                a[k] = mlpos[sg.begin + li];
                b[k] = mrpos[sg.begin + li];
            }
        }
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            if (l0 + k * KD_THREADS < m) {
                ax[k] = rx[a[k]];
                ay[k] = ry[a[k]];
                az[k] = rz[a[k]];
                ai[k] = rid[a[k]];
                bx[k] = rx[b[k]];
                by[k] = ry[b[k]];
                bz[k] = rz[b[k]];
                bi[k] = rid[b[k]];
            }
        }
#pragma unroll
        for (int k = 0; k < KD_ITEMS; ++k) {
            if (l0 + k * KD_THREADS < m) {
                rx[a[k]] = bx[k];
                ry[a[k]] = by[k];
                rz[a[k]] = bz[k];
                rid[a[k]] = bi[k];
                rx[b[k]] = ax[k];
                ry[b[k]] = ay[k];
                rz[b[k]] = az[k];
                rid[b[k]] = ai[k];
            }
        }
    }
}

// Pass 2 runs only on segments with points equal to the cut value: every
// other segment has L2 = m2 = 0.  Listed segments start at their L and keep
// their own split record (copied), written back after the pass.
__global__ void kd_pass2_plan_kernel(const KdSeg* segs, uint32_t S, KdSplit* sp, KdSeg* seg2,
                                     KdSplit* split2, uint32_t* seg2_from, uint32_t* count) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const KdSplit p = sp[s];
    sp[s].L2 = 0;
    sp[s].m2 = 0;
    if (p.eq == 0) return;
    const uint32_t k = atomicAdd(count, 1u);
    KdSeg g = segs[s];
    g.begin = g.begin + p.L;
    seg2[k] = g;
    split2[k] = p;
    seg2_from[k] = s;
}

__global__ void kd_pass2_done_kernel(uint32_t S2, const KdSplit* split2, const uint32_t* seg2_from,
                                     KdSplit* sp) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S2) return;
    sp[seg2_from[k]].L2 = split2[k].L2;
    sp[seg2_from[k]].m2 = split2[k].m2;
}

__global__ void kd_children_kernel(const KdSeg* segs, uint32_t S, const KdSplit* sp, KdSeg* next,
                                   uint32_t* counters, int32_t* c1, int32_t* c2, int32_t* feat,
                                   uint32_t* nb, uint32_t* ne, uint32_t node_cap, uint32_t seg_cap,
                                   KdSeg* small, uint32_t small_max, uint32_t* leaves,
                                   uint32_t leaf_cap, int32_t* ntree) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const KdSeg sg = segs[s];
    const KdSplit p = sp[s];
    const uint32_t count = sg.end - sg.begin;
    const uint32_t lim1 = p.L, lim2 = p.L + p.L2;
    uint32_t index;
    if (lim1 > count / 2) index = lim1;
    else if (lim2 < count / 2) index = lim2;
    else index = count / 2;
    const uint32_t cid = atomicAdd(&counters[1], 2u);
    if (cid + 2 > node_cap) {
        atomicAdd(&counters[2], 1u);
        return;
    }
    c1[sg.node] = (int32_t)cid;
    c2[sg.node] = (int32_t)(cid + 1);
    feat[sg.node] = p.f;
    for (int side = 0; side < 2; ++side) {
        const uint32_t node = cid + side;
        KdSeg ch = sg;
        if (side == 0) {
            ch.end = sg.begin + index;
            ch.hi[p.f] = p.cutval;
        } else {
            ch.begin = sg.begin + index;
            ch.lo[p.f] = p.cutval;
        }
        ch.node = (int32_t)node;
        nb[node] = ch.begin;
        ne[node] = ch.end;
        c1[node] = -1;
        c2[node] = -1;
        feat[node] = 0;
        ntree[node] = sg.pad;
        const uint32_t len = ch.end - ch.begin;
        if (len <= (uint32_t)KD_LEAF) {
            const uint32_t slot = atomicAdd(&counters[4], 1u);
            if (slot < leaf_cap) leaves[slot] = node;
            else atomicAdd(&counters[2], 1u);
        } else if (len <= small_max) {
            const uint32_t slot = atomicAdd(&counters[3], 1u);
            if (slot < seg_cap) small[slot] = ch;
            else atomicAdd(&counters[2], 1u);
        } else {
            const uint32_t slot = atomicAdd(&counters[0], 1u);
            if (slot < seg_cap) next[slot] = ch;
            else atomicAdd(&counters[2], 1u);
        }
    }
}

// Extents of [b, e) by one warp (INT32_MAX / INT32_MIN when empty).
__device__ __forceinline__ void kd_warp_minmax(const int32_t* rx, const int32_t* ry, const int32_t* rz,
                                               uint32_t b, uint32_t e, int lane, int32_t mn[3],
                                               int32_t mx[3]) {
    int32_t v[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, w[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (uint32_t i = b + lane; i < e; i += 32) {
        const int32_t c[3] = {rx[i], ry[i], rz[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = min(v[d], c[d]);
            w[d] = max(w[d], c[d]);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mn[d] = __reduce_min_sync(0xffffffffu, v[d]);
        mx[d] = __reduce_max_sync(0xffffffffu, w[d]);
    }
}

// Leaves made by the level passes: their extents, one warp per leaf.
__global__ void kd_leaf_bbox_kernel(const uint32_t* leaves, uint32_t nleaves, const uint32_t* nb,
                                    const uint32_t* ne, const int32_t* rx, const int32_t* ry,
                                    const int32_t* rz, int32_t* bmin, int32_t* bmax) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nleaves) return;
    const uint32_t node = leaves[w];
    int32_t mn[3], mx[3];
    kd_warp_minmax(rx, ry, rz, nb[node], ne[node], lane, mn, mx);
    if (lane < 3) {
        bmin[3 * node + lane] = mn[lane];
        bmax[3 * node + lane] = mx[lane];
    }
}

// One Hoare pass of nanoflann's planeSplit over [b, e) by one warp: with L
// the count satisfying the predicate, the t-th element from the left failing
// it inside [b, b+L) swaps with the t-th element from the right satisfying it
// inside [b+L, e).  Returns L; *eq (pass 1) counts the elements equal to the
// cut value, the only ones pass 2 can move.  mlpos/mrpos[b ...] are the
// warp's scratch.
template <int PASS>
__device__ uint32_t kd_warp_pass(int32_t* rx, int32_t* ry, int32_t* rz, uint32_t* rid,
                                 uint32_t* mlpos, uint32_t* mrpos, uint32_t b, uint32_t e, int f,
                                 double cut, const Transform& tf, int lane, uint32_t* eq = nullptr) {
    const int32_t* rc = f == 0 ? rx : (f == 1 ? ry : rz);
    const double sc = tf.scale[f], of = tf.offset[f];
    const unsigned lt = (1u << lane) - 1u;
    uint32_t L = 0, neq = 0;
    for (uint32_t base = b; base < e; base += 32) {
        const uint32_t i = base + lane;
        const double v = i < e ? ref_coord(rc[i], sc, of) : 0.0;
        const bool p = i < e && kd_pred<PASS>(v, cut);
        L += __popc(__ballot_sync(0xffffffffu, p));
        if (PASS == 1) neq += __popc(__ballot_sync(0xffffffffu, i < e && v == cut));
    }
    if (eq) *eq = neq;
    uint32_t m = 0;
    for (uint32_t base = b; base < b + L; base += 32) {
        const uint32_t i = base + lane;
        const bool q = i < b + L && !kd_pred<PASS>(ref_coord(rc[i], sc, of), cut);
        const unsigned mask = __ballot_sync(0xffffffffu, q);
        if (q) mlpos[b + m + __popc(mask & lt)] = i;
        m += __popc(mask);
    }
    uint32_t r = 0;
    for (uint32_t base = b + L; base < e; base += 32) {
        const uint32_t i = base + lane;
        const bool q = i < e && kd_pred<PASS>(ref_coord(rc[i], sc, of), cut);
        const unsigned mask = __ballot_sync(0xffffffffu, q);
        if (q) {
            const uint32_t k = r + __popc(mask & lt);
            if (k < m) mrpos[b + (m - 1 - k)] = i;
        }
        r += __popc(mask);
    }
    __syncwarp();
    for (uint32_t t = lane; t < m; t += 32) {
        const uint32_t a = mlpos[b + t], c = mrpos[b + t];
        const int32_t tx = rx[a], ty = ry[a], tz = rz[a];
        const uint32_t ti = rid[a];
        rx[a] = rx[c];
        ry[a] = ry[c];
        rz[a] = rz[c];
        rid[a] = rid[c];
        rx[c] = tx;
        ry[c] = ty;
        rz[c] = tz;
        rid[c] = ti;
    }
    __syncwarp();
    return L;
}

// Builds the whole subtree of each listed segment, one warp per segment,
// depth first with an explicit stack in shared memory.  Same split rules as
// the level passes; nodes are numbered by an atomic counter.  counters[2]
// counts capacity or stack overflows (the host then rebuilds level by level).
__global__ void __launch_bounds__(32 * KD_WARPS) kd_warp_build_kernel(
    const KdSeg* small, uint32_t nsmall, int32_t* rx, int32_t* ry, int32_t* rz, uint32_t* rid,
    uint32_t* mlpos, uint32_t* mrpos, int32_t* c1, int32_t* c2, int32_t* feat, uint32_t* nb,
    uint32_t* ne, int32_t* bmin, int32_t* bmax, uint32_t* counters, uint32_t node_cap,
    const Transform* tfs, int32_t* ntree) {
    __shared__ KdSeg stk[KD_WARPS][KD_WSTACK];
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    KdSeg* st = stk[wl];
    // segments in strides of the grid's warps (capped beside a query)
    for (uint32_t w = blockIdx.x * KD_WARPS + wl; w < nsmall; w += gridDim.x * KD_WARPS) {
        if (lane == 0) st[0] = small[w];
        int top = 1;
        __syncwarp();
        while (top > 0) {
            const KdSeg sg = st[top - 1];
            --top;
            __syncwarp();
            const uint32_t b = sg.begin, e = sg.end, count = e - b;
            const int node = sg.node;
            int32_t mn[3], mx[3];
            kd_warp_minmax(rx, ry, rz, b, e, lane, mn, mx);
            if (lane < 3) {
                bmin[3 * node + lane] = mn[lane];
                bmax[3 * node + lane] = mx[lane];
            }
            if (count <= (uint32_t)KD_LEAF) continue;
            const Transform tf = tfs[sg.pad];
            int f;
            double cut;
            kd_choose_cut(sg.lo, sg.hi, mn, mx, tf, f, cut);
            uint32_t eq = 0;
            const uint32_t L = kd_warp_pass<1>(rx, ry, rz, rid, mlpos, mrpos, b, e, f, cut, tf, lane, &eq);
            // pass 2 (<= cut on [b+L, e), which pass 1 left holding the elements
            // >= cut) moves only elements equal to the cut value: with none, its
            // count is 0 and it swaps nothing
            const uint32_t L2 =
                eq ? kd_warp_pass<2>(rx, ry, rz, rid, mlpos, mrpos, b + L, e, f, cut, tf, lane) : 0u;
            const uint32_t lim1 = L, lim2 = L + L2;
            uint32_t index;
            if (lim1 > count / 2) index = lim1;
            else if (lim2 < count / 2) index = lim2;
            else index = count / 2;
            uint32_t cid = 0;
            if (lane == 0) cid = atomicAdd(&counters[1], 2u);
            cid = __shfl_sync(0xffffffffu, cid, 0);
            if (cid + 2 > node_cap || top + 2 > KD_WSTACK) {
                if (lane == 0) atomicAdd(&counters[2], 1u);
                return;
            }
            if (lane == 0) {
                c1[node] = (int32_t)cid;
                c2[node] = (int32_t)(cid + 1);
                feat[node] = f;
                for (int side = 1; side >= 0; --side) {
                    KdSeg ch = sg;
                    if (side == 0) {
                        ch.end = b + index;
                        ch.hi[f] = cut;
                    } else {
                        ch.begin = b + index;
                        ch.lo[f] = cut;
                    }
                    ch.node = (int32_t)(cid + side);
                    nb[cid + side] = ch.begin;
                    ne[cid + side] = ch.end;
                    c1[cid + side] = -1;
                    c2[cid + side] = -1;
                    feat[cid + side] = 0;
                    ntree[cid + side] = sg.pad;
                    st[top + (1 - side)] = ch;
                }
            }
            top += 2;
            __syncwarp();
        }
    }
}

__global__ void kd_div_kernel(uint32_t nodes, const int32_t* c1, const int32_t* c2,
                              const int32_t* feat, const int32_t* bmin, const int32_t* bmax,
                              const Transform* tfs, const int32_t* ntree, double* dlo, double* dhi) {
    uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nodes || c1[node] < 0) return;
    const int f = feat[node];
    const Transform& tf = tfs[ntree[node]];
    dlo[node] = ref_coord(bmax[3 * c1[node] + f], tf.scale[f], tf.offset[f]);
    dhi[node] = ref_coord(bmin[3 * c2[node] + f], tf.scale[f], tf.offset[f]);
}

// kpos[base + id] = position of point id of the tree starting at base.
__global__ void kd_inverse_kernel(const uint32_t* rid, uint64_t base, uint64_t n, uint32_t* kpos) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        kpos[base + rid[base + i]] = (uint32_t)(base + i);
}

// ---------------------------------------------------------------------------
// search replay
// ---------------------------------------------------------------------------
struct KdResult {
    double dist[KD_CAP];
    uint32_t idx[KD_CAP];
    int count, cap;
    __device__ __forceinline__ void init(int c) {
        cap = c;
        count = 0;
        dist[cap - 1] = DBL_MAX;
    }
    __device__ __forceinline__ double worst() const { return dist[cap - 1]; }
    __device__ __forceinline__ void add(double d, uint32_t id) {
        int i;
        for (i = count; i > 0; --i) {
            if (dist[i - 1] > d) {
                if (i < cap) {
                    dist[i] = dist[i - 1];
                    idx[i] = idx[i - 1];
                }
            } else break;
        }
        if (i < cap) {
            dist[i] = d;
            idx[i] = id;
        }
        if (count < cap) count++;
    }
};

// One DFS frame: the node, the bound it was entered with and, once its
// best child is done, the saved per-dimension distance.  The child order
// and cut distance are recomputed from the node when needed.
struct KdFrame {
    double mind, dst;
    int32_t node, phase;
};

__device__ __forceinline__ double kd_sq(double a, double b) {
    double d = __dsub_rn(a, b);
    return __dmul_rn(d, d);
}

// Squared FP64 distance from q to replica position i, as the reference forms it.
__device__ __forceinline__ double kd_point_dist(const KdDev& kd, const Transform& tf,
                                                const double q[3], uint32_t i) {
    const double p0 = ref_coord(kd.rx[i], tf.scale[0], tf.offset[0]);
    const double p1 = ref_coord(kd.ry[i], tf.scale[1], tf.offset[1]);
    const double p2 = ref_coord(kd.rz[i], tf.scale[2], tf.offset[2]);
    const double d0 = __dsub_rn(q[0], p0);
    const double d1 = __dsub_rn(q[1], p1);
    const double d2 = __dsub_rn(q[2], p2);
    return __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
}

// Returns false when the explicit stack overflowed (never for sane trees).
// WARP: the 32 lanes of a warp replay one row together.  Every lane walks the
// same nodes and keeps the same result list; a leaf's points are measured 32
// at a time and its candidates (below the worst distance taken at the leaf's
// start, as the reference's leaf loop takes it) are inserted by every lane in
// leaf order, so the list is the single-thread replay's exactly.
template <bool WARP>
__device__ bool kd_search(const KdDev& kd, const Transform& tf, const double q[3], KdResult& rs) {
    double dists[3] = {0.0, 0.0, 0.0};
    double distsq = 0.0;
    for (int i = 0; i < 3; ++i) {
        if (q[i] < kd.root_lo[i]) {
            dists[i] = kd_sq(q[i], kd.root_lo[i]);
            distsq = __dadd_rn(distsq, dists[i]);
        }
        if (q[i] > kd.root_hi[i]) {
            dists[i] = kd_sq(q[i], kd.root_hi[i]);
            distsq = __dadd_rn(distsq, dists[i]);
        }
    }
    KdFrame st[KD_STACK];
    int top = 0;
    st[0].node = kd.root;
    st[0].mind = distsq;
    st[0].phase = 0;
    while (top >= 0) {
        const int node = st[top].node;
        const int phase = st[top].phase;
        if (phase == 0 && kd.c1[node] < 0) {
            const double worst = rs.worst();
            const uint32_t b = kd.nb[node], e = kd.ne[node];
            if (WARP) {
                const int lane = threadIdx.x & 31;
                for (uint32_t base = b; base < e; base += 32) {
                    const uint32_t i = base + lane;
                    double dist = 0.0;
                    uint32_t id = 0;
                    bool c = false;
                    if (i < e) {
                        dist = kd_point_dist(kd, tf, q, i);
                        id = kd.rid[i];
                        c = dist < worst;
                    }
                    unsigned m = __ballot_sync(0xffffffffu, c);
                    while (m) {
                        const int l = __ffs(m) - 1;
                        m &= m - 1;
                        rs.add(__shfl_sync(0xffffffffu, dist, l), __shfl_sync(0xffffffffu, id, l));
                    }
                }
            } else {
                for (uint32_t i = b; i < e; ++i) {
                    const double dist = kd_point_dist(kd, tf, q, i);
                    if (dist < worst) rs.add(dist, kd.rid[i]);
                }
            }
            --top;
            continue;
        }
        const int idx = kd.feat[node];
        const double val = q[idx];
        const double diff1 = __dsub_rn(val, kd.dlo[node]);
        const double diff2 = __dsub_rn(val, kd.dhi[node]);
        const bool left_first = __dadd_rn(diff1, diff2) < 0;
        if (phase == 0) {
            st[top].phase = 1;
            if (top + 1 >= KD_STACK) return false;
            ++top;
            st[top].node = left_first ? kd.c1[node] : kd.c2[node];
            st[top].mind = st[top - 1].mind;
            st[top].phase = 0;
        } else if (phase == 1) {
            const double cut = left_first ? kd_sq(val, kd.dhi[node]) : kd_sq(val, kd.dlo[node]);
            const double dst = dists[idx];
            const double mind2 = __dsub_rn(__dadd_rn(st[top].mind, cut), dst);
            dists[idx] = cut;
            st[top].dst = dst;
            st[top].phase = 2;
            if (mind2 <= rs.worst()) {
                if (top + 1 >= KD_STACK) return false;
                ++top;
                st[top].node = left_first ? kd.c2[node] : kd.c1[node];
                st[top].mind = mind2;
                st[top].phase = 0;
            }
        } else {
            dists[idx] = st[top].dst;
            --top;
        }
    }
    return true;
}

// Replays the reference's search for each listed row, one warp per row, and
// writes its K neighbour ids (the reference's order) to nbr[r*K ...].
__global__ void __launch_bounds__(128) kd_search_kernel(KdDev kd, Transform tf, const int32_t* __restrict__ x,
                                 const int32_t* __restrict__ y, const int32_t* __restrict__ z,
                                 const uint32_t* __restrict__ rows, uint32_t nrows, int K,
                                 uint32_t* __restrict__ nbr, uint32_t* __restrict__ counts,
                                 uint32_t* errors, const double* row_k, uint64_t npts) {
    const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= nrows) return;  // whole warps leave together
    const uint32_t id = rows[r];
    const int Kr = row_neighbours(row_k, K, npts, id);  // <= K
    const double q[3] = {ref_coord(x[id], tf.scale[0], tf.offset[0]),
                         ref_coord(y[id], tf.scale[1], tf.offset[1]),
                         ref_coord(z[id], tf.scale[2], tf.offset[2])};
    if (Kr <= 0) {
        if (lane == 0) counts[r] = 0;
        return;
    }
    KdResult rs;
    rs.init(Kr);
    const bool ok = kd_search<true>(kd, tf, q, rs);
    for (int s = lane; s < K; s += 32) nbr[(uint64_t)r * K + s] = s < rs.count ? rs.idx[s] : 0u;
    if (lane == 0) {
        counts[r] = ok ? (uint32_t)rs.count : 0u;
        if (!ok) atomicAdd(errors, 1u);
    }
}

// Covariance of the replayed neighbour lists and the stage projections.
__global__ void kd_finish_kernel(Transform tf, const int32_t* __restrict__ x,
                                 const int32_t* __restrict__ y, const int32_t* __restrict__ z,
                                 const uint32_t* __restrict__ rows, uint32_t nrows, int K,
                                 const uint32_t* __restrict__ nbr,
                                 const uint32_t* __restrict__ counts, StageGroup g,
                                 ExceptionSink ex, int stride, int kpick) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const uint32_t id = rows[r];
    const int32_t qraw[3] = {x[id], y[id], z[id]};
    // with a stride the reference keeps entries 0, stride, ... of its k*stride
    // list, unfilled entries reading point 0 (KDImpl.hpp:359-380)
    const int cnt = stride > 1 ? kpick : (int)counts[r];
    long long s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < cnt; ++s) {
        const uint32_t j = nbr[(uint64_t)r * K + (uint64_t)s * (stride > 1 ? stride : 1)];
        const long long d0 = (long long)x[j] - qraw[0];
        const long long d1 = (long long)y[j] - qraw[1];
        const long long d2 = (long long)z[j] - qraw[2];
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
    const long long n = cnt;
    long long M[6];
    M[0] = n * s2[0] - s1[0] * s1[0];
    M[1] = n * s2[1] - s1[1] * s1[0];
    M[2] = n * s2[2] - s1[1] * s1[1];
    M[3] = n * s2[3] - s1[2] * s1[0];
    M[4] = n * s2[4] - s1[2] * s1[1];
    M[5] = n * s2[5] - s1[2] * s1[2];
    nbg_finish_row(g, tf, ex, id, cnt, M, qraw);
}

// A kNN consumer's epilogue over replayed lists (already in the reference's
// order: the replay is its search).
__global__ void kd_list_finish_kernel(Transform tf, const int32_t* __restrict__ x,
                                      const int32_t* __restrict__ y, const int32_t* __restrict__ z,
                                      const uint32_t* __restrict__ rows, uint32_t nrows, int K,
                                      const uint32_t* __restrict__ nbr,
                                      const uint32_t* __restrict__ counts, ListArgs L,
                                      ExceptionSink ex) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    const uint32_t id = rows[r];
    const int32_t qraw[3] = {x[id], y[id], z[id]};
    const double q64[3] = {ref_coord(qraw[0], tf.scale[0], tf.offset[0]),
                           ref_coord(qraw[1], tf.scale[1], tf.offset[1]),
                           ref_coord(qraw[2], tf.scale[2], tf.offset[2])};
    const int cnt = min((int)counts[r], K);
    uint32_t ids[KD_CAP];
    int off[KD_CAP][3];
    double d[KD_CAP];
    for (int j = 0; j < cnt; ++j) {
        const uint32_t p = nbr[(uint64_t)r * K + j];
        ids[j] = p;
        off[j][0] = x[p] - qraw[0];
        off[j][1] = y[p] - qraw[1];
        off[j][2] = z[p] - qraw[2];
        d[j] = ref_dist2(q64, qraw, off[j], tf);
    }
    list_consume(L, tf, ex, id, qraw, cnt, ids, off, d);
}

// Neighbour-set export: ascending ids into ids_out[id*K ...].
__global__ void kd_scatter_ids_kernel(const uint32_t* __restrict__ rows, uint32_t nrows, int K,
                                      const uint32_t* __restrict__ nbr,
                                      const uint32_t* __restrict__ counts, uint32_t* ids_out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    uint32_t* row = ids_out + (uint64_t)rows[r] * K;
    const int cnt = (int)counts[r];
    for (int s = 0; s < cnt; ++s) {
        const uint32_t v = nbr[(uint64_t)r * K + s];
        int t = s - 1;
        while (t >= 0 && row[t] > v) {
            row[t + 1] = row[t];
            --t;
        }
        row[t + 1] = v;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int kd_alloc(Context* ctx, void** p, size_t bytes, KdForest* kd) {
    int rc = ctx_alloc(ctx, p, bytes);
    if (rc) return rc;
    kd->bytes += bytes;
    kd->blocks.emplace_back(*p, bytes);
    return NBG_OK;
}

static void kd_release(Context* ctx, KdForest* kd, void* p) {
    for (size_t i = 0; i < kd->blocks.size(); ++i)
        if (kd->blocks[i].first == p) {
            ctx_free(ctx, p, kd->blocks[i].second);
            kd->bytes -= kd->blocks[i].second;
            kd->blocks.erase(kd->blocks.begin() + i);
            return;
        }
}

template <class T>
static int kd_grow(Context* ctx, T** p, size_t old_n, size_t new_n, KdForest* kd, cudaStream_t st) {
    T* q = nullptr;
    int rc = kd_alloc(ctx, (void**)&q, new_n * sizeof(T), kd);
    if (rc) return rc;
    if (*p) {
        cudaMemcpyAsync(q, *p, old_n * sizeof(T), cudaMemcpyDeviceToDevice, st);
        cudaStreamSynchronize(st);
        kd_release(ctx, kd, *p);
    }
    *p = q;
    return NBG_OK;
}

uint64_t kd_bytes(uint64_t n) { return n * 28 + (n / 16 + 1024) * 68; }

static void kd_forest_free(Context* ctx, KdForest* f) {
    for (auto& b : f->blocks) ctx_free(ctx, b.first, b.second);
    delete f;
}

void kd_free(Context* ctx, Tile* t) {
    KdReplica* kd = t->kd;
    if (!kd) return;
    KdForest* f = kd->f;
    delete kd;
    t->kd = nullptr;
    if (f && --f->refs <= 0) kd_forest_free(ctx, f);
}

// Builds the tile list of `S` segments; returns the number of tiles.
static int kd_tiles(Context* ctx, KdForest* kd, const KdSeg* segs, uint32_t S, uint32_t* ntiles,
                    cudaStream_t st) {
    kd_seg_tiles_kernel<<<(S + 1 + 255) / 256, 256, 0, st>>>(segs, S, kd->nt);
    size_t tb = kd->scan_bytes;
    cub::DeviceScan::ExclusiveSum(kd->scan_tmp, tb, kd->nt, kd->nt, (int)(S + 1), st);
    uint32_t total = 0;
    cudaMemcpyAsync(&total, kd->nt + S, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_err(ctx, "KD tile scan failed");
        return NBG_ERR_CUDA;
    }
    if (total + 1 > kd->tile_cap) {
        uint32_t cap = std::max<uint32_t>(total + 1, kd->tile_cap * 2);
        if (kd->tile_seg) kd_release(ctx, kd, kd->tile_seg);
        if (kd->tile_cnt) kd_release(ctx, kd, kd->tile_cnt);
        kd->tile_seg = nullptr;
        kd->tile_cnt = nullptr;
        int rc = kd_alloc(ctx, (void**)&kd->tile_seg, (size_t)cap * 4, kd);
        if (!rc) rc = kd_alloc(ctx, (void**)&kd->tile_cnt, (size_t)(cap + 1) * 8, kd);
        if (rc) return rc;
        kd->tile_cap = cap;
    }
    if (total) kd_fill_tiles_kernel<<<(total + 255) / 256, 256, 0, st>>>(kd->nt, S, total, kd->tile_seg);
    NBG_LAUNCHED(3 + (total ? 1 : 0));
    *ntiles = total;
    return NBG_OK;
}

// Blocks of a level-pass launch over `ntiles` tiles: one per tile, or at most
// the forest's cap when the build shares the SMs with a query.
static unsigned kd_grid(const KdForest* kd, uint32_t ntiles) {
    return kd->grid_cap ? std::min(ntiles, kd->grid_cap) : ntiles;
}

// known_tiles: the tile count when the tile map of `segs` is already built
// (~0u: build it).
template <int PASS>
static int kd_pass(Context* ctx, KdForest* kd, const KdSeg* segs, uint32_t S, KdSplit* sp,
                   cudaStream_t st, uint32_t known_tiles = ~0u) {
    uint32_t ntiles = known_tiles;
    if (known_tiles == ~0u) {
        int rc = kd_tiles(ctx, kd, segs, S, &ntiles, st);
        if (rc) return rc;
    }
    if (ntiles) {
        kd_count_kernel<PASS><<<kd_grid(kd, ntiles), KD_THREADS, 0, st>>>(
            segs, kd->nt, kd->tile_seg, sp, kd->rx, kd->ry, kd->rz, kd->tfs, kd->tile_cnt, ntiles);
    }
    cudaMemsetAsync(kd->tile_cnt + ntiles, 0, 8, st);
    size_t tb = kd->scan_bytes;
    cub::DeviceScan::ExclusiveSum(kd->scan_tmp, tb, kd->tile_cnt, kd->tile_cnt, (int)(ntiles + 1), st);
    kd_seg_count_kernel<PASS><<<(S * 32 + 255) / 256, 256, 0, st>>>(segs, S, kd->nt, kd->tile_cnt,
                                                                    sp, kd->rx, kd->ry, kd->rz,
                                                                    kd->tfs);
    if (ntiles) {
        kd_classify_kernel<PASS><<<kd_grid(kd, ntiles), KD_THREADS, 0, st>>>(
            segs, kd->nt, kd->tile_seg, kd->tile_cnt, sp, kd->rx, kd->ry, kd->rz, kd->tfs, kd->mlpos,
            kd->mrpos, ntiles);
        kd_swap_kernel<PASS><<<kd_grid(kd, ntiles), KD_THREADS, 0, st>>>(
            segs, kd->nt, kd->tile_seg, sp, kd->mlpos, kd->mrpos, kd->rx, kd->ry, kd->rz, kd->rid, ntiles);
    }
    NBG_LAUNCHED(3 + (ntiles ? 3 : 0));
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

static int kd_grow_nodes(Context* ctx, KdForest* kd, uint32_t nc, cudaStream_t st) {
    const uint32_t old = kd->node_cap;
    if (nc <= old) return NBG_OK;
    int rc = kd_grow(ctx, &kd->c1, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->c2, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->feat, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->nb, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->ne, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->ntree, old, nc, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->bmin, (size_t)old * 3, (size_t)nc * 3, kd, st);
    if (!rc) rc = kd_grow(ctx, &kd->bmax, (size_t)old * 3, (size_t)nc * 3, kd, st);
    if (rc) return rc;
    kd->node_cap = nc;
    return NBG_OK;
}

static unsigned grid_for(const Context* ctx, uint64_t n) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, ctx->sm_count * 8));
}

// One build of the forest over `tiles`; `small_max` = 0 keeps every level on
// the level passes (the fallback when a warp subtree overflows its stack or
// the node arrays).
static int kd_build(Context* ctx, KdForest* kd, Tile* const* tiles, uint32_t small_max,
                    cudaStream_t st) {
    const int T = kd->ntrees;
    int rc = NBG_OK;
    std::vector<KdSeg> level0, small0;
    std::vector<uint32_t> leaves0;
    std::vector<int32_t> c_init(T, -1), f_init(T, 0), tree_init(T);
    std::vector<uint32_t> nb_init(T), ne_init(T);
    for (int k = 0; k < T; ++k) {
        const Tile* t = tiles[k];
        const uint64_t b = kd->base[k], n = kd->npts[k];
        kd_init_kernel<<<grid_for(ctx, n), 256, 0, st>>>(t->x, t->y, t->z, n, kd->rx + b, kd->ry + b,
                                                         kd->rz + b, kd->rid + b);
        // root: the tile's actual bounding box, as calculateBounds
        const GridParams& g = t->host_gp;
        const int32_t mn[3] = {g.minx, g.miny, g.minz}, mx[3] = {g.maxx, g.maxy, g.maxz};
        KdSeg root;
        root.begin = (uint32_t)b;
        root.end = (uint32_t)(b + n);
        root.node = k;
        root.pad = k;
        for (int d = 0; d < 3; ++d) {
            root.lo[d] = (double)mn[d] * t->tf.scale[d] + t->tf.offset[d];
            root.hi[d] = (double)mx[d] * t->tf.scale[d] + t->tf.offset[d];
            kd->rootbox[6 * k + d] = root.lo[d];
            kd->rootbox[6 * k + 3 + d] = root.hi[d];
        }
        tree_init[k] = k;
        nb_init[k] = root.begin;
        ne_init[k] = root.end;
        if (n > (uint64_t)KD_LEAF && n > small_max) level0.push_back(root);
        else if (n > (uint64_t)KD_LEAF) small0.push_back(root);
        else leaves0.push_back((uint32_t)k);
    }
    NBG_LAUNCHED(T);
    if (level0.size() > kd->seg_cap || small0.size() > kd->seg_cap || leaves0.size() > kd->leaf_cap) {
        set_err(ctx, "KD replica: too many trees for the segment lists");
        return NBG_ERR_UNSUPPORTED;
    }
    // root nodes 0..T-1 (host arrays outlive the copies: the stream is synchronised below)
    cudaMemcpyAsync(kd->c1, c_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->c2, c_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->feat, f_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->nb, nb_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->ne, ne_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->ntree, tree_init.data(), T * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(kd->tfs, kd->tfh.data(), T * sizeof(Transform), cudaMemcpyHostToDevice, st);
    if (!level0.empty())
        cudaMemcpyAsync(kd->seg[0], level0.data(), level0.size() * sizeof(KdSeg), cudaMemcpyHostToDevice, st);
    if (!small0.empty())
        cudaMemcpyAsync(kd->small, small0.data(), small0.size() * sizeof(KdSeg), cudaMemcpyHostToDevice, st);
    if (!leaves0.empty())
        cudaMemcpyAsync(kd->leaves, leaves0.data(), leaves0.size() * 4, cudaMemcpyHostToDevice, st);
    uint32_t cnt[5] = {0, (uint32_t)T, 0, (uint32_t)small0.size(), (uint32_t)leaves0.size()};
    cudaMemcpyAsync(kd->counters, cnt, sizeof(cnt), cudaMemcpyHostToDevice, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_err(ctx, "KD replica init failed");
        return NBG_ERR_CUDA;
    }
    uint32_t node_count = (uint32_t)T;
    uint32_t S = (uint32_t)level0.size();
    int cur = 0;
    while (S > 0) {
        // room for this level's children
        if (node_count + 2 * S > kd->node_cap) {
            rc = kd_grow_nodes(ctx, kd, std::max<uint32_t>(kd->node_cap * 2, node_count + 2 * S + 64), st);
            if (rc) return rc;
        }
        const KdSeg* segs = kd->seg[cur];
        uint32_t ntiles = 0;
        kd_minmax_init_kernel<<<(S + 127) / 128, 128, 0, st>>>(kd->split, S);
        rc = kd_tiles(ctx, kd, segs, S, &ntiles, st);
        if (rc) return rc;
        if (ntiles)
            kd_minmax_kernel<<<kd_grid(kd, ntiles), KD_THREADS, 0, st>>>(segs, kd->nt, kd->tile_seg, kd->rx,
                                                                         kd->ry, kd->rz, kd->split, ntiles);
        kd_split_kernel<<<(S + 127) / 128, 128, 0, st>>>(segs, S, kd->split, kd->tfs, kd->bmin, kd->bmax);
        NBG_LAUNCHED(2 + (ntiles ? 1 : 0));
        // pass 1 runs on the same segments: their tile map is already built
        rc = kd_pass<1>(ctx, kd, segs, S, kd->split, st, ntiles);
        if (rc) return rc;
        // pass 2 only where points equal the cut value
        cudaMemsetAsync(kd->counters + 5, 0, 4, st);
        kd_pass2_plan_kernel<<<(S + 127) / 128, 128, 0, st>>>(segs, S, kd->split, kd->seg2,
                                                              kd->split2, kd->seg2_from,
                                                              kd->counters + 5);
        uint32_t S2 = 0;
        cudaMemcpyAsync(&S2, kd->counters + 5, 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            set_err(ctx, "KD replica pass-2 plan failed");
            return NBG_ERR_CUDA;
        }
        NBG_LAUNCHED(1);
        if (S2) {
            rc = kd_pass<2>(ctx, kd, kd->seg2, S2, kd->split2, st);
            if (rc) return rc;
            kd_pass2_done_kernel<<<(S2 + 127) / 128, 128, 0, st>>>(S2, kd->split2, kd->seg2_from,
                                                                   kd->split);
            NBG_LAUNCHED(1);
        }
        cudaMemsetAsync(kd->counters, 0, 4, st);
        NBG_LAUNCHED(2);
        kd_children_kernel<<<(S + 127) / 128, 128, 0, st>>>(segs, S, kd->split, kd->seg[cur ^ 1],
                                                            kd->counters, kd->c1, kd->c2, kd->feat,
                                                            kd->nb, kd->ne, kd->node_cap,
                                                            kd->seg_cap, kd->small, small_max,
                                                            kd->leaves, kd->leaf_cap, kd->ntree);
        cudaMemcpyAsync(cnt, kd->counters, sizeof(cnt), cudaMemcpyDeviceToHost, st);
        cudaError_t be = cudaGetLastError();
        if (be == cudaSuccess) be = cudaStreamSynchronize(st);
        if (be != cudaSuccess) {
            set_err(ctx, std::string("KD replica build failed: ") + cudaGetErrorString(be));
            return NBG_ERR_CUDA;
        }
        if (cnt[2]) {
            set_err(ctx, "KD replica build ran out of node or segment capacity");
            return NBG_ERR_UNSUPPORTED;
        }
        node_count = cnt[1];
        S = cnt[0];
        cur ^= 1;
    }
    // subtrees of the small segments, one warp each
    const uint32_t nsmall = cnt[3], nleaves = cnt[4];
    const uint64_t n = kd->n;
    if (nsmall) {
        rc = kd_grow_nodes(ctx, kd, std::max<uint32_t>(kd->node_cap, node_count + (uint32_t)(n / 8) + 1024), st);
        if (rc) return rc;
        const uint32_t wblocks = (nsmall + KD_WARPS - 1) / KD_WARPS;
        kd_warp_build_kernel<<<kd->wgrid_cap ? std::min(wblocks, kd->wgrid_cap) : wblocks, 32 * KD_WARPS, 0, st>>>(
            kd->small, nsmall, kd->rx, kd->ry, kd->rz, kd->rid, kd->mlpos, kd->mrpos, kd->c1, kd->c2,
            kd->feat, kd->nb, kd->ne, kd->bmin, kd->bmax, kd->counters, kd->node_cap, kd->tfs,
            kd->ntree);
        NBG_LAUNCHED(1);
    }
    if (nleaves)
        kd_leaf_bbox_kernel<<<(nleaves * 32 + 127) / 128, 128, 0, st>>>(
            kd->leaves, nleaves, kd->nb, kd->ne, kd->rx, kd->ry, kd->rz, kd->bmin, kd->bmax);
    cudaMemcpyAsync(cnt, kd->counters, sizeof(cnt), cudaMemcpyDeviceToHost, st);
    cudaError_t we = cudaGetLastError();
    if (we == cudaSuccess) we = cudaStreamSynchronize(st);
    if (we != cudaSuccess) {
        set_err(ctx, std::string("KD replica subtree build failed: ") + cudaGetErrorString(we));
        return NBG_ERR_CUDA;
    }
    if (cnt[2]) return KD_RETRY;
    node_count = cnt[1];
    kd->node_count = node_count;
    // divlow / divhigh from the children's extents
    const uint32_t nn = node_count;
    if (!kd->dlo || kd->dl_cap < nn) {
        if (kd->dlo) kd_release(ctx, kd, kd->dlo);
        if (kd->dhi) kd_release(ctx, kd, kd->dhi);
        kd->dlo = kd->dhi = nullptr;
        rc = kd_alloc(ctx, (void**)&kd->dlo, (size_t)nn * 8, kd);
        if (!rc) rc = kd_alloc(ctx, (void**)&kd->dhi, (size_t)nn * 8, kd);
        if (rc) return rc;
        kd->dl_cap = nn;
    }
    kd_div_kernel<<<(nn + 127) / 128, 128, 0, st>>>(nn, kd->c1, kd->c2, kd->feat, kd->bmin,
                                                    kd->bmax, kd->tfs, kd->ntree, kd->dlo, kd->dhi);
    if (!kd->kpos) {
        rc = kd_alloc(ctx, (void**)&kd->kpos, n * 4, kd);
        if (rc) return rc;
    }
    for (int k = 0; k < T; ++k)
        kd_inverse_kernel<<<grid_for(ctx, kd->npts[k]), 256, 0, st>>>(kd->rid, kd->base[k],
                                                                      kd->npts[k], kd->kpos);
    NBG_LAUNCHED(1 + T + (nleaves ? 1 : 0));
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_err(ctx, "KD replica extents failed");
        return NBG_ERR_CUDA;
    }
    return NBG_OK;
}

// Builds one forest holding the replicas of every listed tile that has none.
int kd_ensure_many(Context* ctx, Tile* const* tiles, int count, cudaStream_t st, bool beside_query) {
    NBG_RANGE("nbg kd replica build");
    std::vector<Tile*> todo;
    for (int i = 0; i < count; ++i)
        if (!(tiles[i]->kd && tiles[i]->kd->built) && tiles[i]->n > 0) todo.push_back(tiles[i]);
    if (todo.empty()) return NBG_OK;
    for (Tile* t : todo) kd_free(ctx, t);
    KdForest* kd = new KdForest();
    kd->ntrees = (int)todo.size();
    uint64_t n = 0;
    for (Tile* t : todo) {
        kd->base.push_back(n);
        kd->npts.push_back(t->n);
        kd->tfh.push_back(t->tf);
        n += t->n;
    }
    if (n >= (1ull << 32) - 1) {
        delete kd;
        set_err(ctx, "KD replica: more than 2^32 points in one forest");
        return NBG_ERR_UNSUPPORTED;
    }
    kd->n = n;
    if (beside_query && n >= kKdBesideMinPoints) {
        kd->grid_cap = (uint32_t)(kKdBesideBlocksPerSm * ctx->sm_count);
        kd->wgrid_cap = (uint32_t)(kKdBesideWarpBlocksPerSm * ctx->sm_count);
    }
    kd->rootbox.assign(6 * (size_t)kd->ntrees, 0.0);
    const int T = kd->ntrees;
    int rc = kd_alloc(ctx, (void**)&kd->rx, n * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->ry, n * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->rz, n * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->rid, n * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->mlpos, n * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->mrpos, n * 4, kd);
    kd->seg_cap = (uint32_t)(n / 50 + 64 + T);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->seg[0], kd->seg_cap * sizeof(KdSeg), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->seg[1], kd->seg_cap * sizeof(KdSeg), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->seg2, kd->seg_cap * sizeof(KdSeg), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->small, kd->seg_cap * sizeof(KdSeg), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->split, kd->seg_cap * sizeof(KdSplit), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->split2, kd->seg_cap * sizeof(KdSplit), kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->seg2_from, kd->seg_cap * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->nt, (kd->seg_cap + 1) * 4, kd);
    kd->leaf_cap = (uint32_t)(n / 16 + 1024 + T);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->leaves, (size_t)kd->leaf_cap * 4, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->counters, 64, kd);
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->tfs, (size_t)T * sizeof(Transform), kd);
    size_t b1 = 0, b2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b1, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int)(n / KD_TILE + kd->seg_cap + 2));
    cub::DeviceScan::ExclusiveSum(nullptr, b2, (unsigned long long*)nullptr,
                                  (unsigned long long*)nullptr, (int)(n / KD_TILE + kd->seg_cap + 2));
    b1 = std::max(b1, b2);
    kd->scan_bytes = b1;
    if (!rc) rc = kd_alloc(ctx, (void**)&kd->scan_tmp, b1, kd);
    if (!rc) rc = kd_grow_nodes(ctx, kd, (uint32_t)(n / 25 + 64 + 2 * (uint64_t)T), st);
    if (!rc) {
        rc = kd_build(ctx, kd, todo.data(), KD_WARP_MAX, st);
        if (rc == KD_RETRY) {
            // a warp subtree overflowed its stack or the node arrays: redo the
            // whole build with the level passes only
            rc = kd_grow_nodes(ctx, kd, (uint32_t)std::min<uint64_t>(2 * n + 64 + 2 * (uint64_t)T, UINT32_MAX), st);
            if (!rc) rc = kd_build(ctx, kd, todo.data(), 0, st);
            if (rc == KD_RETRY) {
                set_err(ctx, "KD replica build ran out of node capacity");
                rc = NBG_ERR_UNSUPPORTED;
            }
        }
    }
    if (rc) {
        kd_forest_free(ctx, kd);
        return rc;
    }
    for (int k = 0; k < T; ++k) {
        KdReplica* v = new KdReplica();
        v->f = kd;
        v->tree = k;
        v->built = true;
        todo[k]->kd = v;
    }
    kd->refs = T;
    return NBG_OK;
}

int kd_ensure(Context* ctx, Tile* t, cudaStream_t st, bool beside_query) {
    Tile* one[1] = {t};
    return kd_ensure_many(ctx, one, 1, st, beside_query);
}

bool kd_built(const Tile* t) { return t->kd && t->kd->built; }

KdOrder kd_order(const Tile* t) {
    const KdForest* kd = t->kd->f;
    KdOrder o;
    o.c1 = kd->c1;
    o.c2 = kd->c2;
    o.feat = kd->feat;
    o.ne = kd->ne;
    o.dlo = kd->dlo;
    o.dhi = kd->dhi;
    o.kpos = kd->kpos;
    o.root = t->kd->tree;
    o.base = kd->base[t->kd->tree];
    return o;
}

static KdDev kd_view(const Tile* t) {
    const KdForest* kd = t->kd->f;
    const int k = t->kd->tree;
    KdDev v;
    v.rx = kd->rx;
    v.ry = kd->ry;
    v.rz = kd->rz;
    v.rid = kd->rid;
    v.c1 = kd->c1;
    v.c2 = kd->c2;
    v.feat = kd->feat;
    v.nb = kd->nb;
    v.ne = kd->ne;
    v.dlo = kd->dlo;
    v.dhi = kd->dhi;
    v.root = k;
    for (int d = 0; d < 3; ++d) {
        v.root_lo[d] = kd->rootbox[6 * k + d];
        v.root_hi[d] = kd->rootbox[6 * k + 3 + d];
    }
    return v;
}

// Searches the listed rows into per-call scratch (nbr, counts).
static int kd_search_rows(Context* ctx, Tile* t, int K, const uint32_t* rows, uint32_t nrows,
                          uint32_t** nbr, uint32_t** counts, cudaStream_t st,
                          const double* row_k = nullptr) {
    if (K > KD_CAP) return NBG_ERR_INVALID;
    KdForest* kd = t->kd->f;
    *nbr = nullptr;
    *counts = nullptr;
    int arc = ctx_alloc(ctx, (void**)nbr, (size_t)nrows * K * 4);
    if (!arc) arc = ctx_alloc(ctx, (void**)counts, (size_t)nrows * 4);
    if (arc) {
        if (*nbr) ctx_free(ctx, *nbr, (size_t)nrows * K * 4);
        *nbr = nullptr;
        *counts = nullptr;
        return arc;
    }
    cudaMemsetAsync(kd->counters + 2, 0, 4, st);
    kd_search_kernel<<<(nrows + 3) / 4, 128, 0, st>>>(kd_view(t), t->tf, t->x, t->y, t->z,
                                                          rows, nrows, K, *nbr, *counts,
                                                          kd->counters + 2, row_k, t->n);
    NBG_LAUNCHED(1);
    cudaError_t le = cudaGetLastError();
    uint32_t err = 0;
    if (le == cudaSuccess) le = cudaMemcpyAsync(&err, kd->counters + 2, 4, cudaMemcpyDeviceToHost, st);
    if (le == cudaSuccess) le = cudaStreamSynchronize(st);
    if (le != cudaSuccess) {
        set_err(ctx, std::string("exact KD rows: ") + cudaGetErrorString(le));
        return NBG_ERR_CUDA;
    }
    if (err) {
        set_err(ctx, "KD search stack overflow");
        return NBG_ERR_UNSUPPORTED;
    }
    return NBG_OK;
}

int kd_run_rows(Context* ctx, Tile* t, int K, const StageGroup& grp, const ExceptionSink& ex,
                const uint32_t* rows, uint32_t nrows, cudaStream_t st, const double* row_k,
                int stride, int kpick) {
    NBG_RANGE("nbg search replay");
    if (!nrows) return NBG_OK;
    uint32_t *nbr = nullptr, *counts = nullptr;
    int rc = kd_search_rows(ctx, t, K, rows, nrows, &nbr, &counts, st, row_k);
    if (!rc) {
        kd_finish_kernel<<<(nrows + 127) / 128, 128, 0, st>>>(t->tf, t->x, t->y, t->z, rows, nrows,
                                                              K, nbr, counts, grp, ex, stride,
                                                              kpick);
        NBG_LAUNCHED(1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_err(ctx, std::string("exact KD finish: ") + cudaGetErrorString(e));
            rc = NBG_ERR_CUDA;
        }
    }
    if (nbr) ctx_free(ctx, nbr, (size_t)nrows * K * 4);
    if (counts) ctx_free(ctx, counts, (size_t)nrows * 4);
    return rc;
}

int kd_list_rows(Context* ctx, Tile* t, int K, const ListArgs& L, const ExceptionSink& ex,
                 const uint32_t* rows, uint32_t nrows, cudaStream_t st) {
    if (!nrows) return NBG_OK;
    uint32_t *nbr = nullptr, *counts = nullptr;
    int rc = kd_search_rows(ctx, t, K, rows, nrows, &nbr, &counts, st);
    if (!rc) {
        kd_list_finish_kernel<<<(nrows + 127) / 128, 128, 0, st>>>(t->tf, t->x, t->y, t->z, rows,
                                                                   nrows, K, nbr, counts, L, ex);
        NBG_LAUNCHED(1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_err(ctx, std::string("exact KD list: ") + cudaGetErrorString(e));
            rc = NBG_ERR_CUDA;
        }
    }
    if (nbr) ctx_free(ctx, nbr, (size_t)nrows * K * 4);
    if (counts) ctx_free(ctx, counts, (size_t)nrows * 4);
    return rc;
}

int kd_neighbor_rows(Context* ctx, Tile* t, int K, const uint32_t* rows, uint32_t nrows,
                     uint32_t* ids_out, cudaStream_t st) {
    if (!nrows) return NBG_OK;
    uint32_t *nbr = nullptr, *counts = nullptr;
    int rc = kd_search_rows(ctx, t, K, rows, nrows, &nbr, &counts, st);
    if (!rc) {
        kd_scatter_ids_kernel<<<(nrows + 127) / 128, 128, 0, st>>>(rows, nrows, K, nbr, counts,
                                                                   ids_out);
        NBG_LAUNCHED(1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_err(ctx, std::string("exact KD ids: ") + cudaGetErrorString(e));
            rc = NBG_ERR_CUDA;
        }
    }
    if (nbr) ctx_free(ctx, nbr, (size_t)nrows * K * 4);
    if (counts) ctx_free(ctx, counts, (size_t)nrows * 4);
    return rc;
}

// Test hook: copies the tile's replica out (point order as ids, and its
// tree's nodes renumbered in breadth-first order from its root, ranges
// relative to the tile).
int kd_export(Context* ctx, Tile* t, uint32_t* vind, uint32_t* nnodes, int32_t* c1, int32_t* c2,
              int32_t* feat, double* dlo, double* dhi, uint32_t* nb, uint32_t* ne, uint32_t cap,
              cudaStream_t st) {
    int rc = kd_ensure(ctx, t, st);
    if (rc) return rc;
    const KdForest* kd = t->kd->f;
    const int k = t->kd->tree;
    const uint64_t base = kd->base[k];
    const uint32_t nn = kd->node_count;
    std::vector<int32_t> hc1(nn), hc2(nn), hf(nn);
    std::vector<uint32_t> hnb(nn), hne(nn);
    std::vector<double> hlo(nn), hhi(nn);
    cudaMemcpyAsync(vind, kd->rid + base, t->n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hc1.data(), kd->c1, nn * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hc2.data(), kd->c2, nn * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hf.data(), kd->feat, nn * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hlo.data(), kd->dlo, nn * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hhi.data(), kd->dhi, nn * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hnb.data(), kd->nb, nn * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hne.data(), kd->ne, nn * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return NBG_ERR_CUDA;
    std::vector<int32_t> order{(int32_t)k};
    for (size_t q = 0; q < order.size(); ++q) {
        const int32_t v = order[q];
        if (hc1[v] >= 0) {
            order.push_back(hc1[v]);
            order.push_back(hc2[v]);
        }
    }
    std::vector<int32_t> newid(nn, -1);
    for (size_t q = 0; q < order.size(); ++q) newid[order[q]] = (int32_t)q;
    *nnodes = (uint32_t)order.size();
    const uint32_t m = std::min<uint32_t>(cap, (uint32_t)order.size());
    for (uint32_t q = 0; q < m; ++q) {
        const int32_t v = order[q];
        c1[q] = hc1[v] >= 0 ? newid[hc1[v]] : -1;
        c2[q] = hc2[v] >= 0 ? newid[hc2[v]] : -1;
        feat[q] = hf[v];
        dlo[q] = hlo[v];
        dhi[q] = hhi[v];
        nb[q] = (uint32_t)(hnb[v] - base);
        ne[q] = (uint32_t)(hne[v] - base);
    }
    return NBG_OK;
}

}  // namespace nbg

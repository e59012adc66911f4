// nbg_group.cu — group select: G neighbouring queries share one candidate list.
//
// Same answer as the per-thread select (knn_select_kernel, nbg_query.cu): for
// each row, the exact integer neighbourhood sums of its K nearest points (or
// their ids, for the neighbour-set export), or the row handed to the
// tie-order resolver / the exact KD path.  What changes
// is how a warp spends its lanes.  The per-thread ring search gives every
// lane its own rings of cells; neighbouring lanes scan overlapping but not
// equal cell sets, so a warp walks the union of its lanes' cells with most
// lanes masked (8.9 of 32 active on the 32M-point stress tile).  Here a
// subgroup of G lanes (G = 8, 16 or 32: the queries-per-group knob) answers G
// queries from ONE candidate list, and every lane does useful work on every
// candidate:
//
//   order     the block's rows are re-sorted by a Morton key of their
//             coordinates (block-local radix sort), so a subgroup's G
//             queries are spatially compact
//   box ring  the subgroup's bounding box of its queries grown by a margin
//             m_R; the points of the grid cells the box touches are filtered
//             by the lanes in parallel (inside box R, outside box R-1) and
//             staged in shared memory in chunks of G
//   scan      each lane forms the exact integer key of every staged
//             candidate against its own query and inserts keys below its
//             current (K+1)-th into its register top list.  A key packs the
//             squared distance above the candidate's index in the subgroup's
//             list (d2 << idx_bits | index), so the K nearest are known
//             without the per-thread path's second pass over the cells
//   complete  a lane is done when its K-th squared distance is below the
//             squared gap from its query to the outside of box R (faces on
//             the tile's boundary do not count)
//   margin    m_{R+1} = min(1.6 m_R, the largest current K-th distance of
//             the unfinished lanes + 1): the second term finishes, in one
//             more ring, every lane that already holds K candidates
//
// A subgroup whose box would span more than kMaxCols grid columns, whose list
// would pass kCap candidates, or whose margin would pass the key's exact range
// hands its unfinished rows to the per-thread select (a retry list read on the
// device, no host synchronisation).  Ties and far rows are decided exactly as
// the per-thread select decides them: keys compare exact integer squared
// distances, and candidates of equal distance differ only in their index.
#include <cub/block/block_radix_sort.cuh>

#include <climits>

#include "nbg_common.cuh"
#include "nbg_internal.h"
#include "nbg_query.cuh"

namespace nbg {

template <int G>
struct GroupShape {
    static constexpr int kThreads = G == 8 ? 128 : 256;
    static constexpr int kMinBlocks = G == 8 ? 6 : 3;  // resident blocks per SM the registers allow
    static constexpr int kGroups = kThreads / G;
    static constexpr int kIdxBits = G == 32 ? 10 : 9;
    static constexpr uint32_t kCap = 1u << kIdxBits;
    static constexpr uint32_t kD2Max = (1u << (32 - kIdxBits)) - 1u;  // largest exact packed d2
    static constexpr int kMaxCols = 48;
    static constexpr int kStage = 2 * G;
    static constexpr size_t kPosBytes = kCap * 4;
    static constexpr size_t kStageBytes = (size_t)kStage * 16;
    static constexpr size_t kColBytes = ((size_t)2 * (kMaxCols + 1) * 4 + 15) / 16 * 16;
    static constexpr size_t kGroupBytes = kPosBytes + kStageBytes + kColBytes;
    static constexpr size_t kSmem = (size_t)kGroups * kGroupBytes;
};

template <int G>
__device__ __forceinline__ int group_min(int v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <int G>
__device__ __forceinline__ int group_max(int v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Smallest ring R of the grid's cube rings around qc whose outside lies
// beyond squared distance d2 (what the tie-order resolver rescans).
__device__ __forceinline__ int ring_for(const GridParams& g, const QueryCell& qc, uint32_t d2) {
    int R = 0;
    while (R < 256 && outside_gap2(g, qc, R) <= (unsigned long long)d2) ++R;
    return R;
}

template <int KS, int G>
__global__ void __launch_bounds__(GroupShape<G>::kThreads, GroupShape<G>::kMinBlocks)
    knn_group_kernel(const QueryArgs a, const float margin0) {
    using S = GroupShape<G>;
    using Sort = cub::BlockRadixSort<uint32_t, S::kThreads, 1, uint32_t>;
    __shared__ typename Sort::TempStorage sort_tmp;
    __shared__ int s_box[6];
    extern __shared__ __align__(16) unsigned char smem[];

    const uint64_t nrows = a.rows ? a.nq : a.n;
    const uint64_t r0 = (uint64_t)blockIdx.x * S::kThreads;
    if (r0 >= nrows) return;  // whole block
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const uint32_t nvalid = (uint32_t)min((uint64_t)S::kThreads, nrows - r0);
    const GridParams g = *a.gp;

    // ---- block-local Morton order of the rows
    uint32_t pos;
    {
        uint32_t key[1], val[1];
        block_morton_order<S::kThreads>(a, r0, nvalid, s_box, key, val);
        Sort(sort_tmp).Sort(key, val, 0, 31);  // rows past the end sort last
        pos = val[0];
    }
    const bool valid = tid < (int)nvalid;

    // ---- the lane's query
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t id = 0;
    int K = 0;
    if (valid) {
        q = __ldg(&a.gv.sorted[pos]);
        id = __float_as_uint(q.w);
        K = row_neighbours(a.row_k, a.K, a.n, id);
    }
    const int qx = __float2int_rz(q.x), qy = __float2int_rz(q.y), qz = __float2int_rz(q.z);
    // rows without neighbours (OptimalKNN 0) go to the per-thread select
    bool retry = valid && K <= 0;
    bool done = !valid || K <= 0;
    const int off = done ? 0 : KS - (K + 1);
    TopK<KS> top;
    top.init(off);

    // ---- the subgroup
    const int sl = tid & (G - 1);
    const unsigned sgmask =
        G == 32 ? 0xffffffffu : (((1u << (G & 31)) - 1u) << (lane & ~(G - 1) & 31));
    unsigned char* gb = smem + (size_t)(tid / G) * S::kGroupBytes;
    uint32_t* cpos = (uint32_t*)gb;
    float4* stage = (float4*)(gb + S::kPosBytes);
    uint32_t* cbase = (uint32_t*)(gb + S::kPosBytes + S::kStageBytes);
    uint32_t* coff = cbase + (S::kMaxCols + 1);
    const int ex0 = g.maxx - g.minx, ex1 = g.maxy - g.miny, ex2 = g.maxz - g.minz;
    // bounding box of the subgroup's rows (fixed: the boxes below are nested)
    const int blo0 = group_min<G>(done ? INT_MAX : qx), bhi0 = group_max<G>(done ? INT_MIN : qx);
    const int blo1 = group_min<G>(done ? INT_MAX : qy), bhi1 = group_max<G>(done ? INT_MIN : qy);
    const int blo2 = group_min<G>(done ? INT_MAX : qz), bhi2 = group_max<G>(done ? INT_MIN : qz);
    bool live = (__ballot_sync(0xffffffffu, !done) & sgmask) != 0;  // subgroup-uniform
    int m = max(1, (int)((float)g.cell * margin0));
    int plo0 = 1, plo1 = 1, plo2 = 1, phi0 = 0, phi1 = 0, phi2 = 0;  // box R-1 (empty at R = 0)
    uint32_t ncand = 0, nst = 0;  // scanned / staged candidates (subgroup-uniform)
    const int c = g.cell;
    const int kMaxMargin = S::kIdxBits == 10 ? 2047 : 2895;

    // scans the first `np` staged candidates (np subgroup-uniform)
    auto scan_staged = [&](uint32_t np) {
        const uint32_t jw = __reduce_max_sync(0xffffffffu, np);
        for (uint32_t j = 0; j < jw; ++j) {
            const float4 p = stage[j];
            uint32_t kb = dist_key(p.x - q.x, p.y - q.y, p.z - q.z);
            kb = min(kb, KEY_BASE + S::kD2Max);
            const uint32_t key = ((kb - KEY_BASE) << S::kIdxBits) | (ncand + j);
            const bool want = j < np && !done && key < top.k[KS - 1];
            if (__any_sync(0xffffffffu, want)) {
                if (want) top.insert(key);
            }
        }
        ncand += np;
        const uint32_t rest = nst - np;
        float4 keep = make_float4(0.f, 0.f, 0.f, 0.f);
        if ((uint32_t)sl < rest) keep = stage[np + sl];
        __syncwarp();
        if ((uint32_t)sl < rest) stage[sl] = keep;
        __syncwarp();
        nst = rest;
    };

    while (__any_sync(0xffffffffu, live)) {
        const int lo0 = max(blo0 - m, 0), lo1 = max(blo1 - m, 0), lo2 = max(blo2 - m, 0);
        const int hi0 = min(bhi0 + m, ex0), hi1 = min(bhi1 + m, ex1), hi2 = min(bhi2 + m, ex2);
        const int cx0 = lo0 / c, cy0 = lo1 / c, cz0 = lo2 / c;
        const int ncx = hi0 / c - cx0 + 1, ncy = hi1 / c - cy0 + 1, cz1 = hi2 / c;
        int ncols = live ? ncx * ncy : 0;
        if (ncols > S::kMaxCols) {
            retry = retry || !done;
            live = false;
            ncols = 0;
        }
        // column table: the z-run of each touched column inside [cz0, cz1]
        const int ncols_w = __reduce_max_sync(0xffffffffu, ncols);
        uint32_t T = 0;
        for (int p0 = 0; p0 < ncols_w; p0 += G) {
            const int j = p0 + sl;
            uint32_t st = 0, len = 0;
            if (j < ncols) {
                const int cx = cx0 + j % ncx, cy = cy0 + j / ncx;
                const int4 ci = __ldg(&a.gv.colinfo[(uint32_t)cy * (uint32_t)g.gx + (uint32_t)cx]);
                const int zl = max(cz0, ci.y), zh = min(cz1, ci.z);
                if (zl <= zh) {
                    st = __ldg(&a.gv.cstart[(uint32_t)ci.x + (uint32_t)(zl - ci.y)]);
                    len = __ldg(&a.gv.cstart[(uint32_t)ci.x + (uint32_t)(zh - ci.y) + 1u]) - st;
                }
            }
            uint32_t inc = len;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o, G);
                if (sl >= o) inc += v;
            }
            if (j < ncols) {
                cbase[j] = st;
                coff[j] = T + inc - len;
            }
            T += __shfl_sync(0xffffffffu, inc, G - 1, G);
        }
        if (sl == 0) coff[ncols] = T;
        __syncwarp();
        // filter the touched columns' points into the candidate list
        const uint32_t Tw = __reduce_max_sync(0xffffffffu, T);
        int colp = 0;
        for (uint32_t t0 = 0; t0 < Tw; t0 += G) {
            const uint32_t t = t0 + sl;
            bool take = false;
            float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
            uint32_t pp = 0;
            if (t < T) {
                while (coff[colp + 1] <= t) ++colp;
                pp = cbase[colp] + (t - coff[colp]);
                p = __ldg(&a.gv.sorted[pp]);
                const int px = __float2int_rz(p.x), py = __float2int_rz(p.y), pz = __float2int_rz(p.z);
                const bool in_now = px >= lo0 && px <= hi0 && py >= lo1 && py <= hi1 && pz >= lo2 &&
                                    pz <= hi2;
                const bool in_prev = px >= plo0 && px <= phi0 && py >= plo1 && py <= phi1 &&
                                     pz >= plo2 && pz <= phi2;
                take = in_now && !in_prev;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, take) & sgmask;
            const uint32_t cnt = __popc(bal);
            if (live && ncand + nst + cnt > S::kCap) {  // the list would overflow
                retry = retry || !done;
                live = false;
            }
            if (take && live) {
                const uint32_t slot = nst + __popc(bal & ((1u << lane) - 1u));
                stage[slot] = p;
                cpos[ncand + slot] = pp;
            }
            if (live) nst += cnt;
            __syncwarp();
            if (__any_sync(0xffffffffu, nst >= (uint32_t)G)) scan_staged(nst >= (uint32_t)G ? G : 0);
        }
        scan_staged(nst);
        // completion of each lane against box R
        if (live && !done) {
            const uint32_t kth = top.at(off + K - 1);
            if (kth != 0xFFFFFFFFu) {
                const unsigned long long d2 = kth >> S::kIdxBits;
                unsigned long long gap = ~0ull;
                if (lo0 > 0) gap = min(gap, (unsigned long long)(qx - lo0 + 1));
                if (hi0 < ex0) gap = min(gap, (unsigned long long)(hi0 - qx + 1));
                if (lo1 > 0) gap = min(gap, (unsigned long long)(qy - lo1 + 1));
                if (hi1 < ex1) gap = min(gap, (unsigned long long)(hi1 - qy + 1));
                if (lo2 > 0) gap = min(gap, (unsigned long long)(qz - lo2 + 1));
                if (hi2 < ex2) gap = min(gap, (unsigned long long)(hi2 - qz + 1));
                if (gap == ~0ull || d2 < gap * gap) done = true;
            }
        }
        // next margin
        int need = 0;
        if (live && !done) {
            const uint32_t kth = top.at(off + K - 1);
            if (kth == 0xFFFFFFFFu) {
                need = INT_MAX;
            } else {
                const uint32_t d2 = kth >> S::kIdxBits;
                int s = (int)sqrtf((float)d2);
                while ((uint32_t)s * (uint32_t)s < d2) ++s;
                need = s + 1;
            }
        }
        need = group_max<G>(need);
        const bool all_done = (__ballot_sync(0xffffffffu, !done) & sgmask) == 0;
        const bool whole = lo0 == 0 && lo1 == 0 && lo2 == 0 && hi0 == ex0 && hi1 == ex1 && hi2 == ex2;
        if (live && (all_done || whole)) {
            // a lane still open once the box holds the whole tile has fewer
            // than K points to find: the per-thread path decides it
            if (!all_done) retry = retry || !done;
            live = false;
        }
        if (live) {
            const int grown = m + (m >> 1) + (m >> 3) + 1;
            const int mn = max(m + 1, min(grown, need));
            if (mn > kMaxMargin) {
                retry = retry || !done;
                live = false;
            } else {
                plo0 = lo0; plo1 = lo1; plo2 = lo2;
                phi0 = hi0; phi1 = hi1; phi2 = hi2;
                m = mn;
            }
        }
    }

    if (!valid) return;
    if (retry) {
        const uint32_t slot = atomicAdd(&a.counters[6], 1u);
        a.retry_rows[slot] = pos;
        return;
    }
    const uint32_t kk = top.at(off + K - 1) >> S::kIdxBits;
    const uint32_t kk1 = top.at(off + K) >> S::kIdxBits;
    if (kk >= S::kD2Max || kk >= (1u << 23)) {
        // beyond the exact key range: the exact KD path
        atomicAdd(&a.counters[2], 1u);
        defer_row(a, id, false, 0, 0);
        if (a.sums) {
            RowSums zs;
            zs.cnt = 0;
            a.sums[pos] = zs;
        }
        return;
    }
    if (kk == kk1) {
        atomicAdd(&a.counters[1], 1u);
        QueryCell qc;
        qc.qx = qx;
        qc.qy = qy;
        qc.qz = qz;
        qc.cx = qx / c;
        qc.cy = qy / c;
        qc.cz = qz / c;
        const int R = ring_for(g, qc, kk);
        defer_row(a, id, R < 256, KEY_BASE + kk, R);
        if (a.sums) {
            RowSums zs;
            zs.cnt = 0;
            a.sums[pos] = zs;
        }
        return;
    }
    if (a.ids_out) {
        uint32_t* row = a.ids_out + (uint64_t)id * a.K;
        int w = 0;
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            if (s >= off && s < off + K) {
                const float4 p = __ldg(&a.gv.sorted[cpos[top.k[s] & (S::kCap - 1u)]]);
                row[w++] = __float_as_uint(p.w);
            }
        }
        for (int s = 1; s < K; ++s) {  // ascending ids
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
    int s1x = 0, s1y = 0, s1z = 0, sxx = 0, syx = 0, syy = 0, szx = 0, szy = 0, szz = 0;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        if (s >= off && s < off + K) {
            const float4 p = __ldg(&a.gv.sorted[cpos[top.k[s] & (S::kCap - 1u)]]);
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
    a.sums[pos] = out;
}

template <int KS, int G>
static int launch_group_kg(const QueryArgs& q, float margin0, cudaStream_t stream) {
    using S = GroupShape<G>;
    const uint64_t rows = q.rows ? q.nq : q.n;
    const uint64_t blocks = (rows + S::kThreads - 1) / S::kThreads;
    if (!blocks) return NBG_OK;
    // the candidate lists and the sort's storage pass the 48 KB default
    if (cudaFuncSetAttribute(knn_group_kernel<KS, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)S::kSmem) ||
        cudaFuncSetAttribute(knn_group_kernel<KS, G>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100))
        return NBG_ERR_CUDA;
    knn_group_kernel<KS, G><<<(unsigned)blocks, S::kThreads, S::kSmem, stream>>>(q, margin0);
    NBG_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

template <int KS>
static int launch_group_k(const QueryArgs& q, int group, float margin0, cudaStream_t stream) {
    switch (group) {
        case 8: return launch_group_kg<KS, 8>(q, margin0, stream);
        case 16: return launch_group_kg<KS, 16>(q, margin0, stream);
        case 32: return launch_group_kg<KS, 32>(q, margin0, stream);
    }
    return NBG_ERR_INVALID;
}

// The group select for K neighbours (slots: the top list's size, K + 1 or
// more).  Rows it hands back land in q.retry_rows, counted in q.counters[6].
int launch_group_select(const QueryArgs& q, int slots, int group, float margin0,
                        cudaStream_t stream) {
    switch (slots) {
        case 10: return launch_group_k<10>(q, group, margin0, stream);
        case 12: return launch_group_k<12>(q, group, margin0, stream);
        case 14: return launch_group_k<14>(q, group, margin0, stream);
        case 18: return launch_group_k<18>(q, group, margin0, stream);
        case 26: return launch_group_k<26>(q, group, margin0, stream);
        case 34: return launch_group_k<34>(q, group, margin0, stream);
        case 50: return launch_group_k<50>(q, group, margin0, stream);
        case 66: return launch_group_k<66>(q, group, margin0, stream);
    }
    return NBG_ERR_INVALID;
}

}  // namespace nbg

// nbg_consumers.cuh — per-row epilogues of the kNN consumers that read the
// neighbour LIST in the reference's order (filters.nndistance,
// filters.optimalneighborhood, filters.lof, filters.outlier statistical).
//
// The list is what KD3Index::knnSearch returns (KDImpl.hpp:383-396): the
// kref nearest points ordered by squared FP64 distance as the reference forms
// it, points at equal distance in the order its search meets them; a list
// longer than the cloud keeps its caller-initialised tail, point 0 at squared
// distance 0.  The grid path (ordered list kernel) and the search replay both
// end here with the same (ids, offsets, distances), so a row's result does
// not depend on which of them answered it.
#pragma once

#include "nbg_common.cuh"

namespace nbg {

struct ListArgs {
    int32_t kind;        // NBG_STAGE_NNDISTANCE / OPTIMALNEIGHBORHOOD / LOF / OUTLIER
    int32_t kref;        // the reference's list length (may exceed the cloud)
    int32_t mode;        // nndistance: 0 kth, 1 avg
    int32_t kmin;        // optimalneighborhood: min_k
    int32_t stage;       // index of the stage in the caller's array
    int32_t pad;
    StageDev st;         // output columns
    int32_t raw0[3];     // point 0's raw coordinates (the padding entries)
    double* rowval;      // outlier: mean neighbour distance; lof: k-distance (n)
    uint32_t* list_ids;  // lof: ordered ids, n x kref
    double* list_d;      // lof: neighbour distances (not squared), n x kref
};

// Squared FP64 distance as the reference's adaptor forms it
// (KDImpl.hpp:262-270): (q - p) per axis, ((dx*dx + dy*dy) + dz*dz).
__device__ __forceinline__ double ref_dist2(const double q64[3], const int32_t qraw[3],
                                            const int o[3], const Transform& tf) {
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double pc = ref_coord(qraw[d] + o[d], tf.scale[d], tf.offset[d]);
        const double df = __dsub_rn(q64[d], pc);
        acc = __dadd_rn(acc, __dmul_rn(df, df));
    }
    return acc;
}

// One row: `cnt` entries (ids[j], raw offsets off[j] from the query, squared
// distances d[j]) in the reference's order; entries cnt..kref-1 are padding.
__device__ inline void list_consume(const ListArgs& L, const Transform& tf, const ExceptionSink& ex,
                                    uint32_t rid, const int32_t qraw[3], int cnt,
                                    const uint32_t* ids, const int (*off)[3], const double* d) {
    const int kref = L.kref;
    auto dist2 = [&](int j) -> double { return j < cnt ? d[j] : 0.0; };
    if (L.kind == NBG_STAGE_NNDISTANCE) {
        // NNDistanceFilter.cpp:116-137
        double val;
        if (L.mode == 0) {
            val = __dsqrt_rn(dist2(kref - 1));
        } else {
            val = 0.0;
            for (int j = 1; j < kref; ++j) val = __dadd_rn(val, __dsqrt_rn(dist2(j)));
            val = __ddiv_rn(val, (double)(kref - 1));
        }
        nbg_store(L.st, rid, 0, val);
        return;
    }
    if (L.kind == NBG_STAGE_OUTLIER) {
        // OutlierFilter.cpp:139-152: running mean of the neighbour distances
        double m = 0.0;
        for (int j = 1; j < kref; ++j) {
            const double delta = __dsub_rn(__dsqrt_rn(dist2(j)), m);
            m = __dadd_rn(m, __ddiv_rn(delta, (double)j));
        }
        L.rowval[rid] = m;
        return;
    }
    if (L.kind == NBG_STAGE_LOF) {
        // LOFFilter.cpp:85-96: the list and the k-distance
        uint32_t* li = L.list_ids + (uint64_t)rid * kref;
        double* ld = L.list_d + (uint64_t)rid * kref;
        for (int j = 0; j < kref; ++j) {
            li[j] = j < cnt ? ids[j] : 0u;
            ld[j] = __dsqrt_rn(dist2(j));
        }
        const double kd = __dsqrt_rn(dist2(kref - 1));
        L.rowval[rid] = kd;
        nbg_store(L.st, rid, 0, kd);
        return;
    }
    // NBG_STAGE_OPTIMALNEIGHBORHOOD (OptimalNeighborhoodFilter.cpp:79-162):
    // running covariance over the list, the eigenentropy of each k in
    // [min_k, max_k], the first k of least entropy
    double mx = 0.0, my = 0.0, mz = 0.0;
    double b00 = 0.0, b11 = 0.0, b22 = 0.0, b10 = 0.0, b20 = 0.0, b21 = 0.0;
    double best = 1.7976931348623157e308;
    int kopt = 0;
    double r2 = 0.0;
    for (int j = 0; j < kref; ++j) {
        int32_t raw[3];
        if (j < cnt) {
            raw[0] = qraw[0] + off[j][0];
            raw[1] = qraw[1] + off[j][1];
            raw[2] = qraw[2] + off[j][2];
        } else {
            raw[0] = L.raw0[0];
            raw[1] = L.raw0[1];
            raw[2] = L.raw0[2];
        }
        const double dx = __dsub_rn(ref_coord(raw[0], tf.scale[0], tf.offset[0]), mx);
        const double dy = __dsub_rn(ref_coord(raw[1], tf.scale[1], tf.offset[1]), my);
        const double dz = __dsub_rn(ref_coord(raw[2], tf.scale[2], tf.offset[2]), mz);
        const double nn = (double)(j + 1);
        mx = __dadd_rn(mx, __ddiv_rn(dx, nn));
        my = __dadd_rn(my, __ddiv_rn(dy, nn));
        mz = __dadd_rn(mz, __ddiv_rn(dz, nn));
        const double s = __ddiv_rn(__dsub_rn(nn, 1.0), nn);
        const double sdx = __dmul_rn(s, dx), sdy = __dmul_rn(s, dy);
        b00 = __dadd_rn(b00, __dmul_rn(sdx, dx));
        b11 = __dadd_rn(b11, __dmul_rn(sdy, dy));
        b22 = __dadd_rn(b22, __dmul_rn(__dmul_rn(s, dz), dz));
        b10 = __dadd_rn(b10, __dmul_rn(sdx, dy));
        b20 = __dadd_rn(b20, __dmul_rn(sdx, dz));
        b21 = __dadd_rn(b21, __dmul_rn(sdy, dz));
        if (j + 1 < L.kmin) continue;
        // B / (n - 1): with n = 1 every entry is 0/0 and the solver fails
        const double dn = __dsub_rn(nn, 1.0);
        int ok = 0;
        double ev[3], V[9];
        if (j > 0) {
            const double C[6] = {__ddiv_rn(b00, dn), __ddiv_rn(b10, dn), __ddiv_rn(b11, dn),
                                 __ddiv_rn(b20, dn), __ddiv_rn(b21, dn), __ddiv_rn(b22, dn)};
            ok = nbg_eigen_chain(C, ev, V);
        }
        if (!ok) {
            nbg_append_exception(ex, rid, L.stage, NBG_ROW_EIGEN_FAIL);
            return;
        }
        double l2 = fmax(ev[2], 0.0), l1 = fmax(ev[1], 0.0), l0 = fmax(ev[0], 0.0);
        const double sum = __dadd_rn(__dadd_rn(l2, l1), l0);
        l2 = __ddiv_rn(l2, sum);
        l1 = __ddiv_rn(l1, sum);
        l0 = __ddiv_rn(l0, sum);
        const double ent = -__dadd_rn(__dadd_rn(__dmul_rn(l0, log(l0)), __dmul_rn(l1, log(l1))),
                                      __dmul_rn(l2, log(l2)));
        if (ent < best) {
            best = ent;
            kopt = j + 1;
            r2 = dist2(j);
        }
    }
    nbg_store(L.st, rid, 0, (double)kopt);
    nbg_store(L.st, rid, 1, __dsqrt_rn(r2));
}

}  // namespace nbg

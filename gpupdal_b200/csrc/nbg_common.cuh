// nbg_common.cuh — shared device definitions of the B200 neighbourhood path.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "../../include/nbg_b200.h"

#define NBG_MAX_STAGES 4
#define NBG_MAX_RING 24

// Grid of one tile, written on the device by grid_config_kernel so that the
// build never waits on the host for its shape.  Coordinates are raw int32
// relative to the tile minimum; cells are cubes of `cell` raw units.  Each
// (cx, cy) column stores a dense run of cells over its own occupied z-range:
// colinfo[col] = {base, zmin, zmax, 0}, cell (cx, cy, cz) is table entry
// base + cz - zmin, and cstart[entry] is the cell's first point.
struct GridParams {
    int32_t minx, miny, minz;
    int32_t maxx, maxy, maxz;
    int32_t cell;
    int32_t gx, gy, gz;
    uint32_t ncols;    // gx*gy
    uint32_t cap_hit;  // cell size had to grow to fit the column directory
};

// Device pointers of a tile's grid.
struct GridView {
    const float4* sorted;   // points in cell order {x, y, z, id bits}
    const int4* colinfo;    // per column {base, zmin, zmax, 0}
    const uint32_t* cstart; // first point of each table entry (T + 1 entries)
};

// One stage of a fused group, resolved for the device.
struct StageDev {
    int32_t kind;
    int32_t always_up;
    int32_t has_viewpoint;
    int32_t normalize;
    double viewpoint[3];
    uint32_t feature_mask;
    int32_t mode;
    int32_t ndims;
    int32_t ip;       // optimalneighborhood min_k; outlier (radius) min_k
    char* base;
    int64_t point_stride;
    int64_t offset[NBG_MAX_DIMS];
    double t1, t2;    // approximatecoplanar thresh1/2; estimaterank thresh
    double* aux;      // outlier (radius): per-row flag, 1 = outlier (device, n)
};

struct StageGroup {
    int32_t nstages;
    int32_t sign_exact;  // a stage exposes the eigenvector sign, or asks for the plain
                         // FP64 eigensolve: every row through the Eigen chain
    int32_t stage_index[NBG_MAX_STAGES];  // index in the caller's array
    StageDev st[NBG_MAX_STAGES];
    const double* optimal_knn;     // device, may be null
    const double* optimal_radius;  // device, may be null
    uint32_t* resolve_count;       // rows the fast eigensolver handed to the chain (may be null)
    int32_t no_eigen;              // every stage reads the neighbour count only
};

// The KD replica's nodes as the tie-order resolver reads them: a child's
// points are the contiguous range [nb, ne) of the replica's point order, and
// kpos[base + id] is the position of point id in that order.
struct KdOrder {
    const int32_t* c1;
    const int32_t* c2;
    const int32_t* feat;
    const uint32_t* ne;
    const double* dlo;
    const double* dhi;
    const uint32_t* kpos;  // indexed base + point id
    int32_t root;          // the tile's root node
    uint64_t base;         // the tile's first position
};

// Exact integer neighbourhood sums of one row (offsets from the query, raw
// units): s = {S1x, S1y, S1z, Sxx, Syx, Syy, Szx, Szy, Szz}; cnt = 0 marks a
// row the grid path did not finish.
struct RowSums {
    int32_t s[9];
    int32_t cnt;
};

// Per-row exception sink.
struct ExceptionSink {
    nbg_row_exception* rows;
    uint32_t* count;
    uint32_t capacity;
};

// Tile scale/offset as seen by the reference: value = raw*scale + offset.
struct Transform {
    double scale[3];
    double offset[3];
};

// Arguments of the query kernels for one tile and one stage group.
struct QueryArgs {
    GridView gv;
    const GridParams* gp;
    uint64_t n;
    int K;
    int rmax;
    StageGroup grp;
    Transform tf;
    ExceptionSink ex;
    uint32_t* exact_rows;
    uint32_t* counters;  // [0] exact rows, [1] tie rows, [2] incomplete rows, [4] tie list
    uint32_t* ids_out;   // neighbour-set export (null in the fused path)
    uint2* ties;         // tie list {id, (D_K - 2^23 bias) | R << 24}; null: ties go to exact_rows
    uint32_t tie_cap;
    RowSums* sums;       // split form: per sorted position, read by knn_finish_kernel
    const double* row_k; // covariancefeatures optimized: per-point k = OptimalKNN (null: K)
    const uint32_t* rows = nullptr;  // split form: the sorted positions to answer (null: all n)
    uint64_t nq = 0;                 // entries of `rows`
    const uint32_t* nq_dev = nullptr;  // entries of `rows` read on the device (retry launches)
    uint32_t* retry_rows = nullptr;    // group select: rows it hands to the per-thread select
};

// Neighbour count of a row: K, or the point's OptimalKNN rounded half away
// from zero (Utils::numericCast, pdal/util/Utils.hpp:747-764) capped at the
// tile's size, as KD3Index::neighbors(p, k, 1) in
// CovarianceFeaturesFilter.cpp:212-214.
__device__ __forceinline__ int row_neighbours(const double* row_k, int K, uint64_t n, uint32_t id) {
    if (!row_k) return K;
    const double v = row_k[id];
    const double k = v > 0.0 ? floor(v + 0.5) : ceil(v - 0.5);
    return (int)(k < (double)n ? k : (double)n);
}

// One tile of a batch: its query arguments and the first work item (block of
// queries) it owns in the batch's queue.
struct BatchJob {
    QueryArgs q;
    uint64_t first;
};

// ---------------------------------------------------------------------------
// The reference's coordinate, fl(fl(raw*scale) + offset), with no contraction.
__device__ __forceinline__ double ref_coord(int32_t raw, double s, double o) {
    return __dadd_rn(__dmul_rn((double)raw, s), o);
}

// ---------------------------------------------------------------------------
// Eigen 3.4 SelfAdjointEigenSolver<Matrix3d> chain on the device (3x3
// Householder tridiagonalisation, implicit symmetric QR with Wilkinson shift,
// continuous Givens rotations, selection sort).  Keeping the same chain keeps
// the same eigenvector signs as the reference, which filters.normal exposes
// when always_up is false and no viewpoint is given.  evec column-major.
__device__ __forceinline__ void nbg_make_givens(double p, double q, double& c, double& s) {
    if (q == 0.0) {
        c = p < 0.0 ? -1.0 : 1.0;
        s = 0.0;
    } else if (p == 0.0) {
        c = 0.0;
        s = q < 0.0 ? 1.0 : -1.0;
    } else if (fabs(p) > fabs(q)) {
        double t = __ddiv_rn(q, p);
        double u = __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t)));
        if (p < 0.0) u = -u;
        c = __ddiv_rn(1.0, u);
        s = __dmul_rn(-t, c);
    } else {
        double t = __ddiv_rn(p, q);
        double u = __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t)));
        if (q < 0.0) u = -u;
        s = __ddiv_rn(-1.0, u);
        c = __dmul_rn(-t, s);
    }
}

__device__ __forceinline__ double nbg_pos_hypot(double x, double y) {
    double p = fmax(x, y);
    if (p == 0.0) return 0.0;
    double qp = __ddiv_rn(fmin(y, x), p);
    return __dmul_rn(p, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(qp, qp))));
}

// a: symmetric 3x3 (a00,a10,a11,a20,a21,a22 lower triangle).  Returns 1 on
// success.  eval ascending; evec[c*3+r].
__device__ inline int nbg_eigen_chain(const double low[6], double eval[3], double evec[9]) {
    double m00 = low[0], m10 = low[1], m11 = low[2], m20 = low[3], m21 = low[4], m22 = low[5];
    double scale = fmax(fmax(fmax(fabs(m00), fabs(m10)), fmax(fabs(m11), fabs(m20))),
                        fmax(fabs(m21), fabs(m22)));
    if (scale == 0.0) scale = 1.0;
    m00 = __ddiv_rn(m00, scale);
    m10 = __ddiv_rn(m10, scale);
    m11 = __ddiv_rn(m11, scale);
    m20 = __ddiv_rn(m20, scale);
    m21 = __ddiv_rn(m21, scale);
    m22 = __ddiv_rn(m22, scale);
    double diag[3], sub[2];
    double Q[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    diag[0] = m00;
    double v1norm2 = __dmul_rn(m20, m20);
    if (v1norm2 <= DBL_MIN) {
        diag[1] = m11;
        diag[2] = m22;
        sub[0] = m10;
        sub[1] = m21;
    } else {
        double beta = __dsqrt_rn(__dadd_rn(__dmul_rn(m10, m10), v1norm2));
        double invBeta = __ddiv_rn(1.0, beta);
        double m01 = __dmul_rn(m10, invBeta);
        double m02 = __dmul_rn(m20, invBeta);
        double q = __dadd_rn(__dmul_rn(__dmul_rn(2.0, m01), m21),
                             __dmul_rn(m02, __dsub_rn(m22, m11)));
        diag[1] = __dadd_rn(m11, __dmul_rn(m02, q));
        diag[2] = __dsub_rn(m22, __dmul_rn(m02, q));
        sub[0] = beta;
        sub[1] = __dsub_rn(m21, __dmul_rn(m01, q));
        Q[4] = m01;
        Q[5] = m02;
        Q[7] = m02;
        Q[8] = -m01;
    }
    int end = 2, start = 0, iter = 0;
    const double precision_inv = 1.0 / DBL_EPSILON;
    while (end > 0) {
        for (int i = start; i < end; ++i) {
            if (fabs(sub[i]) < DBL_MIN) sub[i] = 0.0;
            else {
                double sc = __dmul_rn(precision_inv, sub[i]);
                if (__dmul_rn(sc, sc) <= __dadd_rn(fabs(diag[i]), fabs(diag[i + 1]))) sub[i] = 0.0;
            }
        }
        while (end > 0 && sub[end - 1] == 0.0) end--;
        if (end <= 0) break;
        iter++;
        if (iter > 90) break;
        start = end - 1;
        while (start > 0 && sub[start - 1] != 0.0) start--;
        double td = __dmul_rn(__dsub_rn(diag[end - 1], diag[end]), 0.5);
        double e = sub[end - 1];
        double mu = diag[end];
        if (td == 0.0) {
            mu = __dsub_rn(mu, fabs(e));
        } else if (e != 0.0) {
            double e2 = __dmul_rn(e, e);
            double h = nbg_pos_hypot(fabs(td), fabs(e));
            double den = __dadd_rn(td, td > 0.0 ? h : -h);
            if (e2 == 0.0) mu = __dsub_rn(mu, __ddiv_rn(e, __ddiv_rn(den, e)));
            else mu = __dsub_rn(mu, __ddiv_rn(e2, den));
        }
        double x = __dsub_rn(diag[start], mu);
        double z = sub[start];
        for (int k = start; k < end && z != 0.0; ++k) {
            double c, s;
            nbg_make_givens(x, z, c, s);
            double sdk = __dadd_rn(__dmul_rn(s, diag[k]), __dmul_rn(c, sub[k]));
            double dkp1 = __dadd_rn(__dmul_rn(s, sub[k]), __dmul_rn(c, diag[k + 1]));
            double t1 = __dsub_rn(__dmul_rn(c, diag[k]), __dmul_rn(s, sub[k]));
            double t2 = __dsub_rn(__dmul_rn(c, sub[k]), __dmul_rn(s, diag[k + 1]));
            diag[k] = __dsub_rn(__dmul_rn(c, t1), __dmul_rn(s, t2));
            diag[k + 1] = __dadd_rn(__dmul_rn(s, sdk), __dmul_rn(c, dkp1));
            sub[k] = __dsub_rn(__dmul_rn(c, sdk), __dmul_rn(s, dkp1));
            if (k > start) sub[k - 1] = __dsub_rn(__dmul_rn(c, sub[k - 1]), __dmul_rn(s, z));
            x = sub[k];
            if (k < end - 1) {
                z = __dmul_rn(-s, sub[k + 1]);
                sub[k + 1] = __dmul_rn(c, sub[k + 1]);
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                double xi = Q[k * 3 + r], yi = Q[(k + 1) * 3 + r];
                Q[k * 3 + r] = __dsub_rn(__dmul_rn(c, xi), __dmul_rn(s, yi));
                Q[(k + 1) * 3 + r] = __dadd_rn(__dmul_rn(s, xi), __dmul_rn(c, yi));
            }
        }
    }
    int ok = iter <= 90;
    if (ok) {
        for (int i = 0; i < 2; ++i) {
            int k = i;
            for (int j = i + 1; j < 3; ++j)
                if (diag[j] < diag[k]) k = j;
            if (k != i) {
                double t = diag[i];
                diag[i] = diag[k];
                diag[k] = t;
                for (int r = 0; r < 3; ++r) {
                    double u = Q[i * 3 + r];
                    Q[i * 3 + r] = Q[k * 3 + r];
                    Q[k * 3 + r] = u;
                }
            }
        }
    }
    eval[0] = __dmul_rn(diag[0], scale);
    eval[1] = __dmul_rn(diag[1], scale);
    eval[2] = __dmul_rn(diag[2], scale);
#pragma unroll
    for (int i = 0; i < 9; ++i) evec[i] = Q[i];
    return ok;
}

// ---------------------------------------------------------------------------
// Fast symmetric 3x3 eigensolve: four fixed cyclic Jacobi sweeps in FP32 on
// the covariance scaled to [-1, 1], then one Jacobi sweep in FP64 on V^T C V
// (nearly diagonal, so its rotations are small-angle: t = a_pq/(a_qq - a_pp))
// and FP64 eigenvalues from the polished diagonal.  Uniform control flow, no
// data-dependent iteration count.  Returns 0 when a polish rotation is not
// small (|t| > 1e-3: eigenvalues too close for the FP32 basis to be a good
// start); the caller then re-solves with the FP64 Eigen chain.
__device__ __forceinline__ void nbg_jrot32(float& app, float& aqq, float& apq, float& arp,
                                           float& arq, float* vp, float* vq) {
    if (apq == 0.0f) return;
    const float theta = 0.5f * (aqq - app) / apq;
    const float t = copysignf(1.0f, theta) / (fabsf(theta) + sqrtf(fmaf(theta, theta, 1.0f)));
    const float c = rsqrtf(fmaf(t, t, 1.0f));
    const float s = t * c;
    app = fmaf(-t, apq, app);
    aqq = fmaf(t, apq, aqq);
    apq = 0.0f;
    const float rp = arp, rq = arq;
    arp = c * rp - s * rq;
    arq = s * rp + c * rq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float a = vp[k], b = vq[k];
        vp[k] = c * a - s * b;
        vq[k] = s * a + c * b;
    }
}

__device__ __forceinline__ bool nbg_jrot64(double& app, double& aqq, double& apq, double& arp,
                                           double& arq, double* vp, double* vq) {
    if (apq == 0.0) return true;
    const double den = aqq - app;
    const double t = apq / den;  // tan of the rotation, first order
    if (!(fabs(t) <= 1e-3)) return false;
    const double c = 1.0 - 0.5 * t * t;
    const double s = t * c;
    app = app - t * apq;
    aqq = aqq + t * apq;
    apq = 0.0;
    const double rp = arp, rq = arq;
    arp = c * rp - s * rq;
    arq = s * rp + c * rq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double a = vp[k], b = vq[k];
        vp[k] = c * a - s * b;
        vq[k] = s * a + c * b;
    }
    return true;
}

// low = {c00, c10, c11, c20, c21, c22}; eval ascending; evec column-major.
__device__ inline bool nbg_eigen_fast(const double low[6], double eval[3], double evec[9]) {
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) m = fmax(m, fabs(low[i]));
    if (m == 0.0) m = 1.0;
    const double inv = 1.0 / m;
    float a00 = (float)(low[0] * inv), a10 = (float)(low[1] * inv), a11 = (float)(low[2] * inv);
    float a20 = (float)(low[3] * inv), a21 = (float)(low[4] * inv), a22 = (float)(low[5] * inv);
    float v0[3] = {1, 0, 0}, v1[3] = {0, 1, 0}, v2[3] = {0, 0, 1};
#pragma unroll
    for (int sweep = 0; sweep < 4; ++sweep) {
        nbg_jrot32(a00, a11, a10, a20, a21, v0, v1);  // (0,1), r = 2
        nbg_jrot32(a00, a22, a20, a10, a21, v0, v2);  // (0,2), r = 1 (a_10 is a_r0, a_21 a_r2)
        nbg_jrot32(a11, a22, a21, a10, a20, v1, v2);  // (1,2), r = 0
    }
    // FP64 polish on B = V^T C V (C scaled by 1/m).  The FP32 basis is first
    // made orthonormal in FP64 (Gram-Schmidt, third vector by cross product
    // with the orientation of the FP32 one), so that B is similar to C.
    double V[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        V[0][k] = v0[k];
        V[1][k] = v1[k];
        V[2][k] = v2[k];
    }
    {
        double r0 = rsqrt(V[0][0] * V[0][0] + V[0][1] * V[0][1] + V[0][2] * V[0][2]);
        for (int k = 0; k < 3; ++k) V[0][k] *= r0;
        const double p01 = V[0][0] * V[1][0] + V[0][1] * V[1][1] + V[0][2] * V[1][2];
        for (int k = 0; k < 3; ++k) V[1][k] -= p01 * V[0][k];
        double r1 = rsqrt(V[1][0] * V[1][0] + V[1][1] * V[1][1] + V[1][2] * V[1][2]);
        for (int k = 0; k < 3; ++k) V[1][k] *= r1;
        const double cx = V[0][1] * V[1][2] - V[0][2] * V[1][1];
        const double cy = V[0][2] * V[1][0] - V[0][0] * V[1][2];
        const double cz = V[0][0] * V[1][1] - V[0][1] * V[1][0];
        const double sg = (cx * V[2][0] + cy * V[2][1] + cz * V[2][2]) < 0 ? -1.0 : 1.0;
        V[2][0] = sg * cx;
        V[2][1] = sg * cy;
        V[2][2] = sg * cz;
    }
    const double C00 = low[0] * inv, C10 = low[1] * inv, C11 = low[2] * inv;
    const double C20 = low[3] * inv, C21 = low[4] * inv, C22 = low[5] * inv;
    double W[3][3];  // W[i] = C * V[i]
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        W[i][0] = C00 * V[i][0] + C10 * V[i][1] + C20 * V[i][2];
        W[i][1] = C10 * V[i][0] + C11 * V[i][1] + C21 * V[i][2];
        W[i][2] = C20 * V[i][0] + C21 * V[i][1] + C22 * V[i][2];
    }
    double b00 = V[0][0] * W[0][0] + V[0][1] * W[0][1] + V[0][2] * W[0][2];
    double b11 = V[1][0] * W[1][0] + V[1][1] * W[1][1] + V[1][2] * W[1][2];
    double b22 = V[2][0] * W[2][0] + V[2][1] * W[2][1] + V[2][2] * W[2][2];
    double b10 = V[1][0] * W[0][0] + V[1][1] * W[0][1] + V[1][2] * W[0][2];
    double b20 = V[2][0] * W[0][0] + V[2][1] * W[0][1] + V[2][2] * W[0][2];
    double b21 = V[2][0] * W[1][0] + V[2][1] * W[1][1] + V[2][2] * W[1][2];
    bool ok = nbg_jrot64(b00, b11, b10, b20, b21, V[0], V[1]);
    ok = ok && nbg_jrot64(b00, b22, b20, b10, b21, V[0], V[2]);
    ok = ok && nbg_jrot64(b11, b22, b21, b10, b20, V[1], V[2]);
    if (!ok) return false;
    // normalise the polished vectors and sort ascending
    double ev[3] = {b00 * m, b11 * m, b22 * m};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double r = rsqrt(V[i][0] * V[i][0] + V[i][1] * V[i][1] + V[i][2] * V[i][2]);
        V[i][0] *= r;
        V[i][1] *= r;
        V[i][2] *= r;
    }
    int o0 = 0, o1 = 1, o2 = 2;
    if (ev[o1] < ev[o0]) { int t = o0; o0 = o1; o1 = t; }
    if (ev[o2] < ev[o1]) { int t = o1; o1 = o2; o2 = t; }
    if (ev[o1] < ev[o0]) { int t = o0; o0 = o1; o1 = t; }
    const int ord[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        eval[c] = ev[ord[c]];
        evec[c * 3 + 0] = V[ord[c]][0];
        evec[c * 3 + 1] = V[ord[c]][1];
        evec[c * 3 + 2] = V[ord[c]][2];
    }
    return true;
}

// ---------------------------------------------------------------------------
// Row epilogue shared by the grid path and the exact KD path.
//
// M = n*S2 - S1*S1^T over the neighbours' raw offsets from the query (exact
// int64), so cov = M * s_i*s_j / (n*(n-1)).  Writes every stage's outputs,
// or appends the reference's skip/throw code to the exception sink.
__device__ inline void nbg_append_exception(const ExceptionSink& ex, uint32_t id, int stage,
                                            int code, uint16_t reserved = 0) {
    uint32_t slot = atomicAdd(ex.count, 1u);
    if (slot < ex.capacity) {
        nbg_row_exception r;
        r.point_id = id;
        r.stage = (uint8_t)stage;
        r.code = (uint8_t)code;
        r.reserved = reserved;
        ex.rows[slot] = r;
    }
}

__device__ __forceinline__ void nbg_store(const StageDev& st, uint32_t id, int d, double v) {
    *reinterpret_cast<double*>(st.base + (int64_t)id * st.point_stride + st.offset[d]) = v;
}

// Md = n*S2 - S1*S1^T of the neighbours' raw offsets (exact integers, as
// doubles), lower triangle m00, m10, m11, m20, m21, m22.
__device__ inline void nbg_finish_row_d(const StageGroup& g, const Transform& tf,
                                        const ExceptionSink& ex, uint32_t id, int nnb,
                                        const double Md[6], const int32_t qraw[3]) {
    // covariance as the reference forms it, up to its float narrowing
    const double s0 = tf.scale[0], s1 = tf.scale[1], s2 = tf.scale[2];
    double denom = (double)nnb * (double)(nnb - 1);
    double C[6];  // c00, c10, c11, c20, c21, c22
    C[0] = Md[0] * (s0 * s0) / denom;
    C[1] = Md[1] * (s1 * s0) / denom;
    C[2] = Md[2] * (s1 * s1) / denom;
    C[3] = Md[3] * (s2 * s0) / denom;
    C[4] = Md[4] * (s2 * s1) / denom;
    C[5] = Md[5] * (s2 * s2) / denom;
    bool zero = true;
    int nonfinite = nnb <= 1;
#pragma unroll
    for (int i = 0; i < 6; ++i) zero = zero && (fabs(C[i]) <= 1e-12);
    if (nnb <= 1) zero = false;
    if (nnb == 0) zero = true;
    double ev[3] = {0, 0, 0}, V[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int ok = 1;
    if (g.no_eigen) zero = true;
    if (!zero) {
        if (nonfinite) ok = 0;
        else if (g.sign_exact) ok = nbg_eigen_chain(C, ev, V);
        else if (!nbg_eigen_fast(C, ev, V)) {
            if (g.resolve_count) atomicAdd(g.resolve_count, 1u);
            ok = nbg_eigen_chain(C, ev, V);
        }
    }
    double p[3] = {ref_coord(qraw[0], tf.scale[0], tf.offset[0]),
                   ref_coord(qraw[1], tf.scale[1], tf.offset[1]),
                   ref_coord(qraw[2], tf.scale[2], tf.offset[2])};
    for (int si = 0; si < g.nstages; ++si) {
        const StageDev& st = g.st[si];
        const int sidx = g.stage_index[si];
        if (st.kind == NBG_STAGE_NORMAL) {
            if (nnb < 3) { nbg_append_exception(ex, id, sidx, NBG_ROW_TOO_FEW); continue; }
            if (zero) { nbg_append_exception(ex, id, sidx, NBG_ROW_ZERO_COV); continue; }
            if (!ok) { nbg_append_exception(ex, id, sidx, NBG_ROW_EIGEN_FAIL); continue; }
            double sum = ev[0] + ev[1] + ev[2];
            double curv = sum != 0.0 ? fabs(ev[0] / sum) : 0.0;
            double n0 = V[0], n1 = V[1], n2 = V[2];
            if (st.has_viewpoint) {
                double dx = st.viewpoint[0] - p[0];
                double dy = st.viewpoint[1] - p[1];
                double dz = st.viewpoint[2] - p[2];
                double dot = __dadd_rn(__dadd_rn(__dmul_rn(dx, n0), __dmul_rn(dy, n1)),
                                       __dmul_rn(dz, n2));
                // viewpoint in the tangent plane: the orientation test leaves the
                // eigensolver's own sign, so take it from the Eigen chain
                if (!g.sign_exact &&
                    fabs(dot) <= 1e-12 * (fabs(dx) + fabs(dy) + fabs(dz))) {
                    double ev2[3], V2[9];
                    if (nbg_eigen_chain(C, ev2, V2)) {
                        n0 = V2[0]; n1 = V2[1]; n2 = V2[2];
                        dot = __dadd_rn(__dadd_rn(__dmul_rn(dx, n0), __dmul_rn(dy, n1)),
                                        __dmul_rn(dz, n2));
                    }
                }
                if (dot < 0) { n0 = -n0; n1 = -n1; n2 = -n2; }
            } else if (st.always_up) {
                // horizontal normal: same rule as above, the chain's sign stands
                if (!g.sign_exact && fabs(n2) <= 1e-12) {
                    double ev2[3], V2[9];
                    if (nbg_eigen_chain(C, ev2, V2)) { n0 = V2[0]; n1 = V2[1]; n2 = V2[2]; }
                }
                if (n2 < 0) { n0 = -n0; n1 = -n1; n2 = -n2; }
            }
            nbg_store(st, id, 0, n0);
            nbg_store(st, id, 1, n1);
            nbg_store(st, id, 2, n2);
            nbg_store(st, id, 3, curv);
        } else if (st.kind == NBG_STAGE_APPROXIMATECOPLANAR) {
            // ApproximateCoplanarFilter.cpp:85-113: skipped on a zero
            // covariance; coplanar when l1 > thresh1*l0 and thresh2*l1 > l2
            if (zero) { nbg_append_exception(ex, id, sidx, NBG_ROW_ZERO_COV); continue; }
            if (!ok) { nbg_append_exception(ex, id, sidx, NBG_ROW_EIGEN_FAIL); continue; }
            nbg_store(st, id, 0, (ev[1] > st.t1 * ev[0] && st.t2 * ev[1] > ev[2]) ? 1.0 : 0.0);
        } else if (st.kind == NBG_STAGE_ESTIMATERANK) {
            // MathUtils.cpp:197-208: JacobiSVD rank of the covariance with
            // the float-cast threshold; singular values of the symmetric
            // matrix are |lambda|, counted when at or above
            // max(threshold * sigma_max, DBL_MIN)
            double a0 = 0, a1 = 0, a2 = 0;
            bool any = false;
#pragma unroll
            for (int i = 0; i < 6; ++i) any = any || C[i] != 0.0;
            if (nnb <= 1) {
                // 0/0 covariance: the SVD rejects the non-finite input
                nbg_store(st, id, 0, 0.0);
                continue;
            }
            if (zero && any) {
                double e2[3], V2[9];
                if (nbg_eigen_chain(C, e2, V2)) { a0 = fabs(e2[0]); a1 = fabs(e2[1]); a2 = fabs(e2[2]); }
            } else if (!zero && ok) {
                a0 = fabs(ev[0]);
                a1 = fabs(ev[1]);
                a2 = fabs(ev[2]);
            }
            const double smax = fmax(a0, fmax(a1, a2));
            const double thr = fmax(smax * (double)(float)st.t1, 2.2250738585072014e-308);
            nbg_store(st, id, 0, (double)((a0 >= thr) + (a1 >= thr) + (a2 >= thr)));
        } else if (st.kind == NBG_STAGE_OUTLIER) {
            // OutlierFilter.cpp:80-96: an inlier has more than size_t(min_k)
            // points (itself included) within the radius; a negative min_k
            // converts to a count no row exceeds
            st.aux[id] = (st.ip >= 0 && nnb > st.ip) ? 0.0 : 1.0;
        } else if (st.kind == NBG_STAGE_EIGENVALUES) {
            if (zero) { nbg_append_exception(ex, id, sidx, NBG_ROW_ZERO_COV); continue; }
            if (!ok) { nbg_append_exception(ex, id, sidx, NBG_ROW_EIGEN_FAIL); continue; }
            double e0 = ev[0], e1 = ev[1], e2 = ev[2];
            if (st.normalize) {
                double sum = e0 + e1 + e2;
                e0 /= sum;
                e1 /= sum;
                e2 /= sum;
            }
            nbg_store(st, id, 0, e0);
            nbg_store(st, id, 1, e1);
            nbg_store(st, id, 2, e2);
        } else {
            if (zero) { nbg_append_exception(ex, id, sidx, NBG_ROW_ZERO_COV); continue; }
            if (!ok) { nbg_append_exception(ex, id, sidx, NBG_ROW_EIGEN_FAIL); continue; }
            double l0 = fmax(ev[2], 0.0), l1 = fmax(ev[1], 0.0), l2 = fmax(ev[0], 0.0);
            double sum = ((0.0 + l0) + l1) + l2;
            if (l0 == 0.0) { nbg_append_exception(ex, id, sidx, NBG_ROW_ZERO_LAMBDA); continue; }
            if (st.mode == NBG_MODE_SQRT) {
                l0 = sqrt(l0);
                l1 = sqrt(l1);
                l2 = sqrt(l2);
            } else if (st.mode == NBG_MODE_NORMALIZED) {
                l0 /= sum;
                l1 /= sum;
                l2 /= sum;
            }
            int w = 0;
            const uint32_t mask = st.feature_mask;
            if (mask & NBG_FEAT_LINEARITY) nbg_store(st, id, w++, (l0 - l1) / l0);
            if (mask & NBG_FEAT_PLANARITY) nbg_store(st, id, w++, (l1 - l2) / l0);
            if (mask & NBG_FEAT_SCATTERING) nbg_store(st, id, w++, l2 / l0);
            if (mask & NBG_FEAT_VERTICALITY) {
                double u0 = l0 * fabs(V[6]) + l1 * fabs(V[3]) + l2 * fabs(V[0]);
                double u1 = l0 * fabs(V[7]) + l1 * fabs(V[4]) + l2 * fabs(V[1]);
                double u2 = l0 * fabs(V[8]) + l1 * fabs(V[5]) + l2 * fabs(V[2]);
                double norm = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
                nbg_store(st, id, w++, u2 / norm);
            }
            if (mask & NBG_FEAT_OMNIVARIANCE) nbg_store(st, id, w++, cbrt(l2 * l1 * l0));
            if (mask & NBG_FEAT_ANISOTROPY) nbg_store(st, id, w++, (l0 - l2) / l0);
            if (mask & NBG_FEAT_EIGENENTROPY)
                nbg_store(st, id, w++, -(l2 * log(l2) + l1 * log(l1) + l0 * log(l0)));
            if (mask & NBG_FEAT_EIGENVALUESUM) nbg_store(st, id, w++, sum);
            if (mask & NBG_FEAT_SURFACEVARIATION) nbg_store(st, id, w++, l2 / sum);
            if (mask & NBG_FEAT_DEMANTKEVERTICALITY) nbg_store(st, id, w++, 1.0 - fabs(V[2]));
            if (mask & NBG_FEAT_DENSITY) {
                double kopt = g.optimal_knn ? g.optimal_knn[id] : 0.0;
                double ropt = g.optimal_radius ? g.optimal_radius[id] : 0.0;
                const double pi = 3.14159265;
                nbg_store(st, id, w++, (kopt + 1.0) / ((4.0 / 3.0) * pi * (ropt * ropt * ropt)));
            }
        }
    }
}

__device__ inline void nbg_finish_row(const StageGroup& g, const Transform& tf,
                                      const ExceptionSink& ex, uint32_t id, int nnb,
                                      const long long M[6], const int32_t qraw[3]) {
    const double Md[6] = {(double)M[0], (double)M[1], (double)M[2],
                          (double)M[3], (double)M[4], (double)M[5]};
    nbg_finish_row_d(g, tf, ex, id, nnb, Md, qraw);
}

// ref_shim.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// The same C entry points as nbg_oracle.cpp (orc_*), but compiled over the
// reference's own vendored nanoflann 1.3.1 and Eigen 3.4 headers where they
// lie in the reference tree (oracle/Makefile passes the include paths; no
// reference source is copied into this repository).  The adapter and the
// per-point loops restate, with the real library types, the reference's
//   pdal/private/KDImpl.hpp:209-381        (KD3ImplT adapter, neighbors)
//   pdal/private/MathUtils.cpp:139-196     (computeCentroid/Covariance)
//   pdal/private/MathUtils.cpp:572-611     (findNormal)
//   filters/NormalFilter.cpp:140-182
//   filters/EigenvaluesFilter.cpp:115-172
//   filters/CovarianceFeaturesFilter.cpp:204-367
// and, through consumers.hpp, the other consumers of the same index
// (approximatecoplanar, estimaterank, nndistance, optimalneighborhood, lof,
// outlier).
// The result is the reference's CPU path without the PDAL framework (which
// needs GDAL and does not build here).  Output goes to oracle/_ref/ only.

#include <nanoflann/nanoflann.hpp>

#include <Eigen/Dense>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>

#include "../include/nbg_b200.h"
#include "consumers.hpp"

namespace {

using PointId = uint64_t;
using PointIdList = std::vector<PointId>;

struct Cloud {
    std::vector<std::array<double, 3>> pts;

    std::size_t kdtree_get_point_count() const { return pts.size(); }
    double kdtree_get_pt(const PointId idx, int dim) const {
        if (idx >= pts.size()) return 0.0;
        return pts[idx][dim];
    }
    double kdtree_distance(const double* p1, const PointId p2, size_t) const {
        double d0 = p1[0] - pts[p2][0];
        double d1 = p1[1] - pts[p2][1];
        double d2 = p1[2] - pts[p2][2];
        return (d0 * d0 + d1 * d1 + d2 * d2);
    }
    template <class BBOX>
    bool kdtree_get_bbox(BBOX& bb) const {
        if (pts.empty()) {
            bb = {};
            return true;
        }
        double lo[3], hi[3];
        for (int d = 0; d < 3; ++d) lo[d] = hi[d] = pts[0][d];
        for (const auto& p : pts)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], p[d]);
                hi[d] = std::max(hi[d], p[d]);
            }
        bb = {{lo[0], hi[0]}, {lo[1], hi[1]}, {lo[2], hi[2]}};
        return true;
    }
};

using KDTree = nanoflann::KDTreeSingleIndexAdaptor<
    nanoflann::L2_Simple_Adaptor<double, Cloud, double>, Cloud, -1, std::size_t>;

struct RefTree {
    Cloud cloud;
    KDTree index;
    RefTree() : index(3, cloud, nanoflann::KDTreeSingleIndexAdaptorParams(100)) {}

    // KD3ImplT::radius (KDImpl.hpp:398-415)
    PointIdList radius(double x, double y, double z, double r) const {
        PointIdList output;
        std::vector<std::pair<std::size_t, double>> ret_matches;
        nanoflann::SearchParams params;
        params.sorted = true;
        std::vector<double> pt{x, y, z};
        const std::size_t count = index.radiusSearch(&pt[0], r * r, ret_matches, params);
        for (std::size_t i = 0; i < count; ++i) output.push_back(ret_matches[i].first);
        return output;
    }

    // KD3ImplT::knnSearch (KDImpl.hpp:383-396): the caller's k-sized
    // vectors, min(n, k) entries filled
    void knn_search(double x, double y, double z, uint64_t k, PointIdList* indices,
                    std::vector<double>* sqr_dists) const {
        k = (std::min<uint64_t>)(cloud.pts.size(), k);
        nanoflann::KNNResultSet<double, PointId, uint64_t> resultSet(k);
        resultSet.init(&indices->front(), &sqr_dists->front());
        std::vector<double> pt{x, y, z};
        index.findNeighbors(resultSet, &pt[0], nanoflann::SearchParams(10));
    }

    PointIdList neighbors(double x, double y, double z, uint64_t k, size_t stride) const {
        k = (std::min<uint64_t>)(cloud.pts.size(), k);
        uint64_t k2 = stride * k;
        PointIdList output(k2);
        if (k2 == 0) return output;  // nanoflann's worstDist would read before its buffer
        std::vector<double> out_dist_sqr(k2);
        std::vector<double> pt{x, y, z};
        nanoflann::KNNResultSet<double, PointId, uint64_t> resultSet(k2);
        resultSet.init(&output[0], &out_dist_sqr[0]);
        index.findNeighbors(resultSet, &pt[0], nanoflann::SearchParams());
        if (stride > 1) {
            for (size_t i = 1; i < k; ++i) output[i] = output[i * stride];
            output.resize(k);
        }
        return output;
    }
};

Eigen::Vector3d centroid(const Cloud& c, const PointIdList& ids) {
    double mx, my, mz;
    mx = my = mz = 0.0;
    uint64_t n(0);
    for (auto const& j : ids) {
        auto update = [&n](double value, double average) {
            double delta, delta_n;
            delta = value - average;
            delta_n = delta / n;
            return average + delta_n;
        };
        n++;
        mx = update(c.pts[j][0], mx);
        my = update(c.pts[j][1], my);
        mz = update(c.pts[j][2], mz);
    }
    Eigen::Vector3d r;
    r << mx, my, mz;
    return r;
}

Eigen::Matrix3d covariance(const Cloud& c, const PointIdList& ids) {
    auto n = ids.size();
    Eigen::Vector3d cen = centroid(c, ids);
    Eigen::MatrixXd A(3, n);
    size_t k = 0;
    for (auto const& j : ids) {
        A(0, k) = static_cast<float>(c.pts[j][0] - cen[0]);
        A(1, k) = static_cast<float>(c.pts[j][1] - cen[1]);
        A(2, k) = static_cast<float>(c.pts[j][2] - cen[2]);
        k++;
    }
    return A * A.transpose() / (ids.size() - 1);
}

int stage_row(const nbg_stage_opts& o, const RefTree& t, uint64_t i, const double* kopt_col,
              const double* ropt_col, double* out) {
    const auto& p = t.cloud.pts[i];
    PointIdList ids;
    if (o.kind == NBG_STAGE_NORMAL) {
        if (o.use_radius) ids = t.radius(p[0], p[1], p[2], o.radius);
        else ids = t.neighbors(p[0], p[1], p[2], (uint64_t)(o.knn + 1), 1);
        if (ids.size() < 3) return NBG_ROW_TOO_FEW;
        auto B = covariance(t.cloud, ids);
        if (B.isZero()) return NBG_ROW_ZERO_COV;
        Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(B);
        if (solver.info() != Eigen::Success) return NBG_ROW_EIGEN_FAIL;
        auto eval = solver.eigenvalues();
        double sum = eval[0] + eval[1] + eval[2];
        double curvature = sum ? std::fabs(eval[0] / sum) : 0;
        Eigen::Vector3d normal = solver.eigenvectors().col(0);
        if (normal.isZero()) return NBG_ROW_EIGEN_FAIL;
        if (o.has_viewpoint) {
            Eigen::Vector3d vp(o.viewpoint[0] - p[0], o.viewpoint[1] - p[1],
                               o.viewpoint[2] - p[2]);
            normal = (vp.dot(normal) < 0 ? Eigen::Vector3d(-normal) : normal);
        } else if (o.always_up) {
            normal = ((normal(2) < 0) ? Eigen::Vector3d(-normal) : normal);
        }
        out[0] = normal[0];
        out[1] = normal[1];
        out[2] = normal[2];
        out[3] = curvature;
        return 0;
    }
    if (o.kind == NBG_STAGE_EIGENVALUES) {
        if (o.use_radius) {
            ids = t.radius(p[0], p[1], p[2], o.radius);
            if (ids.size() < (size_t)o.min_k) return NBG_ROW_RADIUS_FEW;
        } else {
            ids = t.neighbors(p[0], p[1], p[2], (uint64_t)(o.knn + 1), (size_t)o.stride);
        }
        Eigen::Matrix3d B = covariance(t.cloud, ids);
        if (B.isZero()) return NBG_ROW_ZERO_COV;
        Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(B);
        if (solver.info() != Eigen::Success) return NBG_ROW_EIGEN_FAIL;
        Eigen::Vector3d ev = solver.eigenvalues();
        if (o.normalize) {
            double sum = ev[0] + ev[1] + ev[2];
            ev /= sum;
        }
        out[0] = ev[0];
        out[1] = ev[1];
        out[2] = ev[2];
        return 0;
    }
    if (o.optimized) {
        ids = t.neighbors(p[0], p[1], p[2], (uint64_t)kopt_col[i], 1);
    } else if (o.use_radius) {
        ids = t.radius(p[0], p[1], p[2], o.radius);
        if (ids.size() < (size_t)o.min_k) return NBG_ROW_RADIUS_FEW;
    } else {
        ids = t.neighbors(p[0], p[1], p[2], (uint64_t)(o.knn + 1), (size_t)o.stride);
    }
    auto B = covariance(t.cloud, ids);
    if (B.isZero()) return NBG_ROW_ZERO_COV;
    Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(B);
    if (solver.info() != Eigen::Success) return NBG_ROW_EIGEN_FAIL;
    auto ev = solver.eigenvalues();
    std::vector<double> lambda = {((std::max)(ev[2], 0.0)), ((std::max)(ev[1], 0.0)),
                                  ((std::max)(ev[0], 0.0))};
    double sum = std::accumulate(lambda.begin(), lambda.end(), 0.0);
    if (lambda[0] == 0) return NBG_ROW_ZERO_LAMBDA;
    if (o.mode == NBG_MODE_SQRT)
        std::transform(lambda.begin(), lambda.end(), lambda.begin(),
                       [](double v) -> double { return std::sqrt(v); });
    else if (o.mode == NBG_MODE_NORMALIZED)
        std::transform(lambda.begin(), lambda.end(), lambda.begin(),
                       [&sum](double v) -> double { return v / sum; });
    auto V = solver.eigenvectors();
    std::vector<double> v1(3), v2(3), v3(3);
    for (int k = 0; k < 3; k++) {
        v1[k] = V.col(2)(k);
        v2[k] = V.col(1)(k);
        v3[k] = V.col(0)(k);
    }
    int w = 0;
    for (int f = 0; f < NBG_NUM_FEATURES; ++f) {
        if (!(o.feature_mask & (1u << f))) continue;
        double val = 0;
        switch (1u << f) {
            case NBG_FEAT_LINEARITY: val = (lambda[0] - lambda[1]) / lambda[0]; break;
            case NBG_FEAT_PLANARITY: val = (lambda[1] - lambda[2]) / lambda[0]; break;
            case NBG_FEAT_SCATTERING: val = lambda[2] / lambda[0]; break;
            case NBG_FEAT_VERTICALITY: {
                std::vector<double> u(3);
                double norm = 0;
                for (int k = 0; k < 3; k++) {
                    u[k] = lambda[0] * fabs(v1[k]) + lambda[1] * fabs(v2[k]) +
                           lambda[2] * fabs(v3[k]);
                    norm += u[k] * u[k];
                }
                norm = sqrt(norm);
                val = u[2] / norm;
                break;
            }
            case NBG_FEAT_OMNIVARIANCE: val = std::cbrt(lambda[2] * lambda[1] * lambda[0]); break;
            case NBG_FEAT_ANISOTROPY: val = (lambda[0] - lambda[2]) / lambda[0]; break;
            case NBG_FEAT_EIGENENTROPY:
                val = -(lambda[2] * std::log(lambda[2]) + lambda[1] * std::log(lambda[1]) +
                        lambda[0] * std::log(lambda[0]));
                break;
            case NBG_FEAT_EIGENVALUESUM: val = sum; break;
            case NBG_FEAT_SURFACEVARIATION: val = lambda[2] / sum; break;
            case NBG_FEAT_DEMANTKEVERTICALITY: {
                auto e3 = V.col(0);
                val = 1 - std::fabs(e3[2]);
                break;
            }
            case NBG_FEAT_DENSITY: {
                double kopt = kopt_col[i];
                double ropt = ropt_col[i];
                double pi = 3.14159265;
                val = (kopt + 1.0) / ((4.0 / 3.0) * pi * std::pow(ropt, 3));
                break;
            }
        }
        out[w++] = val;
    }
    return 0;
}

// The reference's backend of the shared consumer loops (consumers.hpp):
// its nanoflann search, its computeCovariance, Eigen's solver and JacobiSVD.
struct RefBackend {
    const RefTree* t;
    uint64_t n() const { return t->cloud.pts.size(); }
    double coord(uint64_t i, int d) const { return t->cloud.pts[i][d]; }
    void knn(uint64_t i, uint64_t k, PointIdList& ids, std::vector<double>& d2) const {
        const auto& p = t->cloud.pts[i];
        t->knn_search(p[0], p[1], p[2], k, &ids, &d2);
    }
    PointIdList neighbors(uint64_t i, uint64_t k) const {
        const auto& p = t->cloud.pts[i];
        return t->neighbors(p[0], p[1], p[2], k, 1);
    }
    uint64_t radius_count(uint64_t i, double r) const {
        const auto& p = t->cloud.pts[i];
        return t->radius(p[0], p[1], p[2], r).size();
    }
    int cov_eigenvalues(const PointIdList& ids, int, double ev[3]) const {
        Eigen::Matrix3d B = covariance(t->cloud, ids);
        if (B.isZero()) return NBG_ROW_ZERO_COV;
        Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(B);
        if (solver.info() != Eigen::Success) return NBG_ROW_EIGEN_FAIL;
        for (int c = 0; c < 3; ++c) ev[c] = solver.eigenvalues()[c];
        return 0;
    }
    // MathUtils.cpp:197-208.  A one-point neighbourhood gives a 0/0 matrix
    // whose JacobiSVD rank reads an unset count; 0 is returned for it.
    int rank(const PointIdList& ids, double thresh, int) const {
        if (ids.size() <= 1) return 0;
        Eigen::Matrix3d B = covariance(t->cloud, ids);
        Eigen::JacobiSVD<Eigen::Matrix3d> svd(B);
        svd.setThreshold((float)thresh);
        return (int)svd.rank();
    }
    bool sym_eigenvalues(const double A[3][3], double ev[3]) const {
        Eigen::Matrix3d M;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) M(r, c) = A[r][c];
        Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(M);
        if (solver.info() != Eigen::Success) return false;
        for (int c = 0; c < 3; ++c) ev[c] = solver.eigenvalues()[c];
        return true;
    }
};

template <class F>
void parallel_rows(uint64_t n, int threads, F&& fn) {
    if (threads <= 1 || n < 1024) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> ts;
    uint64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        uint64_t b = std::min<uint64_t>(n, t * chunk), e = std::min<uint64_t>(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back([&, b, e] { fn(b, e); });
    }
    for (auto& t : ts) t.join();
}

}  // namespace

extern "C" {

const char* orc_impl_name(void) { return "reference"; }

// build_threads 0: the KD3 build's own choice, up to eight threads (the
// threaded build yields the serial tree); n > 0 caps it at n threads
void* orc_tree_build_t(const double* x, const double* y, const double* z, uint64_t n,
                       int build_threads) {
    RefTree* t = new RefTree();
    t->cloud.pts.resize(n);
    for (uint64_t i = 0; i < n; ++i) t->cloud.pts[i] = {x[i], y[i], z[i]};
    int threads = n < 256 ? 1 : (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency()));
    if (build_threads > 0) threads = std::min(threads, build_threads);
    t->index.set_build_threads(threads);
    t->index.buildIndex();
    return t;
}

void* orc_tree_build(const double* x, const double* y, const double* z, uint64_t n) {
    return orc_tree_build_t(x, y, z, n, 0);
}

void orc_tree_free(void* h) { delete (RefTree*)h; }

uint64_t orc_tree_neighbors(void* hv, double qx, double qy, double qz, uint64_t k,
                            uint64_t stride, uint64_t* out) {
    RefTree* t = (RefTree*)hv;
    PointIdList ids = t->neighbors(qx, qy, qz, k, stride);
    std::copy(ids.begin(), ids.end(), out);
    return ids.size();
}

void orc_all_neighbors(void* hv, uint64_t k, uint64_t* out, int threads) {
    RefTree* t = (RefTree*)hv;
    const uint64_t n = t->cloud.pts.size();
    const uint64_t k1 = std::min<uint64_t>(n, k);
    parallel_rows(n, threads, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const auto& p = t->cloud.pts[i];
            PointIdList ids = t->neighbors(p[0], p[1], p[2], k, 1);
            std::copy(ids.begin(), ids.end(), out + i * k1);
        }
    });
}

uint64_t orc_tree_num_nodes(void*) { return 0; }

void orc_tree_export(void* hv, uint64_t* vind, int64_t*, int64_t*, int32_t*, double*, double*,
                     uint64_t*, uint64_t*) {
    RefTree* t = (RefTree*)hv;
    std::copy(t->index.vind.begin(), t->index.vind.end(), vind);
}

int orc_eigen_chain(const double* a, double* eval, double* evec_colmajor) {
    Eigen::Matrix3d B;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B(i, j) = a[i * 3 + j];
    Eigen::SelfAdjointEigenSolver<Eigen::Matrix3d> solver(B);
    for (int i = 0; i < 3; ++i) eval[i] = solver.eigenvalues()[i];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) evec_colmajor[c * 3 + r] = solver.eigenvectors()(r, c);
    return solver.info() == Eigen::Success;
}

int orc_run_stage(void* hv, const nbg_stage_opts* opts, const double* optimal_knn,
                  const double* optimal_radius, int mode, double** out_cols, uint8_t* status,
                  int threads) {
    if (mode != 0) return -2;  // the reference has only its own arithmetic
    RefTree* t = (RefTree*)hv;
    const nbg_stage_opts o = *opts;
    if (o.kind > NBG_STAGE_COVARIANCEFEATURES)
        return orc_consumers::run_consumer(RefBackend{t}, o, 0, out_cols, status, threads,
                                           [](uint64_t m, int th, auto&& fn) { parallel_rows(m, th, fn); });
    const uint64_t n = t->cloud.pts.size();
    int nd = o.kind == NBG_STAGE_NORMAL ? 4
             : o.kind == NBG_STAGE_EIGENVALUES ? 3
                                               : __builtin_popcount(o.feature_mask & NBG_FEAT_ALL);
    parallel_rows(n, threads, [&](uint64_t b, uint64_t e) {
        double vals[NBG_MAX_DIMS];
        for (uint64_t i = b; i < e; ++i) {
            int code = stage_row(o, *t, i, optimal_knn, optimal_radius, vals);
            status[i] = (uint8_t)code;
            if (code == 0)
                for (int d = 0; d < nd; ++d) out_cols[d][i] = vals[d];
        }
    });
    return 0;
}

}  // extern "C"

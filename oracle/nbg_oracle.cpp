// nbg_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU restatement of the reference's neighbourhood-geometry path, used only
// as the checker by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline.  Nothing in the product library links or calls this file.
//
// Restated from the reference (paths inside the PDAL fork):
//   * nanoflann 1.3.1 KD-tree build and exact kNN search
//       vendor/nanoflann/nanoflann.hpp:145-208 (KNNResultSet),
//       :640-690 (divideTree), :779-828 (middleSplit_), :837-873 (planeSplit),
//       :875-893 (computeInitialDistances), :1012-1033 (buildIndex),
//       :1059-1079 (findNeighbors), :1184-1250 (searchLevel)
//   * the PDAL KD3 adapter: leaf size 100, bbox = calculateBounds, distance
//       d0*d0 + d1*d1 + d2*d2 in double   pdal/private/KDImpl.hpp:209-381
//   * computeCentroid / computeCovariance / findNormal
//       pdal/private/MathUtils.cpp:139-196, 572-611
//   * Eigen 3.4 SelfAdjointEigenSolver<Matrix3d> (3x3 Householder
//       tridiagonalisation, implicit symmetric QR with Wilkinson shift,
//       continuous Givens rotations, selection sort of eigenvalues)
//       vendor/eigen/Eigen/src/Eigenvalues/SelfAdjointEigenSolver.h:420-570,
//       :835-895; Tridiagonalization.h:464-504; Jacobi/Jacobi.h:228-265
//   * stage projections: filters/NormalFilter.cpp:140-182,
//       filters/EigenvaluesFilter.cpp:115-172,
//       filters/CovarianceFeaturesFilter.cpp:204-367
//
// Two numeric modes:
//   mode 0 ("ref")  the reference's own arithmetic: online centroid, float
//                   narrowing of the centred coordinates, A*A^T/(n-1), the
//                   Eigen QR chain in double.
//   mode 1 ("f64")  the accuracy oracle: the same neighbour sets, the
//                   covariance of the same double coordinates without
//                   narrowing, accumulated and solved (cyclic Jacobi) in
//                   long double.  Eigenvector signs follow the Eigen chain.
//
// Parity of this restatement is pinned against oracle/_ref (the same entry
// points compiled over the reference's vendored nanoflann and Eigen) and the
// golden vectors in tests/golden/.
//
// Build with -ffp-contract=off: the reference's x86-64 build has no FMA
// contraction, and every distance must round exactly as it does there.

#include "../include/nbg_b200.h"
#include "consumers.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// KD-tree (nanoflann 1.3.1 semantics, leaf_max_size 100, IndexType size_t)
// ---------------------------------------------------------------------------
struct Node {
    int64_t child1 = -1, child2 = -1;  // -1 marks a leaf
    uint64_t left = 0, right = 0;      // leaf range into vind
    int divfeat = 0;
    double divlow = 0.0, divhigh = 0.0;
};

class KdTree {
public:
    const double* c[3] = {nullptr, nullptr, nullptr};
    uint64_t n = 0;
    uint64_t leaf_max = 100;
    std::vector<uint64_t> vind;
    std::vector<Node> nodes;  // preorder, root at 0
    double root_lo[3] = {0, 0, 0}, root_hi[3] = {0, 0, 0};

    double get(uint64_t id, int d) const { return c[d][id]; }

    void build() {
        vind.resize(n);
        for (uint64_t i = 0; i < n; ++i) vind[i] = i;
        nodes.clear();
        if (n == 0) return;
        // PointView::calculateBounds (PointView.cpp:159-169): plain min/max
        double lo[3], hi[3];
        for (int d = 0; d < 3; ++d) { lo[d] = hi[d] = get(0, d); }
        for (uint64_t i = 1; i < n; ++i)
            for (int d = 0; d < 3; ++d) {
                double v = get(i, d);
                if (v < lo[d]) lo[d] = v;
                if (v > hi[d]) hi[d] = v;
            }
        nodes.reserve(2 * (n / 50 + 1));
        divide(0, n, lo, hi);
        for (int d = 0; d < 3; ++d) { root_lo[d] = lo[d]; root_hi[d] = hi[d]; }
    }

    // Returns the node index; lo/hi enter as the top-down box and leave as
    // the actual extent of the subtree's points.
    int64_t divide(uint64_t left, uint64_t right, double lo[3], double hi[3]) {
        int64_t id = (int64_t)nodes.size();
        nodes.emplace_back();
        if (right - left <= leaf_max) {
            nodes[id].left = left;
            nodes[id].right = right;
            for (int d = 0; d < 3; ++d) lo[d] = hi[d] = get(vind[left], d);
            for (uint64_t k = left + 1; k < right; ++k)
                for (int d = 0; d < 3; ++d) {
                    double v = get(vind[k], d);
                    if (lo[d] > v) lo[d] = v;
                    if (hi[d] < v) hi[d] = v;
                }
            return id;
        }
        uint64_t idx;
        int cutfeat;
        double cutval;
        middle_split(&vind[left], right - left, idx, cutfeat, cutval, lo, hi);
        nodes[id].divfeat = cutfeat;
        double llo[3], lhi[3], rlo[3], rhi[3];
        for (int d = 0; d < 3; ++d) { llo[d] = rlo[d] = lo[d]; lhi[d] = rhi[d] = hi[d]; }
        lhi[cutfeat] = cutval;
        int64_t c1 = divide(left, left + idx, llo, lhi);
        rlo[cutfeat] = cutval;
        int64_t c2 = divide(left + idx, right, rlo, rhi);
        nodes[id].child1 = c1;
        nodes[id].child2 = c2;
        nodes[id].divlow = lhi[cutfeat];
        nodes[id].divhigh = rlo[cutfeat];
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(llo[d], rlo[d]);
            hi[d] = std::max(lhi[d], rhi[d]);
        }
        return id;
    }

    void min_max(const uint64_t* ind, uint64_t count, int d, double& mn, double& mx) const {
        mn = mx = get(ind[0], d);
        for (uint64_t i = 1; i < count; ++i) {
            double v = get(ind[i], d);
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
    }

    void middle_split(uint64_t* ind, uint64_t count, uint64_t& index, int& cutfeat,
                      double& cutval, const double lo[3], const double hi[3]) const {
        const double EPS = 0.00001;
        double max_span = hi[0] - lo[0];
        for (int i = 1; i < 3; ++i) {
            double span = hi[i] - lo[i];
            if (span > max_span) max_span = span;
        }
        double max_spread = -1;
        cutfeat = 0;
        for (int i = 0; i < 3; ++i) {
            double span = hi[i] - lo[i];
            if (span > (1 - EPS) * max_span) {
                double mn, mx;
                min_max(ind, count, i, mn, mx);
                double spread = mx - mn;
                if (spread > max_spread) {
                    cutfeat = i;
                    max_spread = spread;
                }
            }
        }
        double split_val = (lo[cutfeat] + hi[cutfeat]) / 2;
        double mn, mx;
        min_max(ind, count, cutfeat, mn, mx);
        if (split_val < mn) cutval = mn;
        else if (split_val > mx) cutval = mx;
        else cutval = split_val;
        uint64_t lim1, lim2;
        plane_split(ind, count, cutfeat, cutval, lim1, lim2);
        if (lim1 > count / 2) index = lim1;
        else if (lim2 < count / 2) index = lim2;
        else index = count / 2;
    }

    // Two Hoare-style passes; the unsigned-index guards are part of the
    // behaviour being restated.
    void plane_split(uint64_t* ind, uint64_t count, int f, double cutval, uint64_t& lim1,
                     uint64_t& lim2) const {
        uint64_t left = 0, right = count - 1;
        for (;;) {
            while (left <= right && get(ind[left], f) < cutval) ++left;
            while (right && left <= right && get(ind[right], f) >= cutval) --right;
            if (left > right || !right) break;
            std::swap(ind[left], ind[right]);
            ++left;
            --right;
        }
        lim1 = left;
        right = count - 1;
        for (;;) {
            while (left <= right && get(ind[left], f) <= cutval) ++left;
            while (right && left <= right && get(ind[right], f) > cutval) --right;
            if (left > right || !right) break;
            std::swap(ind[left], ind[right]);
            ++left;
            --right;
        }
        lim2 = left;
    }

    // --- search ------------------------------------------------------------
    struct Result {
        uint64_t cap = 0, count = 0;
        uint64_t* ids = nullptr;
        double* d = nullptr;
        void init(uint64_t* i, double* dd) {
            ids = i;
            d = dd;
            count = 0;
            if (cap) d[cap - 1] = std::numeric_limits<double>::max();
        }
        double worst() const { return d[cap - 1]; }
        void add(double dist, uint64_t id) {
            uint64_t i;
            for (i = count; i > 0; --i) {
                if (d[i - 1] > dist) {
                    if (i < cap) { d[i] = d[i - 1]; ids[i] = ids[i - 1]; }
                } else break;
            }
            if (i < cap) { d[i] = dist; ids[i] = id; }
            if (count < cap) count++;
        }
    };

    // nanoflann's RadiusResultSet (nanoflann.hpp:225-275): keeps every point
    // with dist < radius; its worst distance is the radius itself
    struct RadiusResult {
        double radius = 0.0;
        std::vector<std::pair<uint64_t, double>> found;
        double worst() const { return radius; }
        void add(double dist, uint64_t id) {
            if (dist < radius) found.emplace_back(id, dist);
        }
    };

    double metric(const double* q, uint64_t id) const {
        double r = 0.0;
        for (int d = 0; d < 3; ++d) {
            const double diff = q[d] - get(id, d);
            r += diff * diff;
        }
        return r;
    }

    template <class RS>
    void search_level(RS& rs, const double* q, int64_t node, double mindistsq,
                      double* dists) const {
        const Node& nd = nodes[node];
        if (nd.child1 < 0 && nd.child2 < 0) {
            double worst = rs.worst();
            for (uint64_t i = nd.left; i < nd.right; ++i) {
                const uint64_t index = vind[i];
                double dist = metric(q, index);
                if (dist < worst) rs.add(dist, index);
            }
            return;
        }
        int idx = nd.divfeat;
        double val = q[idx];
        double diff1 = val - nd.divlow;
        double diff2 = val - nd.divhigh;
        int64_t best, other;
        double cut;
        if ((diff1 + diff2) < 0) {
            best = nd.child1;
            other = nd.child2;
            cut = (val - nd.divhigh) * (val - nd.divhigh);
        } else {
            best = nd.child2;
            other = nd.child1;
            cut = (val - nd.divlow) * (val - nd.divlow);
        }
        search_level(rs, q, best, mindistsq, dists);
        double dst = dists[idx];
        mindistsq = mindistsq + cut - dst;
        dists[idx] = cut;
        if (mindistsq * 1.0f <= rs.worst()) search_level(rs, q, other, mindistsq, dists);
        dists[idx] = dst;
    }

    // KD3ImplT::radius(x, y, z, r): ids with squared distance < r*r, sorted by
    // distance (KDImpl.hpp:398-415; radiusSearch with params.sorted)
    void radius_neighbors(const double q[3], double r, std::vector<uint64_t>& out) const {
        RadiusResult rs;
        rs.radius = r * r;
        out.clear();
        if (n == 0) return;
        double dists[3] = {0, 0, 0};
        double distsq = 0.0;
        for (int i = 0; i < 3; ++i) {
            if (q[i] < root_lo[i]) {
                dists[i] = (q[i] - root_lo[i]) * (q[i] - root_lo[i]);
                distsq += dists[i];
            }
            if (q[i] > root_hi[i]) {
                dists[i] = (q[i] - root_hi[i]) * (q[i] - root_hi[i]);
                distsq += dists[i];
            }
        }
        search_level(rs, q, 0, distsq, dists);
        std::stable_sort(rs.found.begin(), rs.found.end(),
                         [](const std::pair<uint64_t, double>& a, const std::pair<uint64_t, double>& b) {
                             return a.second < b.second;
                         });
        for (auto& f : rs.found) out.push_back(f.first);
    }

    // KD3ImplT::knnSearch (KDImpl.hpp:383-396): min(n, k) entries of the
    // caller's k-sized vectors filled in the search's order
    void knn_search(const double q[3], uint64_t k, std::vector<uint64_t>& ids,
                    std::vector<double>& d2) const {
        Result rs;
        rs.cap = std::min<uint64_t>(n, k);
        if (rs.cap == 0) return;
        rs.init(ids.data(), d2.data());
        double dists[3] = {0, 0, 0};
        double distsq = 0.0;
        for (int i = 0; i < 3; ++i) {
            if (q[i] < root_lo[i]) {
                dists[i] = (q[i] - root_lo[i]) * (q[i] - root_lo[i]);
                distsq += dists[i];
            }
            if (q[i] > root_hi[i]) {
                dists[i] = (q[i] - root_hi[i]) * (q[i] - root_hi[i]);
                distsq += dists[i];
            }
        }
        search_level(rs, q, 0, distsq, dists);
    }

    // KD3ImplT::neighbors(x, y, z, k, stride): returns the id list
    void neighbors(const double q[3], uint64_t k, uint64_t stride,
                   std::vector<uint64_t>& out) const {
        k = std::min<uint64_t>(n, k);
        uint64_t k2 = stride * k;
        out.assign(k2, 0);
        std::vector<double> dist(k2);
        Result rs;
        rs.cap = k2;
        rs.init(out.data(), dist.data());
        // k = 0: the reference's result set then reads outside its (empty)
        // buffer (KDImpl.hpp:357-371 with nanoflann's worstDist); the only
        // observable outcome is the empty neighbourhood, returned here
        if (n != 0 && k2 != 0) {
            double dists[3] = {0, 0, 0};
            double distsq = 0.0;
            for (int i = 0; i < 3; ++i) {
                if (q[i] < root_lo[i]) {
                    dists[i] = (q[i] - root_lo[i]) * (q[i] - root_lo[i]);
                    distsq += dists[i];
                }
                if (q[i] > root_hi[i]) {
                    dists[i] = (q[i] - root_hi[i]) * (q[i] - root_hi[i]);
                    distsq += dists[i];
                }
            }
            search_level(rs, q, 0, distsq, dists);
        }
        if (stride > 1) {
            for (uint64_t i = 1; i < k; ++i) out[i] = out[i * stride];
            out.resize(k);
        }
    }
};

// ---------------------------------------------------------------------------
// Eigen 3.4 SelfAdjointEigenSolver<Matrix3d> restated (double).
// Returns 1 on success (ComputationInfo::Success), 0 on NoConvergence.
// evec is column-major: evec[c*3 + r] = component r of eigenvector c.
// ---------------------------------------------------------------------------
static void make_givens(double p, double q, double& c, double& s) {
    if (q == 0.0) {
        c = p < 0.0 ? -1.0 : 1.0;
        s = 0.0;
    } else if (p == 0.0) {
        c = 0.0;
        s = q < 0.0 ? 1.0 : -1.0;
    } else if (std::fabs(p) > std::fabs(q)) {
        double t = q / p;
        double u = std::sqrt(1.0 + t * t);
        if (p < 0.0) u = -u;
        c = 1.0 / u;
        s = -t * c;
    } else {
        double t = p / q;
        double u = std::sqrt(1.0 + t * t);
        if (q < 0.0) u = -u;
        s = -1.0 / u;
        c = -t * s;
    }
}

static double pos_hypot(double x, double y) {
    if (std::isinf(x) || std::isinf(y)) return std::numeric_limits<double>::infinity();
    if (std::isnan(x) || std::isnan(y)) return std::numeric_limits<double>::quiet_NaN();
    double p = std::max(x, y);
    if (p == 0.0) return 0.0;
    double qp = std::min(y, x) / p;
    return p * std::sqrt(1.0 + qp * qp);
}

int eigen_chain(const double A[3][3], double eval[3], double evec[9]) {
    // lower triangle, scaled into [-1, 1]
    double m[3][3] = {{A[0][0], 0, 0}, {A[1][0], A[1][1], 0}, {A[2][0], A[2][1], A[2][2]}};
    double scale = 0.0;
    bool has_nan = false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double a = std::fabs(m[i][j]);
            if (std::isnan(a)) has_nan = true;
            if (a > scale) scale = a;
        }
    if (has_nan) scale = std::numeric_limits<double>::quiet_NaN();
    if (scale == 0.0) scale = 1.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) m[i][j] /= scale;

    double diag[3], sub[2];
    double Q[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // column-major
    {
        const double tol = DBL_MIN;
        diag[0] = m[0][0];
        double v1norm2 = m[2][0] * m[2][0];
        if (v1norm2 <= tol) {
            diag[1] = m[1][1];
            diag[2] = m[2][2];
            sub[0] = m[1][0];
            sub[1] = m[2][1];
        } else {
            double beta = std::sqrt(m[1][0] * m[1][0] + v1norm2);
            double invBeta = 1.0 / beta;
            double m01 = m[1][0] * invBeta;
            double m02 = m[2][0] * invBeta;
            double q = 2.0 * m01 * m[2][1] + m02 * (m[2][2] - m[1][1]);
            diag[1] = m[1][1] + m02 * q;
            diag[2] = m[2][2] - m02 * q;
            sub[0] = beta;
            sub[1] = m[2][1] - m01 * q;
            // rows (1,0,0), (0,m01,m02), (0,m02,-m01) in column-major
            Q[0] = 1; Q[1] = 0; Q[2] = 0;
            Q[3] = 0; Q[4] = m01; Q[5] = m02;
            Q[6] = 0; Q[7] = m02; Q[8] = -m01;
        }
    }

    const int n = 3;
    int end = n - 1, start = 0, iter = 0;
    const double considerAsZero = DBL_MIN;
    const double precision_inv = 1.0 / DBL_EPSILON;
    const int maxIterations = 30;
    while (end > 0) {
        for (int i = start; i < end; ++i) {
            if (std::fabs(sub[i]) < considerAsZero) sub[i] = 0.0;
            else {
                const double scaled = precision_inv * sub[i];
                if (scaled * scaled <= (std::fabs(diag[i]) + std::fabs(diag[i + 1]))) sub[i] = 0.0;
            }
        }
        while (end > 0 && sub[end - 1] == 0.0) end--;
        if (end <= 0) break;
        iter++;
        if (iter > maxIterations * n) break;
        start = end - 1;
        while (start > 0 && sub[start - 1] != 0.0) start--;
        // Francis implicit QR step with Wilkinson shift
        double td = (diag[end - 1] - diag[end]) * 0.5;
        double e = sub[end - 1];
        double mu = diag[end];
        if (td == 0.0) {
            mu -= std::fabs(e);
        } else if (e != 0.0) {
            const double e2 = e * e;
            const double h = pos_hypot(std::fabs(td), std::fabs(e));
            if (e2 == 0.0) mu -= e / ((td + (td > 0.0 ? h : -h)) / e);
            else mu -= e2 / (td + (td > 0.0 ? h : -h));
        }
        double x = diag[start] - mu;
        double z = sub[start];
        for (int k = start; k < end && z != 0.0; ++k) {
            double c, s;
            make_givens(x, z, c, s);
            double sdk = s * diag[k] + c * sub[k];
            double dkp1 = s * sub[k] + c * diag[k + 1];
            diag[k] = c * (c * diag[k] - s * sub[k]) - s * (c * sub[k] - s * diag[k + 1]);
            diag[k + 1] = s * sdk + c * dkp1;
            sub[k] = c * sdk - s * dkp1;
            if (k > start) sub[k - 1] = c * sub[k - 1] - s * z;
            x = sub[k];
            if (k < end - 1) {
                z = -s * sub[k + 1];
                sub[k + 1] = c * sub[k + 1];
            }
            for (int r = 0; r < 3; ++r) {
                double xi = Q[k * 3 + r], yi = Q[(k + 1) * 3 + r];
                Q[k * 3 + r] = c * xi - s * yi;
                Q[(k + 1) * 3 + r] = s * xi + c * yi;
            }
        }
    }
    int ok = iter <= maxIterations * n;
    if (ok) {
        for (int i = 0; i < n - 1; ++i) {
            int k = i;
            for (int j = i + 1; j < n; ++j)
                if (diag[j] < diag[k]) k = j;
            if (k != i) {
                std::swap(diag[i], diag[k]);
                for (int r = 0; r < 3; ++r) std::swap(Q[i * 3 + r], Q[k * 3 + r]);
            }
        }
    }
    for (int i = 0; i < 3; ++i) eval[i] = diag[i] * scale;
    for (int i = 0; i < 9; ++i) evec[i] = Q[i];
    return ok;
}

// Cyclic Jacobi in long double for the accuracy oracle.  Ascending order.
static void jacobi_ld(const long double A[3][3], long double eval[3], long double V[3][3]) {
    long double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { a[i][j] = A[i][j]; V[i][j] = (i == j) ? 1.0L : 0.0L; }
    for (int sweep = 0; sweep < 64; ++sweep) {
        long double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        long double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0L || off <= 1e-40L * dg) break;
        static const int P[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (int r = 0; r < 3; ++r) {
            int p = P[r][0], q = P[r][1];
            if (a[p][q] == 0.0L) continue;
            long double theta = (a[q][q] - a[p][p]) / (2.0L * a[p][q]);
            long double t = (theta >= 0 ? 1.0L : -1.0L) /
                            (fabsl(theta) + sqrtl(theta * theta + 1.0L));
            long double c = 1.0L / sqrtl(t * t + 1.0L), s = t * c;
            for (int k = 0; k < 3; ++k) {  // A <- A J
                long double akp = a[k][p], akq = a[k][q];
                a[k][p] = c * akp - s * akq;
                a[k][q] = s * akp + c * akq;
            }
            for (int k = 0; k < 3; ++k) {  // A <- J^T A
                long double apk = a[p][k], aqk = a[q][k];
                a[p][k] = c * apk - s * aqk;
                a[q][k] = s * apk + c * aqk;
            }
            for (int k = 0; k < 3; ++k) {
                long double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
    int order[3] = {0, 1, 2};
    std::sort(order, order + 3, [&](int i, int j) { return a[i][i] < a[j][j]; });
    long double W[3][3];
    for (int c = 0; c < 3; ++c) {
        eval[c] = a[order[c]][order[c]];
        for (int r = 0; r < 3; ++r) W[r][c] = V[r][order[c]];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) V[r][c] = W[r][c];
}

// ---------------------------------------------------------------------------
// One neighbourhood -> eigensystem (both modes)
// ---------------------------------------------------------------------------
struct Eig {
    int zero = 0;  // covariance isZero()
    int ok = 1;    // solver success
    double ev[3] = {0, 0, 0};
    double vec[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // column-major
};

static Eig eigensystem(const double* const X[3], const std::vector<uint64_t>& ids, int mode) {
    Eig r;
    const size_t n = ids.size();
    double B[3][3];
    if (mode == 0) {
        // computeCentroid: online mean
        double mean[3] = {0, 0, 0};
        uint64_t cnt = 0;
        for (uint64_t j : ids) {
            cnt++;
            for (int d = 0; d < 3; ++d) {
                double delta = X[d][j] - mean[d];
                double delta_n = delta / (double)cnt;
                mean[d] = mean[d] + delta_n;
            }
        }
        std::vector<double> A(3 * n);
        for (size_t k = 0; k < n; ++k)
            for (int d = 0; d < 3; ++d)
                A[d * n + k] = (double)(float)(X[d][ids[k]] - mean[d]);
        const double denom = (double)(size_t)(n - 1);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (size_t k = 0; k < n; ++k) s += A[i * n + k] * A[j * n + k];
                B[i][j] = s / denom;
            }
    } else {
        long double mean[3] = {0, 0, 0};
        for (uint64_t j : ids)
            for (int d = 0; d < 3; ++d) mean[d] += (long double)X[d][j];
        for (int d = 0; d < 3; ++d) mean[d] /= (long double)n;
        long double S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (uint64_t j : ids) {
            long double dv[3];
            for (int d = 0; d < 3; ++d) dv[d] = (long double)X[d][j] - mean[d];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) S[a][b] += dv[a] * dv[b];
        }
        long double denom = (long double)n - 1.0L;
        long double C[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                C[a][b] = S[a][b] / denom;
                B[a][b] = (double)C[a][b];
            }
        if (n == 1) {  // the reference divides 0 by n-1 = 0
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) B[a][b] = std::numeric_limits<double>::quiet_NaN();
        }
        bool zero = true;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                if (!(std::fabs(B[a][b]) <= 1e-12)) zero = false;
        r.zero = zero;
        if (zero) return r;
        if (n == 1) { r.ok = 0; return r; }
        long double ev[3], V[3][3];
        jacobi_ld(C, ev, V);
        // eigenvector signs follow the Eigen chain on the same matrix
        double cev[3], cvec[9];
        eigen_chain(B, cev, cvec);
        for (int c = 0; c < 3; ++c) {
            long double dot = 0;
            for (int rr = 0; rr < 3; ++rr) dot += V[rr][c] * (long double)cvec[c * 3 + rr];
            long double sg = dot < 0 ? -1.0L : 1.0L;
            r.ev[c] = (double)ev[c];
            for (int rr = 0; rr < 3; ++rr) r.vec[c * 3 + rr] = (double)(sg * V[rr][c]);
        }
        return r;
    }
    bool zero = true;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            if (!(std::fabs(B[a][b]) <= 1e-12)) zero = false;
    r.zero = zero;
    if (zero) return r;
    r.ok = eigen_chain(B, r.ev, r.vec);
    return r;
}

static int ndims_of(const nbg_stage_opts& o) {
    if (o.kind == NBG_STAGE_NORMAL) return 4;
    if (o.kind == NBG_STAGE_EIGENVALUES) return 3;
    return __builtin_popcount(o.feature_mask & NBG_FEAT_ALL);
}

// Per-point stage logic; returns the row exception code (0 = written).
static int project(const nbg_stage_opts& o, const Eig& e, size_t nnb, const double p[3],
                   double kopt, double ropt, double* out) {
    if (o.kind == NBG_STAGE_NORMAL) {
        if (nnb < 3) return NBG_ROW_TOO_FEW;
        if (e.zero) return NBG_ROW_ZERO_COV;
        if (!e.ok) return NBG_ROW_EIGEN_FAIL;
        double sum = e.ev[0] + e.ev[1] + e.ev[2];
        double curvature = sum ? std::fabs(e.ev[0] / sum) : 0;
        double nv[3] = {e.vec[0], e.vec[1], e.vec[2]};
        if (nv[0] == 0.0 && nv[1] == 0.0 && nv[2] == 0.0) return NBG_ROW_EIGEN_FAIL;
        if (o.has_viewpoint) {
            double dx = o.viewpoint[0] - p[0];
            double dy = o.viewpoint[1] - p[1];
            double dz = o.viewpoint[2] - p[2];
            double dot = dx * nv[0] + dy * nv[1] + dz * nv[2];
            if (dot < 0) for (double& v : nv) v = -v;
        } else if (o.always_up) {
            if (nv[2] < 0) for (double& v : nv) v = -v;
        }
        out[0] = nv[0];
        out[1] = nv[1];
        out[2] = nv[2];
        out[3] = curvature;
        return 0;
    }
    if (o.kind == NBG_STAGE_EIGENVALUES) {
        if (e.zero) return NBG_ROW_ZERO_COV;
        if (!e.ok) return NBG_ROW_EIGEN_FAIL;
        double ev[3] = {e.ev[0], e.ev[1], e.ev[2]};
        if (o.normalize) {
            double sum = ev[0] + ev[1] + ev[2];
            for (double& v : ev) v /= sum;
        }
        out[0] = ev[0];
        out[1] = ev[1];
        out[2] = ev[2];
        return 0;
    }
    // covariance features
    if (e.zero) return NBG_ROW_ZERO_COV;
    if (!e.ok) return NBG_ROW_EIGEN_FAIL;
    double lambda[3] = {std::max(e.ev[2], 0.0), std::max(e.ev[1], 0.0), std::max(e.ev[0], 0.0)};
    double sum = 0.0;
    sum = sum + lambda[0];
    sum = sum + lambda[1];
    sum = sum + lambda[2];
    if (lambda[0] == 0) return NBG_ROW_ZERO_LAMBDA;
    if (o.mode == NBG_MODE_SQRT) {
        for (double& v : lambda) v = std::sqrt(v);
    } else if (o.mode == NBG_MODE_NORMALIZED) {
        for (double& v : lambda) v = v / sum;
    }
    double v1[3], v2[3], v3[3];
    for (int i = 0; i < 3; ++i) {
        v1[i] = e.vec[2 * 3 + i];
        v2[i] = e.vec[1 * 3 + i];
        v3[i] = e.vec[0 * 3 + i];
    }
    int w = 0;
    for (int f = 0; f < NBG_NUM_FEATURES; ++f) {
        if (!(o.feature_mask & (1u << f))) continue;
        double val = 0.0;
        switch (1u << f) {
            case NBG_FEAT_LINEARITY: val = (lambda[0] - lambda[1]) / lambda[0]; break;
            case NBG_FEAT_PLANARITY: val = (lambda[1] - lambda[2]) / lambda[0]; break;
            case NBG_FEAT_SCATTERING: val = lambda[2] / lambda[0]; break;
            case NBG_FEAT_VERTICALITY: {
                double u[3], norm = 0;
                for (int i = 0; i < 3; ++i) {
                    u[i] = lambda[0] * std::fabs(v1[i]) + lambda[1] * std::fabs(v2[i]) +
                           lambda[2] * std::fabs(v3[i]);
                    norm += u[i] * u[i];
                }
                norm = std::sqrt(norm);
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
            case NBG_FEAT_DEMANTKEVERTICALITY: val = 1 - std::fabs(e.vec[0 * 3 + 2]); break;
            case NBG_FEAT_DENSITY: {
                double pi = 3.14159265;
                val = (kopt + 1.0) / ((4.0 / 3.0) * pi * std::pow(ropt, 3));
                break;
            }
        }
        out[w++] = val;
    }
    return 0;
}

template <class F>
static void parallel_rows(uint64_t n, int threads, F&& fn) {
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

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI (ctypes) — shared with oracle/ref_shim.cpp
// ---------------------------------------------------------------------------
using orc::KdTree;

struct OrcTree {
    KdTree t;
    std::vector<double> X, Y, Z;
};

// The port's backend of the shared consumer loops (consumers.hpp).
struct PortBackend {
    const OrcTree* h;
    uint64_t n() const { return h->t.n; }
    double coord(uint64_t i, int d) const { return d == 0 ? h->X[i] : d == 1 ? h->Y[i] : h->Z[i]; }
    void knn(uint64_t i, uint64_t k, std::vector<uint64_t>& ids, std::vector<double>& d2) const {
        const double q[3] = {h->X[i], h->Y[i], h->Z[i]};
        h->t.knn_search(q, k, ids, d2);
    }
    std::vector<uint64_t> neighbors(uint64_t i, uint64_t k) const {
        const double q[3] = {h->X[i], h->Y[i], h->Z[i]};
        std::vector<uint64_t> ids;
        h->t.neighbors(q, k, 1, ids);
        return ids;
    }
    uint64_t radius_count(uint64_t i, double r) const {
        const double q[3] = {h->X[i], h->Y[i], h->Z[i]};
        std::vector<uint64_t> ids;
        h->t.radius_neighbors(q, r, ids);
        return ids.size();
    }
    int cov_eigenvalues(const std::vector<uint64_t>& ids, int mode, double ev[3]) const {
        const double* X[3] = {h->X.data(), h->Y.data(), h->Z.data()};
        orc::Eig e = orc::eigensystem(X, ids, mode);
        if (e.zero) return NBG_ROW_ZERO_COV;
        if (!e.ok) return NBG_ROW_EIGEN_FAIL;
        for (int c = 0; c < 3; ++c) ev[c] = e.ev[c];
        return 0;
    }
    // JacobiSVD rank (MathUtils.cpp:197-208): singular values of the
    // symmetric covariance are |lambda|, counted when at or above
    // max(float(thresh) * sigma_max, DBL_MIN).  A one-point neighbourhood
    // (0/0 covariance) has no defined rank in the reference; 0 here.
    int rank(const std::vector<uint64_t>& ids, double thresh, int mode) const {
        if (ids.size() <= 1) return 0;
        const double* X[3] = {h->X.data(), h->Y.data(), h->Z.data()};
        orc::Eig e = orc::eigensystem(X, ids, mode);
        if (e.zero || !e.ok) return 0;
        double a[3] = {std::fabs(e.ev[0]), std::fabs(e.ev[1]), std::fabs(e.ev[2])};
        double smax = std::max(a[0], std::max(a[1], a[2]));
        double thr = std::max(smax * (double)(float)thresh, std::numeric_limits<double>::min());
        return (a[0] >= thr) + (a[1] >= thr) + (a[2] >= thr);
    }
    bool sym_eigenvalues(const double A[3][3], double ev[3]) const {
        double vec[9];
        return orc::eigen_chain(A, ev, vec) != 0;
    }
};

extern "C" {

const char* orc_impl_name(void) { return "port"; }

void* orc_tree_build(const double* x, const double* y, const double* z, uint64_t n) {
    OrcTree* h = new OrcTree();
    h->X.assign(x, x + n);
    h->Y.assign(y, y + n);
    h->Z.assign(z, z + n);
    h->t.c[0] = h->X.data();
    h->t.c[1] = h->Y.data();
    h->t.c[2] = h->Z.data();
    h->t.n = n;
    h->t.build();
    return h;
}

// the port's build is serial: the thread count changes nothing
void* orc_tree_build_t(const double* x, const double* y, const double* z, uint64_t n, int) {
    return orc_tree_build(x, y, z, n);
}

void orc_tree_free(void* h) { delete (OrcTree*)h; }

// KD3ImplT::neighbors; writes min(n,k) ids, returns that count.
uint64_t orc_tree_neighbors(void* hv, double qx, double qy, double qz, uint64_t k,
                            uint64_t stride, uint64_t* out) {
    OrcTree* h = (OrcTree*)hv;
    double q[3] = {qx, qy, qz};
    std::vector<uint64_t> ids;
    h->t.neighbors(q, k, stride, ids);
    std::copy(ids.begin(), ids.end(), out);
    return ids.size();
}

// Neighbour lists (reference order) of every point as query; rows of k1 ids.
void orc_all_neighbors(void* hv, uint64_t k, uint64_t* out, int threads) {
    OrcTree* h = (OrcTree*)hv;
    const uint64_t n = h->t.n;
    const uint64_t k1 = std::min<uint64_t>(n, k);
    orc::parallel_rows(n, threads, [&](uint64_t b, uint64_t e) {
        std::vector<uint64_t> ids;
        for (uint64_t i = b; i < e; ++i) {
            double q[3] = {h->X[i], h->Y[i], h->Z[i]};
            h->t.neighbors(q, k, 1, ids);
            std::copy(ids.begin(), ids.end(), out + i * k1);
        }
    });
}

uint64_t orc_tree_num_nodes(void* hv) { return ((OrcTree*)hv)->t.nodes.size(); }

// Tree export (preorder nodes) for the GPU replica's structural parity test.
void orc_tree_export(void* hv, uint64_t* vind, int64_t* child1, int64_t* child2,
                     int32_t* divfeat, double* divlow, double* divhigh, uint64_t* left,
                     uint64_t* right) {
    OrcTree* h = (OrcTree*)hv;
    std::copy(h->t.vind.begin(), h->t.vind.end(), vind);
    for (size_t i = 0; i < h->t.nodes.size(); ++i) {
        const orc::Node& nd = h->t.nodes[i];
        child1[i] = nd.child1;
        child2[i] = nd.child2;
        divfeat[i] = nd.divfeat;
        divlow[i] = nd.divlow;
        divhigh[i] = nd.divhigh;
        left[i] = nd.left;
        right[i] = nd.right;
    }
}

// Eigen chain on one matrix (row-major 3x3); returns success.
int orc_eigen_chain(const double* a, double* eval, double* evec_colmajor) {
    double A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = a[i * 3 + j];
    return orc::eigen_chain(A, eval, evec_colmajor);
}

// The whole per-point loop of one stage.  out_cols[d] are n-long double
// columns (dims in the stage's order); status[i] receives the row code.
// Returns 0, or -1 for invalid options.
int orc_run_stage(void* hv, const nbg_stage_opts* opts, const double* optimal_knn,
                  const double* optimal_radius, int mode, double** out_cols, uint8_t* status,
                  int threads) {
    OrcTree* h = (OrcTree*)hv;
    const nbg_stage_opts o = *opts;
    const uint64_t n = h->t.n;
    const int nd = orc::ndims_of(o);
    const double* X[3] = {h->X.data(), h->Y.data(), h->Z.data()};
    if (o.kind > NBG_STAGE_COVARIANCEFEATURES)
        return orc_consumers::run_consumer(PortBackend{h}, o, mode, out_cols, status, threads,
                                           [](uint64_t m, int th, auto&& fn) {
                                               orc::parallel_rows(m, th, fn);
                                           });
    if (o.kind < 1 || o.kind > 3) return -1;
    orc::parallel_rows(n, threads, [&](uint64_t b, uint64_t e) {
        std::vector<uint64_t> ids;
        double vals[NBG_MAX_DIMS];
        for (uint64_t i = b; i < e; ++i) {
            double q[3] = {X[0][i], X[1][i], X[2][i]};
            uint64_t k, stride = o.stride > 0 ? (uint64_t)o.stride : 1;
            double kopt_i = optimal_knn ? optimal_knn[i] : 0.0;
            double ropt_i = optimal_radius ? optimal_radius[i] : 0.0;
            if (o.use_radius && !(o.kind == NBG_STAGE_COVARIANCEFEATURES && o.optimized)) {
                // NormalFilter.cpp:149-150; EigenvaluesFilter.cpp:121-134;
                // CovarianceFeaturesFilter.cpp:216-225
                h->t.radius_neighbors(q, o.radius, ids);
                if (o.kind != NBG_STAGE_NORMAL && ids.size() < (size_t)o.min_k) {
                    status[i] = NBG_ROW_RADIUS_FEW;
                    continue;
                }
                orc::Eig eg = orc::eigensystem(X, ids, mode);
                int code = orc::project(o, eg, ids.size(), q, kopt_i, ropt_i, vals);
                status[i] = (uint8_t)code;
                if (code == 0)
                    for (int d = 0; d < nd; ++d) out_cols[d][i] = vals[d];
                continue;
            }
            if (o.kind == NBG_STAGE_NORMAL) {
                k = (uint64_t)(o.knn + 1);
                stride = 1;
            } else if (o.kind == NBG_STAGE_COVARIANCEFEATURES && o.optimized) {
                k = (uint64_t)optimal_knn[i];
                stride = 1;
            } else {
                k = (uint64_t)(o.knn + 1);
            }
            h->t.neighbors(q, k, stride, ids);
            orc::Eig eg = orc::eigensystem(X, ids, mode);
            double kopt = optimal_knn ? optimal_knn[i] : 0.0;
            double ropt = optimal_radius ? optimal_radius[i] : 0.0;
            int code = orc::project(o, eg, ids.size(), q, kopt, ropt, vals);
            status[i] = (uint8_t)code;
            if (code == 0)
                for (int d = 0; d < nd; ++d) out_cols[d][i] = vals[d];
        }
    });
    return 0;
}

}  // extern "C"

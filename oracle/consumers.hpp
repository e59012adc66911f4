// consumers.hpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// The per-point loops of the other consumers of the KD3 index, restated once
// and shared by the FP64 port (nbg_oracle.cpp) and the reference shim
// (ref_shim.cpp), which differ only in the backend: the search (the port's
// nanoflann restatement or the reference's vendored nanoflann) and the
// eigen / SVD solvers (the port's Eigen-chain restatement or the reference's
// vendored Eigen).  Each loop follows the reference's filter:
//   filters/ApproximateCoplanarFilter.cpp:80-114
//   filters/EstimateRankFilter.cpp:76-84 with MathUtils.cpp:197-208
//   filters/NNDistanceFilter.cpp:108-138
//   filters/OptimalNeighborhoodFilter.cpp:71-163
//   filters/LOFFilter.cpp:66-139
//   filters/OutlierFilter.cpp:75-229
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "../include/nbg_b200.h"

namespace orc_consumers {

// Backend B supplies:
//   uint64_t n() const;  double coord(uint64_t i, int d) const;
//   void knn(uint64_t i, uint64_t k, std::vector<uint64_t>& ids,
//            std::vector<double>& d2) const;   // KD3Impl::knnSearch: the
//                                             // caller's k-sized vectors,
//                                             // min(n, k) of them filled
//   std::vector<uint64_t> neighbors(uint64_t i, uint64_t k) const;
//   uint64_t radius_count(uint64_t i, double r) const;
//   int cov_eigenvalues(const std::vector<uint64_t>& ids, int mode, double ev[3]) const;
//       // 0, NBG_ROW_ZERO_COV or NBG_ROW_EIGEN_FAIL (computeCovariance + solver)
//   int rank(const std::vector<uint64_t>& ids, double thresh, int mode) const;
//   bool sym_eigenvalues(const double A[3][3], double ev[3]) const;   // ascending
// PR: parallel_rows(n, threads, fn(begin, end)).
template <class B, class PR>
int run_consumer(const B& b, const nbg_stage_opts& o, int mode, double** out, uint8_t* status,
                 int threads, PR&& parallel_rows) {
    const uint64_t n = b.n();
    if (o.kind == NBG_STAGE_APPROXIMATECOPLANAR || o.kind == NBG_STAGE_ESTIMATERANK) {
        if (o.knn < 1) return -1;
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; ++i) {
                std::vector<uint64_t> ids = b.neighbors(i, (uint64_t)o.knn);
                if (o.kind == NBG_STAGE_ESTIMATERANK) {
                    out[0][i] = (double)b.rank(ids, o.thresh1, mode);
                    status[i] = 0;
                    continue;
                }
                double ev[3];
                int code = b.cov_eigenvalues(ids, mode, ev);
                status[i] = (uint8_t)code;
                if (code) continue;
                out[0][i] = (ev[1] > o.thresh1 * ev[0] && o.thresh2 * ev[1] > ev[2]) ? 1.0 : 0.0;
            }
        });
        return 0;
    }
    if (o.kind == NBG_STAGE_NNDISTANCE) {
        const uint64_t k = (uint64_t)o.knn + 1;
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            std::vector<uint64_t> ids;
            std::vector<double> d2;
            for (uint64_t i = lo; i < hi; ++i) {
                ids.assign(k, 0);
                d2.assign(k, 0.0);
                b.knn(i, k, ids, d2);
                double val;
                if (o.mode == 0) {
                    val = std::sqrt(d2[k - 1]);
                } else {
                    val = 0;
                    for (size_t j = 1; j < k; ++j) val += std::sqrt(d2[j]);
                    val /= (k - 1);
                }
                out[0][i] = val;
                status[i] = 0;
            }
        });
        return 0;
    }
    if (o.kind == NBG_STAGE_OPTIMALNEIGHBORHOOD) {
        const uint64_t kmin = (uint64_t)o.min_k, kmax = (uint64_t)o.knn;
        if (kmin < 1 || kmin > kmax) return -1;
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            std::vector<uint64_t> ids;
            std::vector<double> d2;
            for (uint64_t i = lo; i < hi; ++i) {
                ids.assign(kmax, 0);
                d2.assign(kmax, 0.0);
                b.knn(i, kmax, ids, d2);
                double minentropy = std::numeric_limits<double>::max();
                uint64_t kopt = 0;
                double ropt = 0.0;
                double mx = 0, my = 0, mz = 0;
                double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                int code = 0;
                for (uint64_t k = 0; k < kmax && !code; ++k) {
                    const uint64_t q = ids[k];
                    double dx = b.coord(q, 0) - mx;
                    double dy = b.coord(q, 1) - my;
                    double dz = b.coord(q, 2) - mz;
                    double nn = double(k + 1);
                    mx += dx / nn;
                    my += dy / nn;
                    mz += dz / nn;
                    double s = (nn - 1) / nn;
                    M[0][0] = M[0][0] + s * dx * dx;
                    M[1][1] = M[1][1] + s * dy * dy;
                    M[2][2] = M[2][2] + s * dz * dz;
                    M[1][0] = M[0][1] = M[0][1] + s * dx * dy;
                    M[2][0] = M[0][2] = M[0][2] + s * dx * dz;
                    M[1][2] = M[2][1] = M[2][1] + s * dy * dz;
                    if (k + 1 < kmin) continue;
                    double A[3][3];
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) A[r][c] = M[r][c] / (nn - 1);
                    double ev[3];
                    if (!b.sym_eigenvalues(A, ev)) {
                        code = NBG_ROW_EIGEN_FAIL;
                        break;
                    }
                    double l[3] = {std::max(ev[2], 0.0), std::max(ev[1], 0.0), std::max(ev[0], 0.0)};
                    double sum = 0.0;
                    for (double v : l) sum += v;
                    for (double& v : l) v = v / sum;
                    double entropy = -(l[2] * std::log(l[2]) + l[1] * std::log(l[1]) +
                                       l[0] * std::log(l[0]));
                    if (entropy < minentropy) {
                        minentropy = entropy;
                        kopt = k + 1;
                        ropt = d2[k];
                    }
                }
                status[i] = (uint8_t)code;
                if (code) continue;
                out[0][i] = (double)kopt;
                out[1][i] = std::sqrt(ropt);
            }
        });
        return 0;
    }
    if (o.kind == NBG_STAGE_LOF) {
        const uint64_t k = (uint64_t)o.knn + 1;
        std::vector<uint64_t> mid(n * k);
        std::vector<double> md(n * k), kdist(n), lrd(n);
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            std::vector<uint64_t> ids;
            std::vector<double> d2;
            for (uint64_t i = lo; i < hi; ++i) {
                ids.assign(k, 0);
                d2.assign(k, 0.0);
                b.knn(i, k, ids, d2);
                for (uint64_t j = 0; j < k; ++j) {
                    mid[i * k + j] = ids[j];
                    md[i * k + j] = std::sqrt(d2[j]);
                }
                kdist[i] = std::sqrt(d2[k - 1]);
                out[0][i] = kdist[i];
                status[i] = 0;
            }
        });
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; ++i) {
                double M1 = 0.0;
                uint64_t c = 0;
                for (uint64_t j = 0; j < k; ++j) {
                    double kd = kdist[mid[i * k + j]];
                    double reach = (std::max)(kd, md[i * k + j]);
                    M1 += (reach - M1) / ++c;
                }
                lrd[i] = 1.0 / M1;
                out[1][i] = lrd[i];
            }
        });
        parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; ++i) {
                double M1 = 0.0;
                uint64_t c = 0;
                for (uint64_t j = 0; j < k; ++j) {
                    double ratio = lrd[mid[i * k + j]] / lrd[i];
                    M1 += (ratio - M1) / ++c;
                }
                out[2][i] = M1;
            }
        });
        return 0;
    }
    if (o.kind == NBG_STAGE_OUTLIER) {
        std::vector<char> outlier(n, 0);
        if (o.mode == 1) {
            parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
                for (uint64_t i = lo; i < hi; ++i)
                    outlier[i] = !(b.radius_count(i, o.radius) > (uint64_t)o.min_k);
            });
        } else {
            const uint64_t count = (uint64_t)o.knn + 1;
            std::vector<double> distances(n, 0.0);
            parallel_rows(n, threads, [&](uint64_t lo, uint64_t hi) {
                std::vector<uint64_t> ids;
                std::vector<double> d2;
                for (uint64_t i = lo; i < hi; ++i) {
                    ids.assign(count, 0);
                    d2.assign(count, 0.0);
                    b.knn(i, count, ids, d2);
                    for (size_t j = 1; j < count; ++j) {
                        double delta = std::sqrt(d2[j]) - distances[i];
                        distances[i] += (delta / j);
                    }
                }
            });
            size_t cnt = 0;
            double M1 = 0.0, M2 = 0.0;
            for (double d : distances) {
                size_t n1 = cnt;
                cnt++;
                double delta = d - M1;
                double delta_n = delta / cnt;
                M1 += delta_n;
                M2 += delta * delta_n * n1;
            }
            double stdev = std::sqrt(M2 / (cnt - 1.0));
            double threshold = M1 + o.thresh1 * stdev;
            for (uint64_t i = 0; i < n; ++i) outlier[i] = !(distances[i] < threshold);
        }
        uint64_t nout = 0;
        for (char c : outlier) nout += c != 0;
        for (uint64_t i = 0; i < n; ++i) status[i] = 0;
        if (nout && nout < n)
            for (uint64_t i = 0; i < n; ++i)
                if (outlier[i]) out[0][i] = (double)o.label;
        return (int)std::min<uint64_t>(nout, 0x7FFFFFFF);
    }
    return -1;
}

}  // namespace orc_consumers

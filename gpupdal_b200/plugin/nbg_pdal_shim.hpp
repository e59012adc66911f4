// nbg_pdal_shim.hpp — the PDAL-independent part of the PDAL plugin
// (nbg_pdal_plugin.cpp): which stages it registers and under which options,
// the option object handed to nbg_filter_create, the exact recovery of a
// view's raw LAS integers from its double coordinates, and one stage run
// through the C ABI.  Header-only, so the plugin and its tests share it.
//
// PDAL resolves a stage type against its built-in (static) stages before it
// looks for a plugin library, and registering a plugin never replaces an
// existing name (pdal/PluginManager.cpp:357-375, pdal/PluginManager.hpp:
// 111-122).  A plugin therefore cannot take over "filters.normal"; it
// registers "filters.b200normal" and the like, each accepting exactly the
// options of the filter it stands for, so a pipeline moves to it by renaming
// the stage types and nothing else.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "nbg_b200.h"

namespace nbg_pdal {

struct StageSpec {
    const char* plugin_type;  // registered name (libpdal_plugin_filter_<suffix>.so)
    const char* base_type;    // the reference filter whose options it takes
    std::vector<const char*> options;
};

// The reference filters' options (their addArgs): NormalFilter.cpp:85-97,
// EigenvaluesFilter.cpp:77-87, CovarianceFeaturesFilter.cpp:102-113,
// ApproximateCoplanarFilter.cpp:66-71, EstimateRankFilter.cpp:66-70,
// NNDistanceFilter.cpp:95-99, OptimalNeighborhoodFilter.cpp:62-66,
// LOFFilter.cpp:62-65, OutlierFilter.cpp:62-71.
inline const std::vector<StageSpec>& stages() {
    static const std::vector<StageSpec> s = {
        {"filters.b200normal", "filters.normal", {"knn", "radius", "viewpoint", "always_up", "refine"}},
        {"filters.b200eigenvalues", "filters.eigenvalues", {"knn", "normalize", "stride", "radius", "min_k"}},
        {"filters.b200covariancefeatures", "filters.covariancefeatures",
         {"knn", "threads", "feature_set", "stride", "radius", "min_k", "mode", "optimized"}},
        {"filters.b200approximatecoplanar", "filters.approximatecoplanar", {"knn", "thresh1", "thresh2"}},
        {"filters.b200estimaterank", "filters.estimaterank", {"knn", "thresh"}},
        {"filters.b200nndistance", "filters.nndistance", {"mode", "k"}},
        {"filters.b200optimalneighborhood", "filters.optimalneighborhood", {"min_k", "max_k"}},
        {"filters.b200lof", "filters.lof", {"minpts"}},
        {"filters.b200outlier", "filters.outlier",
         {"method", "min_k", "radius", "mean_k", "multiplier", "class"}},
    };
    return s;
}

inline const StageSpec* find_stage(const std::string& plugin_type) {
    for (const auto& s : stages())
        if (plugin_type == s.plugin_type) return &s;
    return nullptr;
}

// The options the user set, as the JSON object nbg_filter_create parses
// (every value as a JSON string: the stage layer reads values as text, as
// ProgramArgs does).
inline std::string options_json(const std::vector<std::pair<std::string, std::string>>& set) {
    std::string o = "{";
    for (size_t i = 0; i < set.size(); ++i) {
        if (i) o += ",";
        auto quote = [&](const std::string& v) {
            o += '"';
            for (char c : v) {
                if (c == '"' || c == '\\') {
                    o += '\\';
                    o += c;
                } else if ((unsigned char)c < 0x20) {
                    char b[8];
                    std::snprintf(b, sizeof b, "\\u%04x", (unsigned)(unsigned char)c);
                    o += b;
                } else {
                    o += c;
                }
            }
            o += '"';
        };
        quote(set[i].first);
        o += ":";
        quote(set[i].second);
    }
    return o + "}";
}

// raw[i] such that fl(fl(raw*scale) + offset) == v[i] bit for bit, the way a
// LAS reader forms the double; false (and the first offending index) when a
// coordinate is not of that form or its raw value leaves int32.
inline bool recover_raw(const double* v, uint64_t n, double scale, double offset, int32_t* raw,
                        uint64_t* bad) {
    for (uint64_t i = 0; i < n; ++i) {
        const double r = std::nearbyint((v[i] - offset) / scale);
        if (!(r >= -2147483648.0 && r <= 2147483647.0)) {
            if (bad) *bad = i;
            return false;
        }
        const int32_t k = (int32_t)r;
        volatile double p = (double)k * scale;  // two roundings, as the reader
        const double back = p + offset;
        if (std::memcmp(&back, &v[i], sizeof(double)) != 0) {
            if (bad) *bad = i;
            return false;
        }
        raw[i] = k;
    }
    return true;
}

// One stage of `base_type` over one cloud: x/y/z doubles (the view's), the
// scale/offset they came from, outputs as dims columns of n doubles (rows the
// reference skips keep their values).  OptimalKNN / OptimalRadius columns
// may be null.  Returns NBG_OK, or an NBG_ERR_* with `err` holding the
// message the reference would throw; `log` receives the stage's log lines.
inline int run_stage(nbg_context* ctx, const char* base_type, const std::string& options,
                     const double* x, const double* y, const double* z, uint64_t n,
                     const double scale[3], const double offset[3], const double* optimal_knn,
                     const double* optimal_radius, std::vector<double*>& columns,
                     std::string& log, std::string& err, nbg_run_stats* stats_out = nullptr) {
    char ebuf[1024] = {0};
    nbg_filter* f = nullptr;
    int rc = nbg_filter_create(base_type, options.c_str(), optimal_knn != nullptr,
                               optimal_radius != nullptr, &f, ebuf, sizeof ebuf);
    if (rc) {
        err = ebuf;
        return rc;
    }
    struct Guard {
        nbg_filter* f;
        nbg_tile* t = nullptr;
        nbg_context* c;
        ~Guard() {
            if (t) nbg_tile_free(c, t);
            nbg_filter_free(f);
        }
    } g{f, nullptr, ctx};
    nbg_stage_opts o;
    rc = nbg_filter_options(f, &o);
    if (rc) {
        err = std::string(base_type) + ": stride * (knn + 1) above 65 is not supported here";
        return rc;
    }
    std::vector<int32_t> raw(3 * n);
    const double* c[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
        uint64_t bad = 0;
        if (!recover_raw(c[d], n, scale[d], offset[d], raw.data() + d * n, &bad)) {
            err = std::string(base_type) + ": point " + std::to_string(bad) +
                  " is not a raw integer times the scale plus the offset";
            return NBG_ERR_UNSUPPORTED;
        }
    }
    rc = nbg_tile_upload(ctx, raw.data(), raw.data() + n, raw.data() + 2 * n, n, scale, offset, 0,
                         nullptr, &g.t);
    if (rc) {
        err = nbg_last_error(ctx);
        return rc;
    }
    nbg_columns col{};
    col.base = nullptr;
    col.point_stride = 8;
    col.on_device = 0;
    char names[512];
    nbg_filter_dims(f, names, sizeof names);
    int nd = names[0] ? 1 : 0;
    for (char* p = names; *p; ++p) nd += *p == ',';
    if ((int)columns.size() != nd || nd > NBG_MAX_DIMS) {
        err = "output column count does not match the stage";
        return NBG_ERR_INVALID;
    }
    // columns may be anywhere: one nbg_columns per stage needs one base, so
    // the offsets are taken relative to the first column
    col.base = nd ? columns[0] : nullptr;
    col.ndims = nd;
    for (int d = 0; d < nd; ++d)
        col.offset[d] = (int64_t)((const char*)columns[d] - (const char*)columns[0]);
    uint32_t cap = (uint32_t)std::min<uint64_t>(n + 1024, 1u << 24), nex = 0;
    std::vector<nbg_row_exception> ex(cap);
    nbg_run_stats stats{};
    rc = nbg_run(ctx, g.t, &o, 1, &col, optimal_knn, optimal_radius, 0, ex.data(), cap, &nex, &stats,
                 nullptr);
    if (rc) {
        err = nbg_last_error(ctx);
        return rc;
    }
    rc = nbg_filter_report(f, ex.data(), std::min(nex, cap), 0, ebuf, sizeof ebuf);
    nbg_filter_outcome(f, &stats);
    log = nbg_filter_log(f);
    if (stats_out) *stats_out = stats;
    if (rc) {
        err = ebuf;
        return rc;
    }
    return NBG_OK;
}

}  // namespace nbg_pdal

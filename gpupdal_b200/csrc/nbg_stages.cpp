// nbg_stages.cpp — the stage layer above the C ABI: PDAL pipeline JSON and
// the options, dimensions, checks and per-row messages of filters.normal,
// filters.eigenvalues and filters.covariancefeatures, and of the other
// consumers of the same index (filters.approximatecoplanar, estimaterank,
// nndistance, optimalneighborhood, lof, outlier).
//
// Mirrors, for a drop-in of an existing pipeline:
//   NormalFilter::addArgs/addDimensions/prepared      filters/NormalFilter.cpp:85-138
//   NormalFilter::compute (skip log lines)            filters/NormalFilter.cpp:140-160
//   math::findNormal messages                         pdal/private/MathUtils.cpp:572-611
//   EigenvaluesFilter::addArgs/prepared/filter        filters/EigenvaluesFilter.cpp:77-172
//   CovarianceFeaturesFilter::addArgs/addDimensions/prepared/setDimensionality
//                                                     filters/CovarianceFeaturesFilter.cpp:71-262
//   ProgramArgs value errors                          pdal/util/ProgramArgs.hpp:415-435
// Option values come from the stage's JSON object: numbers, booleans or the
// strings PDAL's ProgramArgs would parse.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/nbg_b200.h"

namespace {

// ---------------------------------------------------------------------------
// JSON (the subset pipelines use)
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0;
    std::string str;  // String; for Number also the literal text
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json* get(const std::string& k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct Parser {
    const char* p;
    const char* end;
    std::string err;
    void ws() {
        while (p < end && std::isspace((unsigned char)*p)) ++p;
    }
    bool fail(const std::string& m) {
        if (err.empty()) err = m;
        return false;
    }
    bool lit(const char* s) {
        size_t n = std::strlen(s);
        if ((size_t)(end - p) >= n && std::strncmp(p, s, n) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    bool string(std::string& out) {
        if (p >= end || *p != '"') return fail("expected a string");
        ++p;
        out.clear();
        while (p < end && *p != '"') {
            char c = *p++;
            if (c == '\\') {
                if (p >= end) return fail("bad escape");
                char e = *p++;
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (end - p < 4) return fail("bad \\u escape");
                        unsigned v = (unsigned)std::strtoul(std::string(p, 4).c_str(), nullptr, 16);
                        p += 4;
                        if (v < 0x80) out += (char)v;
                        else if (v < 0x800) {
                            out += (char)(0xC0 | (v >> 6));
                            out += (char)(0x80 | (v & 0x3F));
                        } else {
                            out += (char)(0xE0 | (v >> 12));
                            out += (char)(0x80 | ((v >> 6) & 0x3F));
                            out += (char)(0x80 | (v & 0x3F));
                        }
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (p >= end) return fail("unterminated string");
        ++p;
        return true;
    }
    bool value(Json& v, int depth = 0) {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (p >= end) return fail("unexpected end of JSON");
        if (*p == '{') {
            ++p;
            v.kind = Json::Object;
            ws();
            if (p < end && *p == '}') {
                ++p;
                return true;
            }
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (p >= end || *p != ':') return fail("expected ':'");
                ++p;
                Json c;
                if (!value(c, depth + 1)) return false;
                v.obj.emplace_back(k, std::move(c));
                ws();
                if (p < end && *p == ',') {
                    ++p;
                    continue;
                }
                if (p < end && *p == '}') {
                    ++p;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (*p == '[') {
            ++p;
            v.kind = Json::Array;
            ws();
            if (p < end && *p == ']') {
                ++p;
                return true;
            }
            for (;;) {
                Json c;
                if (!value(c, depth + 1)) return false;
                v.arr.push_back(std::move(c));
                ws();
                if (p < end && *p == ',') {
                    ++p;
                    continue;
                }
                if (p < end && *p == ']') {
                    ++p;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (*p == '"') {
            v.kind = Json::String;
            return string(v.str);
        }
        if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
            return true;
        }
        if (lit("false")) {
            v.kind = Json::Bool;
            return true;
        }
        if (lit("null")) return true;
        const char* s = p;
        while (p < end && (std::isdigit((unsigned char)*p) || *p == '-' || *p == '+' || *p == '.' ||
                           *p == 'e' || *p == 'E'))
            ++p;
        if (p == s) return fail("unexpected character in JSON");
        v.kind = Json::Number;
        v.str.assign(s, p);
        char* e = nullptr;
        v.num = std::strtod(v.str.c_str(), &e);
        if (!e || *e) return fail("bad number");
        return true;
    }
};

bool parse_json(const char* text, Json& out, std::string& err) {
    Parser ps{text, text + std::strlen(text), {}};
    if (!ps.value(out)) {
        err = ps.err;
        return false;
    }
    ps.ws();
    if (ps.p != ps.end) {
        err = "trailing characters after JSON";
        return false;
    }
    return true;
}

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

// The text ProgramArgs would have parsed for an option.
std::string raw_text(const Json& v) {
    switch (v.kind) {
        case Json::String: return v.str;
        case Json::Number: return v.str;
        case Json::Bool: return v.b ? "true" : "false";
        default: return "";
    }
}

struct ArgError {
    std::string msg;
};

int64_t arg_int(const Json& v, const std::string& name) {
    const std::string s = trim(raw_text(v));
    char* e = nullptr;
    long long x = std::strtoll(s.c_str(), &e, 10);
    if (s.empty() || !e || *e) throw ArgError{"Invalid value '" + s + "' for argument '" + name + "'."};
    return x;
}

double arg_double(const Json& v, const std::string& name) {
    const std::string s = trim(raw_text(v));
    char* e = nullptr;
    double x = std::strtod(s.c_str(), &e);
    if (s.empty() || !e || *e) throw ArgError{"Invalid value '" + s + "' for argument '" + name + "'."};
    return x;
}

bool arg_bool(const Json& v, const std::string& name) {
    if (v.kind == Json::Bool) return v.b;
    const std::string s = lower(trim(raw_text(v)));
    if (s == "true" || s == "1") return true;
    if (s == "false" || s == "0") return false;
    throw ArgError{"Invalid value '" + raw_text(v) + "' for argument '" + name + "'."};
}

std::vector<std::string> arg_list(const Json& v) {
    std::vector<std::string> out;
    if (v.kind == Json::Array) {
        for (auto& e : v.arr) out.push_back(raw_text(e));
    } else {
        // a single string may hold a comma-separated list
        std::stringstream ss(raw_text(v));
        std::string item;
        while (std::getline(ss, item, ',')) out.push_back(item);
    }
    return out;
}

// Viewpoint as WKT ("POINT (x y z)", "POINT Z (x y z)", "POINT (x y)") or
// GeoJSON ({"type": "Point", "coordinates": [x, y, z]}, as an object or text).
bool parse_point(const Json& v, double xyz[3]) {
    xyz[0] = xyz[1] = xyz[2] = 0.0;
    const Json* coords = nullptr;
    Json tmp;
    if (v.kind == Json::Object) {
        coords = v.get("coordinates");
    } else if (v.kind == Json::String) {
        const std::string s = trim(v.str);
        if (!s.empty() && s[0] == '{') {
            std::string err;
            if (!parse_json(s.c_str(), tmp, err)) return false;
            coords = tmp.get("coordinates");
        } else {
            const std::string u = lower(s);
            if (u.compare(0, 5, "point") != 0) return false;
            size_t a = s.find('('), b = s.rfind(')');
            if (a == std::string::npos || b == std::string::npos || b < a) return false;
            std::stringstream ss(s.substr(a + 1, b - a - 1));
            double c[3] = {0, 0, 0};
            int k = 0;
            while (k < 3 && (ss >> c[k])) ++k;
            if (k < 2) return false;
            for (int d = 0; d < 3; ++d) xyz[d] = c[d];
            return true;
        }
    }
    if (!coords || coords->kind != Json::Array || coords->arr.size() < 2) return false;
    for (size_t d = 0; d < 3 && d < coords->arr.size(); ++d) {
        if (coords->arr[d].kind != Json::Number) return false;
        xyz[d] = coords->arr[d].num;
    }
    return true;
}

const char* kFeatureNames[NBG_NUM_FEATURES] = {
    "Linearity",    "Planarity",     "Scattering",      "Verticality",
    "Omnivariance", "Anisotropy",    "Eigenentropy",    "EigenvalueSum",
    "SurfaceVariation", "DemantkeVerticality", "Density"};

}  // namespace

struct nbg_filter {
    std::string type;
    nbg_stage_opts opts{};
    std::vector<std::string> dims;  // registered output dimensions, in order
    std::string log;                // lines the stage logged (warnings, skips)
    bool radius_set = false;
    double radius = 0.0;
    int64_t min_k = 3;
};

struct nbg_pipeline {
    std::vector<std::string> types;
    std::vector<std::string> options;  // each stage's options as JSON text
};

namespace {

std::string to_json(const Json& v) {
    std::ostringstream o;
    switch (v.kind) {
        case Json::Null: o << "null"; break;
        case Json::Bool: o << (v.b ? "true" : "false"); break;
        case Json::Number: o << v.str; break;
        case Json::String: {
            o << '"';
            for (char c : v.str) {
                if (c == '"' || c == '\\') o << '\\' << c;
                else if (c == '\n') o << "\\n";
                else o << c;
            }
            o << '"';
            break;
        }
        case Json::Array: {
            o << '[';
            for (size_t i = 0; i < v.arr.size(); ++i) o << (i ? "," : "") << to_json(v.arr[i]);
            o << ']';
            break;
        }
        case Json::Object: {
            o << '{';
            for (size_t i = 0; i < v.obj.size(); ++i) {
                Json k;
                k.kind = Json::String;
                k.str = v.obj[i].first;
                o << (i ? "," : "") << to_json(k) << ':' << to_json(v.obj[i].second);
            }
            o << '}';
            break;
        }
    }
    return o.str();
}

void copy_err(char* err, size_t len, const std::string& msg) {
    if (!err || !len) return;
    std::snprintf(err, len, "%s", msg.c_str());
}

// Options every stage accepts and this layer does not use.
bool common_option(const std::string& k) {
    static const char* names[] = {"type", "tag", "inputs", "user_data", "log", "option_file",
                                  "where", "where_merge"};
    for (const char* n : names)
        if (k == n) return true;
    return false;
}

}  // namespace

extern "C" int nbg_filter_create(const char* type, const char* options_json, int32_t has_optimal_knn,
                                 int32_t has_optimal_radius, nbg_filter** out, char* err,
                                 size_t err_len) {
    if (!type || !out) return NBG_ERR_INVALID;
    *out = nullptr;
    Json o;
    std::string perr;
    if (options_json && *options_json && !parse_json(options_json, o, perr)) {
        copy_err(err, err_len, std::string(type) + ": options are not valid JSON: " + perr);
        return NBG_ERR_INVALID;
    }
    if (o.kind == Json::Null) o.kind = Json::Object;
    if (o.kind != Json::Object) {
        copy_err(err, err_len, std::string(type) + ": options must be a JSON object");
        return NBG_ERR_INVALID;
    }
    std::unique_ptr<nbg_filter> f(new nbg_filter());
    f->type = type;
    nbg_stage_opts& s = f->opts;
    s.stride = 1;
    const std::string t = type;
    auto has = [&](const char* k) { return o.get(k) != nullptr; };
    try {
        std::vector<std::string> allowed;
        if (t == "filters.normal") {
            allowed = {"knn", "radius", "viewpoint", "always_up", "refine"};
            s.kind = NBG_STAGE_NORMAL;
            s.knn = 8;
            s.always_up = 1;
            if (has("knn")) s.knn = (int32_t)arg_int(*o.get("knn"), "knn");
            if (has("radius")) {
                f->radius = arg_double(*o.get("radius"), "radius");
                f->radius_set = true;
            }
            if (has("viewpoint")) {
                if (!parse_point(*o.get("viewpoint"), s.viewpoint))
                    throw ArgError{"Invalid value '" + raw_text(*o.get("viewpoint")) +
                                   "' for argument 'viewpoint'."};
                s.has_viewpoint = 1;
            }
            if (has("always_up")) s.always_up = arg_bool(*o.get("always_up"), "always_up");
            if (has("refine")) s.refine = arg_bool(*o.get("refine"), "refine");
            f->dims = {"NormalX", "NormalY", "NormalZ", "Curvature"};
            // prepared()
            if (s.always_up && s.has_viewpoint) {
                f->log += "Viewpoint provided. Ignoring always_up = TRUE.\n";
                s.always_up = 0;
            }
            if (f->radius_set && has("knn")) throw ArgError{"Cannot set both knn and radius."};
        } else if (t == "filters.eigenvalues") {
            allowed = {"knn", "normalize", "stride", "radius", "min_k"};
            s.kind = NBG_STAGE_EIGENVALUES;
            s.knn = 8;
            if (has("knn")) s.knn = (int32_t)arg_int(*o.get("knn"), "knn");
            if (has("normalize")) s.normalize = arg_bool(*o.get("normalize"), "normalize");
            if (has("stride")) s.stride = (int32_t)arg_int(*o.get("stride"), "stride");
            if (has("radius")) {
                f->radius = arg_double(*o.get("radius"), "radius");
                f->radius_set = true;
            }
            if (has("min_k")) f->min_k = arg_int(*o.get("min_k"), "min_k");
            f->dims = {"Eigenvalue0", "Eigenvalue1", "Eigenvalue2"};
            if (f->radius_set) {
                f->log += "Radius has been set. Ignoring knn and stride values.\n";
                if (f->radius <= 0.0) f->log += "Radius must be greater than 0.\n";
            } else {
                f->log += "No radius specified. Proceeding with knn and stride, but ignoring min_k.\n";
            }
        } else if (t == "filters.covariancefeatures") {
            allowed = {"knn", "threads", "feature_set", "stride", "radius", "min_k", "mode",
                       "optimized"};
            s.kind = NBG_STAGE_COVARIANCEFEATURES;
            s.knn = 10;
            s.mode = NBG_MODE_SQRT;
            if (has("knn")) s.knn = (int32_t)arg_int(*o.get("knn"), "knn");
            if (has("threads")) (void)arg_int(*o.get("threads"), "threads");
            if (has("stride")) s.stride = (int32_t)arg_int(*o.get("stride"), "stride");
            if (has("radius")) {
                f->radius = arg_double(*o.get("radius"), "radius");
                f->radius_set = true;
            }
            if (has("min_k")) f->min_k = arg_int(*o.get("min_k"), "min_k");
            if (has("mode")) {
                const std::string m = lower(trim(raw_text(*o.get("mode"))));
                if (m == "raw") s.mode = NBG_MODE_RAW;
                else if (m == "sqrt") s.mode = NBG_MODE_SQRT;
                else if (m == "normalized") s.mode = NBG_MODE_NORMALIZED;
                else throw ArgError{"Invalid value '" + raw_text(*o.get("mode")) +
                                    "' for argument 'mode'."};
            }
            if (has("optimized")) s.optimized = arg_bool(*o.get("optimized"), "optimized");
            // addDimensions(): feature names, case-insensitive and trimmed
            std::vector<std::string> fs = {"dimensionality"};
            if (has("feature_set")) fs = arg_list(*o.get("feature_set"));
            uint32_t mask = 0;
            std::vector<int> order;
            auto add = [&](int b) {
                if (!(mask & (1u << b))) order.push_back(b);
                mask |= 1u << b;
            };
            for (auto& raw : fs) {
                const std::string n = lower(trim(raw));
                if (n == "dimensionality") {
                    for (int b = 0; b < 4; ++b) add(b);
                } else if (n == "all") {
                    for (int b = 0; b < NBG_NUM_FEATURES; ++b) add(b);
                } else {
                    for (int b = 0; b < NBG_NUM_FEATURES; ++b)
                        if (n == lower(kFeatureNames[b])) add(b);
                }
            }
            s.feature_mask = mask;
            for (int b = 0; b < NBG_NUM_FEATURES; ++b)
                if (mask & (1u << b)) f->dims.push_back(kFeatureNames[b]);
            // prepared()
            if ((mask & NBG_FEAT_DENSITY) && !(has_optimal_knn && has_optimal_radius))
                throw ArgError{"Density feature requires OptimalKNN and OptimalRadius dimensions, "
                               "which are missing in the input PointView."};
            if (s.optimized && !has_optimal_knn)
                throw ArgError{"Missing OptimalKNN dimension in input PointView."};
        } else if (t == "filters.approximatecoplanar") {
            // ApproximateCoplanarFilter.cpp:66-77
            allowed = {"knn", "thresh1", "thresh2"};
            s.kind = NBG_STAGE_APPROXIMATECOPLANAR;
            s.knn = 8;
            s.thresh1 = 25.0;
            s.thresh2 = 6.0;
            if (has("knn")) s.knn = (int32_t)arg_int(*o.get("knn"), "knn");
            if (has("thresh1")) s.thresh1 = arg_double(*o.get("thresh1"), "thresh1");
            if (has("thresh2")) s.thresh2 = arg_double(*o.get("thresh2"), "thresh2");
            f->dims = {"Coplanar"};
        } else if (t == "filters.estimaterank") {
            // EstimateRankFilter.cpp:66-74
            allowed = {"knn", "thresh"};
            s.kind = NBG_STAGE_ESTIMATERANK;
            s.knn = 8;
            s.thresh1 = 0.01;
            if (has("knn")) s.knn = (int32_t)arg_int(*o.get("knn"), "knn");
            if (has("thresh")) s.thresh1 = arg_double(*o.get("thresh"), "thresh");
            f->dims = {"Rank"};
        } else if (t == "filters.nndistance") {
            // NNDistanceFilter.cpp:66-105: mode kth / avg, case-insensitive
            allowed = {"mode", "k"};
            s.kind = NBG_STAGE_NNDISTANCE;
            s.knn = 10;
            s.mode = 0;
            if (has("k")) {
                const int64_t k = arg_int(*o.get("k"), "k");
                if (k < 0) throw ArgError{"Invalid value '" + raw_text(*o.get("k")) + "' for argument 'k'."};
                s.knn = (int32_t)std::min<int64_t>(k, INT32_MAX);
            }
            if (has("mode")) {
                const std::string m = lower(trim(raw_text(*o.get("mode"))));
                if (m == "kth") s.mode = 0;
                else if (m == "avg") s.mode = 1;
                else throw ArgError{"Invalid value '" + raw_text(*o.get("mode")) +
                                    "' for argument 'mode'."};
            }
            f->dims = {"NNDistance"};
        } else if (t == "filters.optimalneighborhood") {
            // OptimalNeighborhoodFilter.cpp:62-71
            allowed = {"min_k", "max_k"};
            s.kind = NBG_STAGE_OPTIMALNEIGHBORHOOD;
            int64_t kmin = 10, kmax = 14;
            if (has("min_k")) kmin = arg_int(*o.get("min_k"), "min_k");
            if (has("max_k")) kmax = arg_int(*o.get("max_k"), "max_k");
            if (kmin < 0) throw ArgError{"Invalid value '" + std::to_string(kmin) + "' for argument 'min_k'."};
            if (kmax < 0) throw ArgError{"Invalid value '" + std::to_string(kmax) + "' for argument 'max_k'."};
            s.knn = (int32_t)std::min<int64_t>(kmax, INT32_MAX);
            f->min_k = kmin;
            f->dims = {"OptimalKNN", "OptimalRadius"};
        } else if (t == "filters.lof") {
            // LOFFilter.cpp:62-70
            allowed = {"minpts"};
            s.kind = NBG_STAGE_LOF;
            s.knn = 10;
            if (has("minpts")) {
                const int64_t k = arg_int(*o.get("minpts"), "minpts");
                if (k < 0) throw ArgError{"Invalid value '" + raw_text(*o.get("minpts")) +
                                          "' for argument 'minpts'."};
                s.knn = (int32_t)std::min<int64_t>(k, INT32_MAX);
            }
            f->dims = {"NNDistance", "LocalReachabilityDistance", "LocalOutlierFactor"};
        } else if (t == "filters.outlier") {
            // OutlierFilter.cpp:62-76, 171-189: an unrecognised method leaves
            // the view unchanged with a warning
            allowed = {"method", "min_k", "radius", "mean_k", "multiplier", "class"};
            s.kind = NBG_STAGE_OUTLIER;
            s.knn = 8;
            s.thresh1 = 2.0;
            s.radius = 1.0;
            s.label = 7;  // ClassLabel::LowPoint
            f->min_k = 2;
            std::string method = "statistical";
            if (has("method")) method = raw_text(*o.get("method"));
            if (has("min_k")) f->min_k = arg_int(*o.get("min_k"), "min_k");
            if (has("radius")) s.radius = arg_double(*o.get("radius"), "radius");
            if (has("mean_k")) s.knn = (int32_t)arg_int(*o.get("mean_k"), "mean_k");
            if (has("multiplier")) s.thresh1 = arg_double(*o.get("multiplier"), "multiplier");
            if (has("class")) {
                const int64_t c = arg_int(*o.get("class"), "class");
                if (c < 0 || c > 255) throw ArgError{"Invalid value '" + raw_text(*o.get("class")) +
                                                     "' for argument 'class'."};
                s.label = (int32_t)c;
            }
            const std::string m = lower(method);
            if (m == "statistical") s.mode = 0;
            else if (m == "radius") s.mode = 1;
            else {
                s.mode = 2;
                f->log += "Requested method is unrecognized. Please choose from \"statistical\" or "
                          "\"radius\".\n";
            }
            f->dims = {"Classification"};
        } else {
            copy_err(err, err_len, "unknown stage type '" + t + "' (this library runs "
                                   "filters.normal, filters.eigenvalues, filters.covariancefeatures, "
                                   "filters.approximatecoplanar, filters.estimaterank, "
                                   "filters.nndistance, filters.optimalneighborhood, filters.lof, "
                                   "filters.outlier)");
            return NBG_ERR_INVALID;
        }
        for (auto& kv : o.obj) {
            if (common_option(kv.first)) continue;
            if (std::find(allowed.begin(), allowed.end(), kv.first) == allowed.end())
                throw ArgError{"Unexpected argument '" + kv.first + "'."};
        }
        if (s.knn < 0 && s.kind != NBG_STAGE_OUTLIER)
            throw ArgError{"Invalid value '" + std::to_string(s.knn) + "' for argument 'knn'."};
    } catch (const ArgError& e) {
        copy_err(err, err_len, t + ": " + e.msg);
        return NBG_ERR_INVALID;
    }
    *out = f.release();
    return NBG_OK;
}

extern "C" int nbg_filter_options(const nbg_filter* f, nbg_stage_opts* out) {
    if (!f || !out) return NBG_ERR_INVALID;
    *out = f->opts;
    if (f->opts.kind > NBG_STAGE_COVARIANCEFEATURES) {
        // the other consumers keep their own min_k (outlier's may be negative)
        out->min_k = (int32_t)std::max<int64_t>(INT32_MIN, std::min<int64_t>(f->min_k, INT32_MAX));
        return NBG_OK;
    }
    if (f->radius_set) {
        out->use_radius = 1;
        out->radius = f->radius;
        out->min_k = (int32_t)std::max<int64_t>(0, std::min<int64_t>(f->min_k, INT32_MAX));
        out->knn = 0;  // the reference zeroes or ignores knn with a radius
        return NBG_OK;
    }
    out->min_k = (int32_t)std::max<int64_t>(0, std::min<int64_t>(f->min_k, INT32_MAX));
    if (f->opts.stride > 1 && (int64_t)f->opts.stride * (f->opts.knn + 1) > 65)
        return NBG_ERR_UNSUPPORTED;
    return NBG_OK;
}

extern "C" int nbg_filter_dims(const nbg_filter* f, char* names, size_t len) {
    if (!f || !names || !len) return NBG_ERR_INVALID;
    std::string s;
    for (size_t i = 0; i < f->dims.size(); ++i) s += (i ? "," : "") + f->dims[i];
    if (s.size() + 1 > len) return NBG_ERR_INVALID;
    std::memcpy(names, s.c_str(), s.size() + 1);
    return NBG_OK;
}

extern "C" const char* nbg_filter_log(const nbg_filter* f) { return f ? f->log.c_str() : ""; }

extern "C" int nbg_filter_report(nbg_filter* f, const nbg_row_exception* ex, uint32_t n,
                                 int32_t stage_index, char* err, size_t err_len) {
    if (!f || (n && !ex)) return NBG_ERR_INVALID;
    // rows in point order, as the reference's loop meets them
    std::vector<nbg_row_exception> rows;
    for (uint32_t i = 0; i < n; ++i)
        if (ex[i].stage == (uint8_t)stage_index) rows.push_back(ex[i]);
    std::sort(rows.begin(), rows.end(),
              [](const nbg_row_exception& a, const nbg_row_exception& b) { return a.point_id < b.point_id; });
    const bool normal = f->opts.kind == NBG_STAGE_NORMAL;
    for (const auto& r : rows) {
        std::ostringstream o;
        const std::string id = std::to_string(r.point_id);
        if (normal) {
            o << "Skipping point " << id << ": ";
            if (r.code == NBG_ROW_TOO_FEW) o << "Not enough neighbors to compute normal.";
            else if (r.code == NBG_ROW_ZERO_COV)
                o << "Covariance matrix is all zeros. This suggests a large number of redundant points.";
            else o << "Cannot perform eigen decomposition during normal calculation.";
            f->log += o.str() + "\n";
            continue;
        }
        if (r.code == NBG_ROW_RADIUS_FEW) {
            o << "Skipping point " << id << ". Found " << r.reserved << " neighbors but required "
              << f->min_k << ".";
            f->log += o.str() + "\n";
            continue;
        }
        if (r.code == NBG_ROW_ZERO_COV) {
            o << "Skipping point " << id << ". Covariance matrix is all zeros. This suggests a large "
                 "number of redundant points. Consider using filters.sample with a small radius to "
                 "remove redundant points.";
            f->log += o.str() + "\n";
            continue;
        }
        // the reference throws from its per-point loop at the first such row
        std::string msg = r.code == NBG_ROW_ZERO_LAMBDA
                              ? "Eigenvalues are all 0. Can't compute local features."
                              : "Cannot perform eigen decomposition.";
        copy_err(err, err_len, f->type + ": " + msg);
        return NBG_ERR_INVALID;
    }
    return NBG_OK;
}

extern "C" int nbg_filter_outcome(nbg_filter* f, const nbg_run_stats* stats) {
    if (!f || !stats) return NBG_ERR_INVALID;
    // OutlierFilter.cpp:191-226
    if (f->opts.kind == NBG_STAGE_OUTLIER && f->opts.mode != 2 && stats->outliers + stats->inliers) {
        if (!stats->inliers)
            f->log += "Requested filter would remove all points. Try a larger radius/smaller "
                      "minimum neighbors.\n";
        else if (!stats->outliers)
            f->log += "Filtered cloud has no outliers!\n";
    }
    return NBG_OK;
}

extern "C" void nbg_filter_free(nbg_filter* f) { delete f; }

extern "C" int nbg_pipeline_parse(const char* json, nbg_pipeline** out, char* err, size_t err_len) {
    if (!json || !out) return NBG_ERR_INVALID;
    *out = nullptr;
    Json v;
    std::string perr;
    if (!parse_json(json, v, perr)) {
        copy_err(err, err_len, "pipeline is not valid JSON: " + perr);
        return NBG_ERR_INVALID;
    }
    const Json* list = &v;
    if (v.kind == Json::Object) list = v.get("pipeline");
    if (!list || list->kind != Json::Array) {
        copy_err(err, err_len, "pipeline JSON must be an array or an object with a \"pipeline\" array");
        return NBG_ERR_INVALID;
    }
    std::unique_ptr<nbg_pipeline> p(new nbg_pipeline());
    for (const Json& st : list->arr) {
        if (st.kind == Json::String) {
            // a bare file name: a reader (first) or writer stage
            p->types.push_back("file");
            p->options.push_back(to_json(st));
            continue;
        }
        if (st.kind != Json::Object) {
            copy_err(err, err_len, "pipeline stage must be a string or an object");
            return NBG_ERR_INVALID;
        }
        const Json* ty = st.get("type");
        p->types.push_back(ty && ty->kind == Json::String ? ty->str : "");
        p->options.push_back(to_json(st));
    }
    *out = p.release();
    return NBG_OK;
}

extern "C" int32_t nbg_pipeline_size(const nbg_pipeline* p) { return p ? (int32_t)p->types.size() : 0; }

extern "C" const char* nbg_pipeline_type(const nbg_pipeline* p, int32_t i) {
    if (!p || i < 0 || i >= (int32_t)p->types.size()) return "";
    return p->types[i].c_str();
}

extern "C" const char* nbg_pipeline_options(const nbg_pipeline* p, int32_t i) {
    if (!p || i < 0 || i >= (int32_t)p->options.size()) return "";
    return p->options[i].c_str();
}

extern "C" void nbg_pipeline_free(nbg_pipeline* p) { delete p; }

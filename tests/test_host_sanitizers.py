"""The host-side runtime under AddressSanitizer and UndefinedBehaviorSanitizer
(float-to-int overflow included): the stage layer (nbg_stages.cpp: pipeline
JSON, every filter's options, dims, logs, row reports) and the PDAL plugin
shim's host helpers, driven with valid, malformed and extreme inputs.  Any
sanitizer report fails the test.  (The CUDA library itself needs the device;
its host code is exercised by the GPU tests.)"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "nbg_b200.h"
#include "nbg_pdal_shim.hpp"

static int calls = 0;

static void pipeline(const std::string& j) {
    nbg_pipeline* p = nullptr;
    char err[256];
    ++calls;
    if (nbg_pipeline_parse(j.c_str(), &p, err, sizeof err) == NBG_OK && p) {
        for (int32_t i = 0; i < nbg_pipeline_size(p); ++i) {
            const char* t = nbg_pipeline_type(p, i);
            const char* o = nbg_pipeline_options(p, i);
            if (t && o) std::strlen(t), std::strlen(o);
        }
        nbg_pipeline_type(p, -1);
        nbg_pipeline_type(p, nbg_pipeline_size(p));
        nbg_pipeline_free(p);
    }
}

static void filter(const char* type, const std::string& opts, int kopt, int ropt) {
    nbg_filter* f = nullptr;
    char err[64];  // short on purpose: messages are truncated, never overrun
    ++calls;
    if (nbg_filter_create(type, opts.c_str(), kopt, ropt, &f, err, sizeof err) != NBG_OK || !f) return;
    nbg_stage_opts o;
    nbg_filter_options(f, &o);
    char dims[8], big[1024];
    nbg_filter_dims(f, dims, sizeof dims);
    nbg_filter_dims(f, big, sizeof big);
    std::vector<nbg_row_exception> ex = {{5, 0, NBG_ROW_TOO_FEW, 0}, {2, 0, NBG_ROW_ZERO_COV, 0},
                                         {4000000000u, 0, NBG_ROW_EIGEN_FAIL, 0},
                                         {7, 1, NBG_ROW_RADIUS_FEW, 65535}, {9, 0, 200, 0}};
    nbg_filter_report(f, ex.data(), (uint32_t)ex.size(), 0, err, sizeof err);
    nbg_filter_report(f, ex.data(), (uint32_t)ex.size(), 1, err, sizeof err);
    nbg_filter_report(f, nullptr, 0, 0, err, sizeof err);
    nbg_run_stats st;
    std::memset(&st, 0, sizeof st);
    nbg_filter_outcome(f, &st);
    st.outliers = 3;
    nbg_filter_outcome(f, &st);
    st.inliers = 9;
    nbg_filter_outcome(f, &st);
    std::strlen(nbg_filter_log(f));
    nbg_filter_free(f);
}

int main() {
    const std::vector<std::string> pipes = {
        "[]", "{}", "[\"in.las\", {\"type\": \"filters.normal\", \"knn\": 8}, \"out.las\"]",
        "{\"pipeline\": [{\"type\": \"filters.covariancefeatures\", \"feature_set\": \"all\"}]}",
        "[{\"type\": \"filters.normal\", \"viewpoint\": \"POINT (1 2 3)\", \"x\": [1, {\"a\": null}, true, false, -1.5e3]}]",
        "[{\"type\": \"a\\u00e9\\n\\t\\\\\\\"b\"}]", "[{\"type\": \"\\ud83d\\ude00\"}]",
        "[", "]", "[{", "[{\"type\"", "[{\"type\":", "[{\"type\": 1}]", "[{\"type\": \"x\",}]",
        "[\"unterminated", "[\"bad escape \\q\"]", "[\"\\u12\"]", "[\"\\u\"]", "{\"pipeline\": 3}",
        "[1, 2, 3]", "[null]", "nul", "tru", "-", "1e99999", "[-]", "[1e]", "[\"\x01\"]", "",
        std::string(200000, '['), std::string(200000, '{'), "[" + std::string(5000, ' ') + "]",
    };
    for (const auto& j : pipes) pipeline(j);
    std::string deep;
    for (int i = 0; i < 300; ++i) deep += "{\"a\": [";
    pipeline("[{\"type\": \"filters.normal\", \"x\": " + deep + "]");
    const char* types[] = {"filters.normal", "filters.eigenvalues", "filters.covariancefeatures",
                           "filters.approximatecoplanar", "filters.estimaterank",
                           "filters.nndistance", "filters.optimalneighborhood", "filters.lof",
                           "filters.outlier", "filters.unknown", ""};
    const std::vector<std::string> opts = {
        "{}", "{\"knn\": 8}", "{\"knn\": \"8\"}", "{\"knn\": -3}", "{\"knn\": 1e400}",
        "{\"knn\": 4294967297}", "{\"knn\": 0.5}", "{\"knn\": \"eight\"}", "{\"knn\": null}",
        "{\"knn\": [8]}", "{\"radius\": 1.0}", "{\"radius\": -1}", "{\"radius\": \"nan\"}",
        "{\"knn\": 8, \"radius\": 1}", "{\"viewpoint\": \"POINT (1 2 3)\"}",
        "{\"viewpoint\": \"POINT (1 2)\"}", "{\"viewpoint\": \"POINT (a b c)\"}",
        "{\"viewpoint\": \"" + std::string(10000, '(') + "\"}", "{\"always_up\": \"false\"}",
        "{\"always_up\": \"maybe\"}", "{\"feature_set\": \"all\"}",
        "{\"feature_set\": \"Linearity,Planarity,,Nope\"}", "{\"feature_set\": \"" + std::string(5000, ',') + "\"}",
        "{\"mode\": \"raw\"}", "{\"mode\": \"bogus\"}", "{\"stride\": 0}", "{\"stride\": 1000000}",
        "{\"optimized\": true}", "{\"min_k\": -1}", "{\"thresh1\": 1e308, \"thresh2\": -1e308}",
        "{\"k\": 3, \"mode\": \"avg\"}", "{\"min_k\": 20, \"max_k\": 10}", "{\"minpts\": 1}",
        "{\"method\": \"radius\", \"radius\": 0, \"min_k\": 0}", "{\"method\": \"nope\"}",
        "{\"mean_k\": 0, \"multiplier\": -2, \"class\": 300}", "{\"threads\": -1}",
        "{\"unknown_option\": 1}", "not json", "{\"knn\": 8", "[1]", "",
    };
    for (const char* t : types)
        for (const auto& o : opts)
            for (int k = 0; k < 2; ++k) filter(t, o, k, k);
    // the PDAL plugin shim's host helpers
    for (const auto& s : nbg_pdal::stages()) nbg_pdal::find_stage(s.plugin_type);
    nbg_pdal::find_stage("filters.nothing");
    nbg_pdal::find_stage("");
    nbg_pdal::options_json({{"a\"b", "c\\d"}, {"ctl", std::string("\x01\x1f\x7f", 3)},
                            {"", ""}, {"utf8", "\xc3\xa9\xff"}});
    const double inf = std::numeric_limits<double>::infinity();
    const double nan = std::numeric_limits<double>::quiet_NaN();
    std::vector<double> v = {0.0, 0.01, -0.01, 21474836.47, -21474836.48, 21474836.48, -21474836.49,
                             1e300, -1e300, inf, -inf, nan, 5e-324, 123.456789};
    std::vector<int32_t> raw(v.size());
    uint64_t bad = 0;
    for (double scale : {0.01, 0.001, 1.0, 1e-300, 1e300})
        for (double off : {0.0, 512000.0, -1e300, 1e300}) nbg_pdal::recover_raw(v.data(), v.size(), scale, off, raw.data(), &bad);
    nbg_pdal::recover_raw(v.data(), 0, 0.01, 0.0, raw.data(), &bad);
    std::printf("ok %d\n", calls);
    return 0;
}
"""


def test_host_runtime_under_asan_ubsan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-g", "-pthread",
                           "-fsanitize=address,undefined,float-cast-overflow",
                           "-fno-sanitize-recover=all", "-fno-omit-frame-pointer",
                           "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "gpupdal_b200", "plugin"),
                           str(src), os.path.join(ROOT, "gpupdal_b200", "csrc", "nbg_stages.cpp"),
                           "-o", str(exe)])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=600)
    report = r.stdout + r.stderr
    assert r.returncode == 0, report[-4000:]
    assert "runtime error" not in report and "AddressSanitizer" not in report, report[-4000:]
    assert r.stdout.startswith("ok ")

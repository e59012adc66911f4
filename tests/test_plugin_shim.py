"""The PDAL plugin's PDAL-independent part (gpupdal_b200/plugin/nbg_pdal_shim.hpp),
compiled here into a small driver program: the stages it registers and
their options (accepted by the stage layer under the reference filters'
names), the option object it builds, the exact recovery of raw LAS integers
from a view's doubles, and (GPU) one stage run through the C ABI, equal to
the same stage run through the Python binding.  The PDAL glue itself
(nbg_pdal_plugin.cpp) needs PDAL's generated headers and libpdalcpp, which
this image does not have."""
import json
import os
import subprocess

import numpy as np
import pytest

from gpupdal_b200 import synthetic as syn
from gpupdal_b200.stages import Filter

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <fstream>
#include <iostream>
#include "nbg_pdal_shim.hpp"

static std::vector<char> slurp(const char* p) {
    std::ifstream f(p, std::ios::binary);
    return std::vector<char>(std::istreambuf_iterator<char>(f), {});
}

int main(int argc, char** argv) {
    std::string mode = argv[1];
    if (mode == "stages") {
        std::printf("[");
        bool first = true;
        for (const auto& s : nbg_pdal::stages()) {
            std::printf("%s{\"plugin\": \"%s\", \"base\": \"%s\", \"options\": [", first ? "" : ",",
                        s.plugin_type, s.base_type);
            for (size_t i = 0; i < s.options.size(); ++i)
                std::printf("%s\"%s\"", i ? "," : "", s.options[i]);
            std::printf("]}");
            first = false;
        }
        std::printf("]\n");
        return 0;
    }
    if (mode == "json") {
        std::cout << nbg_pdal::options_json({{"knn", "8"}, {"viewpoint", "POINT (1 \"2\" 3)"},
                                             {"feature_set", "a\\b\tc"}})
                  << "\n";
        return 0;
    }
    if (mode == "raw") {
        // argv: file of doubles, scale, offset -> prints first bad index or "ok" + raws
        std::vector<char> b = slurp(argv[2]);
        const uint64_t n = b.size() / 8;
        std::vector<int32_t> raw(n);
        uint64_t bad = 0;
        if (!nbg_pdal::recover_raw((const double*)b.data(), n, std::atof(argv[3]), std::atof(argv[4]),
                                   raw.data(), &bad)) {
            std::printf("bad %llu\n", (unsigned long long)bad);
            return 0;
        }
        std::printf("ok");
        for (uint64_t i = 0; i < n; ++i) std::printf(" %d", raw[i]);
        std::printf("\n");
        return 0;
    }
    // run: x y z files, base type, options json, ndims, output file
    std::vector<char> bx = slurp(argv[2]), by = slurp(argv[3]), bz = slurp(argv[4]);
    const uint64_t n = bx.size() / 8;
    const int nd = std::atoi(argv[7]);
    std::vector<std::vector<double>> out(nd, std::vector<double>(n, 0.0));
    std::vector<double*> cols;
    for (auto& o : out) cols.push_back(o.data());
    nbg_context* ctx = nullptr;
    if (nbg_create(&ctx, 0, 0) != NBG_OK) return 3;
    const double scale[3] = {0.01, 0.01, 0.01}, offset[3] = {0, 0, 0};
    std::string log, err;
    int rc = nbg_pdal::run_stage(ctx, argv[5], argv[6], (const double*)bx.data(),
                                 (const double*)by.data(), (const double*)bz.data(), n, scale,
                                 offset, nullptr, nullptr, cols, log, err);
    if (rc) {
        std::fprintf(stderr, "rc %d: %s\n", rc, err.c_str());
        return 4;
    }
    std::ofstream f(argv[8], std::ios::binary);
    for (auto& o : out) f.write((const char*)o.data(), n * 8);
    std::printf("%s", log.c_str());
    nbg_destroy(ctx);
    return 0;
}
"""


def _driver(tmp_path):
    from gpupdal_b200 import build
    lib = build.build()
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I",
                           os.path.join(ROOT, "gpupdal_b200", "plugin"), str(src), "-o", str(exe),
                           lib, f"-Wl,-rpath,{os.path.dirname(lib)}"])
    return str(exe)


VALUES = {"knn": "8", "radius": "1.0", "viewpoint": "POINT (0 0 0)", "always_up": "true",
          "refine": "false", "normalize": "true", "stride": "1", "min_k": "3", "threads": "2",
          "feature_set": "all", "optimized": "false", "thresh1": "25", "thresh2": "6",
          "thresh": "0.01", "k": "5", "max_k": "14", "minpts": "10", "method": "radius",
          "mean_k": "8", "multiplier": "2", "class": "7"}
MODES = {"filters.covariancefeatures": "raw", "filters.nndistance": "avg"}


def test_plugin_stages_take_the_reference_options(tmp_path):
    exe = _driver(tmp_path)
    specs = json.loads(subprocess.check_output([exe, "stages"], text=True))
    assert len(specs) == 9
    for s in specs:
        assert s["plugin"] == "filters.b200" + s["base"].split(".")[1]
        for opt in s["options"]:
            v = MODES.get(s["base"], "") if opt == "mode" else VALUES[opt]
            if s["base"] == "filters.normal" and opt == "radius":
                continue  # knn and radius together are refused, as in the reference
            Filter(s["base"], {opt: v}, True, True)  # raises on an unknown option
        f = Filter(s["base"], {}, True, True)
        assert f.dims()


def test_plugin_options_json(tmp_path):
    exe = _driver(tmp_path)
    text = subprocess.check_output([exe, "json"], text=True).strip()
    assert json.loads(text) == {"knn": "8", "viewpoint": 'POINT (1 "2" 3)', "feature_set": "a\\b\tc"}


def test_plugin_raw_recovery(tmp_path):
    exe = _driver(tmp_path)
    raw = np.array([0, 1, -7, 123456789, -2000000000], np.int64)
    v = raw * 0.01 + 512000.0
    p = tmp_path / "v.bin"
    v.astype(np.float64).tofile(p)
    out = subprocess.check_output([exe, "raw", str(p), "0.01", "512000"], text=True).split()
    assert out[0] == "ok" and [int(t) for t in out[1:]] == raw.tolist()
    w = v.copy()
    w[3] = np.nextafter(w[3], np.inf)  # not of the form raw*scale+offset
    w.tofile(p)
    assert subprocess.check_output([exe, "raw", str(p), "0.01", "512000"], text=True).split() == ["bad", "3"]


@pytest.mark.gpu
def test_plugin_run_stage_matches_binding(nbg, tmp_path):
    exe = _driver(tmp_path)
    x, y, z = syn.stress(1_000_000, 2)
    m = (x < 8000) & (y < 8000)
    x, y, z = x[m], y[m], z[m]
    files = []
    for name, v in zip("xyz", (x, y, z)):
        p = tmp_path / f"{name}.bin"
        syn.to_double(v).tofile(p)
        files.append(str(p))
    tile = nbg.tile(x, y, z)
    for base, opts in [("filters.normal", {"knn": "12"}),
                       ("filters.covariancefeatures", {"knn": "10", "feature_set": "Linearity,Omnivariance"}),
                       ("filters.lof", {"minpts": "9"})]:
        f = Filter(base, opts)
        o, _ = f.options()
        nd = len(f.dims())
        outp = tmp_path / "out.bin"
        subprocess.check_call([exe, "run", *files, base, json.dumps(opts), str(nd), str(outp)])
        got = np.fromfile(outp, np.float64).reshape(nd, len(x))
        want, ex, _ = nbg.run(tile, [o])
        assert np.array_equal(got, want[0], equal_nan=True), base

"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer: a driver
compiled together with oracle/nbg_oracle.cpp builds a tree over a cloud with
exact duplicates and collinear points, queries neighbours (strided too),
and runs every stage kind in both oracle modes; any sanitizer report fails
the test.  (The device code has no sanitizer on this hardware pool; it is
held to the oracle instead.)"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include "nbg_oracle.cpp"

#include <cstdio>
#include <vector>

static nbg_stage_opts base(int kind, int knn) {
    nbg_stage_opts o;
    std::memset(&o, 0, sizeof o);
    o.kind = kind;
    o.knn = knn;
    o.always_up = 1;
    o.stride = 1;
    o.min_k = 3;
    o.mode = NBG_MODE_SQRT;
    o.feature_mask = NBG_FEAT_ALL;
    return o;
}

int main() {
    const uint64_t n = 3000;
    std::vector<double> x(n), y(n), z(n);
    uint64_t s = 12345;
    auto rnd = [&]() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return (double)((s >> 33) % 20000) * 0.01;
    };
    for (uint64_t i = 0; i < n; ++i) {
        if (i % 10 == 9) {  // exact duplicate of the previous point
            x[i] = x[i - 1]; y[i] = y[i - 1]; z[i] = z[i - 1];
        } else if (i % 10 == 8) {  // on one line
            x[i] = (double)(i % 97); y[i] = 2.0 * x[i]; z[i] = 5.0;
        } else {
            x[i] = rnd(); y[i] = rnd(); z[i] = rnd() * 0.05;
        }
    }
    std::vector<double> kopt(n, 10.0), ropt(n);
    for (uint64_t i = 0; i < n; ++i) ropt[i] = 0.3 + (double)(i % 13) * 0.1;
    void* t = orc_tree_build_t(x.data(), y.data(), z.data(), n, 2);
    std::vector<uint64_t> ids(64);
    for (uint64_t q = 0; q < n; q += 97) orc_tree_neighbors(t, x[q], y[q], z[q], 16, 2, ids.data());
    std::vector<uint64_t> all(n * 9);
    orc_all_neighbors(t, 9, all.data(), 2);
    std::vector<std::vector<double>> cols(NBG_MAX_DIMS, std::vector<double>(n));
    std::vector<double*> cp;
    for (auto& c : cols) cp.push_back(c.data());
    std::vector<uint8_t> st(n);
    std::vector<nbg_stage_opts> stages;
    stages.push_back(base(NBG_STAGE_NORMAL, 8));
    { auto o = base(NBG_STAGE_NORMAL, 8); o.always_up = 0; stages.push_back(o); }
    { auto o = base(NBG_STAGE_NORMAL, 8); o.has_viewpoint = 1; o.viewpoint[0] = 100;
      o.viewpoint[1] = 100; o.viewpoint[2] = 50; stages.push_back(o); }
    { auto o = base(NBG_STAGE_EIGENVALUES, 8); o.normalize = 1; stages.push_back(o); }
    { auto o = base(NBG_STAGE_EIGENVALUES, 8); o.stride = 2; stages.push_back(o); }
    { auto o = base(NBG_STAGE_EIGENVALUES, 8); o.use_radius = 1; o.radius = 1.5; stages.push_back(o); }
    stages.push_back(base(NBG_STAGE_COVARIANCEFEATURES, 10));
    { auto o = base(NBG_STAGE_COVARIANCEFEATURES, 10); o.optimized = 1; o.mode = NBG_MODE_NORMALIZED;
      stages.push_back(o); }
    { auto o = base(NBG_STAGE_APPROXIMATECOPLANAR, 8); o.thresh1 = 25; o.thresh2 = 6; stages.push_back(o); }
    { auto o = base(NBG_STAGE_ESTIMATERANK, 8); o.thresh1 = 0.01; stages.push_back(o); }
    { auto o = base(NBG_STAGE_NNDISTANCE, 10); o.mode = 1; stages.push_back(o); }
    { auto o = base(NBG_STAGE_OPTIMALNEIGHBORHOOD, 14); o.min_k = 10; stages.push_back(o); }
    stages.push_back(base(NBG_STAGE_LOF, 10));
    { auto o = base(NBG_STAGE_OUTLIER, 8); o.mode = 0; o.thresh1 = 2.0; o.label = 7; o.min_k = 2;
      stages.push_back(o); }
    { auto o = base(NBG_STAGE_OUTLIER, 8); o.mode = 1; o.radius = 1.0; o.label = 7; o.min_k = 2;
      stages.push_back(o); }
    int bad = 0;
    for (auto& o : stages)
        for (int mode = 0; mode < 2; ++mode)
            if (orc_run_stage(t, &o, kopt.data(), ropt.data(), mode, cp.data(), st.data(), 2) < 0) {
                std::printf("stage %d mode %d failed\n", o.kind, mode);
                ++bad;
            }
    double ev[3], vec[9];
    const double a[9] = {2, 1, 0, 1, 2, 0, 0, 0, 1};
    orc_eigen_chain(a, ev, vec);
    orc_tree_free(t);
    std::printf("ok %d\n", bad);
    return bad ? 1 : 0;
}
"""


def test_oracle_under_asan_ubsan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-g", "-ffp-contract=off", "-pthread",
                           "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                           "-fno-omit-frame-pointer", "-I", os.path.join(ROOT, "oracle"),
                           str(src), "-o", str(exe)])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=600)
    report = r.stdout + r.stderr
    assert r.returncode == 0, report[-4000:]
    assert "runtime error" not in report and "AddressSanitizer" not in report, report[-4000:]
    assert "ok 0" in r.stdout

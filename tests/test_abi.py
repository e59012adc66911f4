"""The C ABI library loads and exports every symbol include/nbg_b200.h
declares, and the ctypes mirror has the header's layout (CPU only; no call
here touches a GPU)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from gpupdal_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nbg_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nbg_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("nbg_create", "nbg_destroy", "nbg_tile_upload", "nbg_run", "nbg_last_error",
                 "nbg_neighbor_sets"):
        assert must in names


def test_library_exports_every_declared_symbol(lib_path):
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True).stdout
    for n in declared_functions():
        assert re.search(rf"\bT {n}\b", out), n


def test_ctypes_layout_matches_header():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "nbg_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(nbg_stage_opts), sizeof(nbg_columns),
         sizeof(nbg_row_exception), sizeof(nbg_run_stats));
  printf("%zu %zu %zu %zu\n", offsetof(nbg_stage_opts, viewpoint),
         offsetof(nbg_stage_opts, feature_mask), offsetof(nbg_columns, offset),
         offsetof(nbg_run_stats, grid_ms));
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(nbg_request), sizeof(nbg_request_result),
         offsetof(nbg_request, stages), offsetof(nbg_request, user_tag),
         offsetof(nbg_request_result, stats), offsetof(nbg_run_stats, kd_build_ms));
  printf("%zu %zu %zu\n", sizeof(nbg_las_info), offsetof(nbg_las_info, point_count),
         offsetof(nbg_las_info, max));
  printf("%zu %zu %zu\n", sizeof(nbg_tune_entry), offsetof(nbg_tune_entry, cell_factor),
         offsetof(nbg_run_stats, output_chunks));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "l")
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe])
        lines = subprocess.check_output([exe], text=True).split("\n")
    sizes = [int(v) for v in lines[0].split()]
    offs = [int(v) for v in lines[1].split()]
    assert sizes == [ctypes.sizeof(abi.StageOpts), ctypes.sizeof(abi.Columns),
                     ctypes.sizeof(abi.RowException), ctypes.sizeof(abi.RunStats)]
    assert offs == [abi.StageOpts.viewpoint.offset, abi.StageOpts.feature_mask.offset,
                    abi.Columns.offset.offset, abi.RunStats.grid_ms.offset]
    served = [int(v) for v in lines[2].split()]
    assert served == [ctypes.sizeof(abi.Request), ctypes.sizeof(abi.RequestResult),
                      abi.Request.stages.offset, abi.Request.user_tag.offset,
                      abi.RequestResult.stats.offset, abi.RunStats.kd_build_ms.offset]
    las = [int(v) for v in lines[3].split()]
    assert las == [ctypes.sizeof(abi.LasInfo), abi.LasInfo.point_count.offset,
                   abi.LasInfo.max.offset]
    tune = [int(v) for v in lines[4].split()]
    assert tune == [ctypes.sizeof(abi.TuneEntry), abi.TuneEntry.cell_factor.offset,
                    abi.RunStats.output_chunks.offset]


def test_loader_fails_loudly_without_the_library(tmp_path):
    with pytest.raises(RuntimeError):
        abi._LIB = None
        try:
            abi.load_library(str(tmp_path / "missing.so"))
        finally:
            abi._LIB = None

"""The PDAL plugin translation unit compiles against PDAL's own headers.

gpupdal_b200/plugin/compile_check.py generates the two headers a PDAL build
writes (pdal/Dimension.hpp with PDAL's dimbuilder from pdal/Dimension.json,
pdal_features.hpp from its template) and compiles nbg_pdal_plugin.cpp to an
object against the reference tree's headers (no link: libpdalcpp needs
GDAL).  The object must define the plugin entry point PDAL's loader calls
(PF_initPlugin, pdal/PluginHelper.hpp) and the stage class's Filter
overrides.  Runs where the reference tree is present (the build container).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_tree():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    tree = ge.REFERENCE_TREE
    if not os.path.isfile(os.path.join(tree, "pdal", "Dimension.json")):
        pytest.skip("no PDAL source tree to compile against")
    return tree


def test_plugin_translation_unit_compiles():
    tree = _reference_tree()
    sys.path.insert(0, os.path.join(ROOT, "gpupdal_b200", "plugin"))
    import compile_check
    try:
        obj = compile_check.compile_plugin(tree)
    except subprocess.CalledProcessError as e:
        pytest.fail(f"plugin compile failed:\n{e.stderr[-3000:]}")
    syms = subprocess.run(["nm", "-C", obj], capture_output=True, text=True, check=True).stdout
    defined = {ln.split(" ", 2)[2] for ln in syms.splitlines() if ln[17:19] in ("T ", "W ")}
    assert "PF_initPlugin" in defined
    for m in ("filter(pdal::PointView&)", "addArgs(pdal::ProgramArgs&)",
              "addDimensions(pdal::PointLayout*)", "prepared(pdal::BasePointTable&)"):
        assert any(s.startswith("pdal::B200NeighbourhoodFilter::" + m) for s in defined), m

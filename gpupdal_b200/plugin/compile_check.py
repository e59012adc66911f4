"""Compiles the PDAL plugin translation unit against a PDAL source tree.

    python gpupdal_b200/plugin/compile_check.py <pdal-source-root>

The plugin (nbg_pdal_plugin.cpp) is written against PDAL's public headers,
two of which a PDAL build generates rather than ships: pdal/Dimension.hpp
(written by PDAL's own dimbuilder tool from pdal/Dimension.json) and
pdal_features.hpp (CMake's configure_file of pdal_features.hpp.in).  This
recipe does what a PDAL build does for them, inside _build/ beside this file:

1. compiles the tree's dimbuilder (dimbuilder/DimBuilder.cpp with
   pdal/util/Utils.cpp, as its CMakeLists.txt does) and runs it on
   pdal/Dimension.json;
2. configures pdal_features.hpp from its template with the tree's project
   version and every optional feature off;
3. compiles nbg_pdal_plugin.cpp to an object (no link: libpdalcpp needs GDAL,
   absent here) with the tree's include paths and the generated headers.

Returns the object's path; raises CalledProcessError with the compiler's
output when a step fails.  Nothing here is part of the library: the plugin is
built by CMake (CMakeLists.txt) wherever PDAL is installed.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BUILD = os.path.join(HERE, "_build")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise subprocess.CalledProcessError(r.returncode, cmd, r.stdout, r.stderr)
    return r


def _project_version(src):
    with open(os.path.join(src, "CMakeLists.txt")) as f:
        m = re.search(r"project\(\s*PDAL\s+VERSION\s+(\d+)\.(\d+)\.(\d+)", f.read())
    return tuple(m.groups()) if m else ("0", "0", "0")


def configure_features(src, out_path):
    """pdal_features.hpp from its template: @VAR@ substituted, every
    #cmakedefine left undefined (no optional PDAL feature)."""
    major, minor, patch = _project_version(src)
    vals = {"PDAL_VERSION_MAJOR": major, "PDAL_VERSION_MINOR": minor,
            "PDAL_VERSION_PATCH": patch, "PDAL_VERSION": f"{major}.{minor}.{patch}",
            "GIT_SHA1": "unknown", "PDAL_BUILD_TYPE": "Release", "PDAL_PLUGIN_INSTALL_PATH": ""}
    out = []
    with open(os.path.join(src, "pdal_features.hpp.in")) as f:
        for line in f:
            m = re.match(r"\s*#cmakedefine\s+(\w+)", line)
            if m:
                out.append(f"/* #undef {m.group(1)} */\n")
                continue
            out.append(re.sub(r"@(\w+)@", lambda g: vals.get(g.group(1), ""), line))
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    with open(out_path, "w") as f:
        f.writelines(out)


def compile_plugin(src, cxx="g++"):
    src = os.path.abspath(src)
    gen = os.path.join(BUILD, "gen")
    os.makedirs(os.path.join(gen, "pdal"), exist_ok=True)
    inc = ["-I", gen, "-I", src, "-I", os.path.join(src, "vendor"),
           "-I", os.path.join(src, "vendor", "nlohmann"),
           "-I", os.path.join(src, "vendor", "utfcpp", "source"),
           "-I", os.path.join(src, "vendor", "eigen")]
    # 1. the tree's dimbuilder, then Dimension.hpp from Dimension.json
    dimb = os.path.join(BUILD, "dimbuilder")
    _run([cxx, "-std=c++17", "-O1", *inc, os.path.join(src, "dimbuilder", "DimBuilder.cpp"),
          os.path.join(src, "pdal", "util", "Utils.cpp"), "-o", dimb, "-ldl"])
    _run([dimb, os.path.join(src, "pdal", "Dimension.json"),
          os.path.join(gen, "pdal", "Dimension.hpp")])
    # 2. the feature header
    configure_features(src, os.path.join(gen, "pdal_features.hpp"))
    # 3. the plugin translation unit, compiled to an object
    obj = os.path.join(BUILD, "nbg_pdal_plugin.o")
    _run([cxx, "-std=c++17", "-O1", "-fPIC", "-c", *inc, "-I", os.path.join(ROOT, "include"),
          os.path.join(HERE, "nbg_pdal_plugin.cpp"), "-o", obj])
    return obj


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    try:
        print(compile_plugin(sys.argv[1]))
    except subprocess.CalledProcessError as e:
        sys.exit(f"{' '.join(e.cmd)}\n{e.stderr[-4000:]}")

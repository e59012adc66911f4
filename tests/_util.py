"""Helpers shared by the tests: golden fixtures and the stated tolerances.

Tolerances (the bar of the parity tests):
  * neighbour id sets: bit-exact
  * row status (skip / throw codes): exact
  * eigenvalues: |d| <= 1e-5 * max(lambda_max, tiny)  (normwise relative)
  * normals: ||d|| <= 1e-5 on rows whose relative eigen-gap
    (lambda1 - lambda0) / lambda2 is >= 1e-4 (below that the eigenvector is
    not determined by the data; the reference's own choice is arbitrary).
    With always_up, a row whose NormalZ is within `sign_eps` of zero has no
    determined sign (the flip test n_z < 0 sees rounding residue); such rows
    are compared up to sign.  sign_eps is 1e-9 against the FP64 oracle and
    1e-6 against the reference's own outputs, whose float narrowing moves
    NormalZ by up to ~1e-7
  * curvature and ratio features in [0, 1]: |d| <= 1e-5
  * EigenvalueSum, Omnivariance, Eigenentropy, Density: relative 1e-5 of
    max(|value|, lambda scale)
  * NaN positions equal, except rows whose smallest eigenvalue is below
    1e-12 * lambda_max (an exact zero vs a rounding residue)
"""
from __future__ import annotations

import os

import numpy as np

from gpupdal_b200 import abi
from gpupdal_b200 import synthetic as syn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def opts_from_bytes(b):
    o = abi.StageOpts()
    import ctypes
    ctypes.memmove(ctypes.addressof(o), bytes(b), ctypes.sizeof(o))
    return o


def doubles(g):
    return tuple(syn.to_double(g[k]) for k in ("x", "y", "z"))


def sorted_rows(a):
    return np.sort(np.asarray(a, dtype=np.int64), axis=1)


def eigen_scale(eig_f64):
    """lambda_max per row from an eigenvalues (3, n) array."""
    return np.maximum(np.abs(eig_f64).max(axis=0), 1e-300)


def compare_stage(opts, got, want, want_status, got_status, lam=None, label="", gap_min=1e-4,
                  tol=TOL, sign_eps=1e-9):
    """Asserts `got` (ndims, n) matches `want` within the stated bars.

    `lam` is the (3, n) ascending eigenvalue array of the accuracy oracle
    (scale and eigen-gap of each row); rows whose relative gap is below
    `gap_min` are exempt from eigenvector-dependent dimensions."""
    assert np.array_equal(got_status, want_status), (
        f"{label}: status differs on {np.count_nonzero(got_status != want_status)} rows")
    ok = want_status == 0
    dims = abi.stage_dims(opts)
    n = got.shape[1]
    if lam is not None:
        lmax = eigen_scale(lam)
        gap = (lam[1] - lam[0]) / lmax
        degenerate = lam[0] < 1e-12 * lmax
    else:
        lmax, gap, degenerate = np.ones(n), np.ones(n), np.zeros(n, bool)
    if opts.kind == abi.STAGE_COVARIANCEFEATURES:
        lscale = {abi.MODE_SQRT: np.sqrt(lmax), abi.MODE_RAW: lmax}.get(opts.mode, np.ones(n))
    else:
        lscale = lmax
    vec_ok = gap >= gap_min
    if opts.kind == abi.STAGE_NORMAL and opts.always_up and not opts.has_viewpoint:
        flat = np.abs(want[2]) < sign_eps
        if flat.any():
            got = got.copy()
            flip = flat & (np.abs(got[:3] - want[:3]).sum(0) > np.abs(got[:3] + want[:3]).sum(0))
            got[:3, flip] = -got[:3, flip]
    for d, name in enumerate(dims):
        g, w = got[d][ok], want[d][ok]
        nan_ok = ~degenerate[ok]
        assert np.array_equal(np.isnan(g)[nan_ok], np.isnan(w)[nan_ok]), f"{label}:{name} NaN positions"
        fin = np.isfinite(g) & np.isfinite(w)
        ls = lscale[ok]
        if name.startswith("Eigenvalue"):
            bar = tol if opts.normalize else tol * lmax[ok]
        elif name in ("NormalX", "NormalY", "NormalZ", "DemantkeVerticality", "Verticality"):
            bar = np.where(vec_ok[ok], tol, np.inf)
        elif name == "Omnivariance":
            bar = tol * ls
        elif name == "Eigenentropy":
            bar = tol * np.maximum(np.abs(w), ls * (1.0 + np.abs(np.log(np.maximum(ls, 1e-300)))))
        elif name == "EigenvalueSum":
            bar = tol * np.abs(w)
        elif name == "Density":
            bar = 1e-9 * np.abs(w)
        else:
            bar = tol
        err = np.abs(g - w)
        bad = fin & ~(err <= bar)
        assert not bad.any(), (f"{label}:{name} {bad.sum()} rows over the bar, max err "
                               f"{err[fin].max():.3e}")


def status_from_exceptions(n, ex, stage=0):
    s = np.zeros(n, np.uint8)
    e = ex[ex["stage"] == stage]
    s[e["point_id"]] = e["code"]
    return s

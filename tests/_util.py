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
    NormalZ by up to ~1e-7.  With always_up=false the sign is the Eigen
    chain's; rows whose exact covariance has a zero off-diagonal entry
    (lattice symmetry) take a branch decided by rounding residue and are
    compared up to sign; the sign itself is checked against the reference's
    own outputs (the FP64 oracle's sign is only an alignment).  Rows whose
    chain sign flips under a 1e-7 relative perturbation of the exact covariance
    are compared up to sign as well (sign_unstable_rows)
  * curvature and ratio features in [0, 1]: |d| <= 1e-5 (SurfaceVariation,
    unbounded in normalized mode: relative 1e-5 above 1)
  * EigenvalueSum, Omnivariance, Eigenentropy, Density: relative 1e-5 of
    max(|value|, lambda scale); Omnivariance and Eigenentropy of rows whose
    smallest eigenvalue is below the oracle's noise level (1e-8 * lambda_max
    against the FP64 oracle, 1e-6 against the reference's float-narrowed
    outputs; collinear neighbourhoods: zero exactly here) are not compared
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
    """abi.StageOpts from the bytes a golden file stored; files written before
    the radius fields existed hold a shorter record (radius off, min_k 3)."""
    import ctypes
    o = abi.StageOpts()
    raw = bytes(b)
    if len(raw) < ctypes.sizeof(o):
        o.min_k = 3
    ctypes.memmove(ctypes.addressof(o), raw, min(len(raw), ctypes.sizeof(o)))
    return o


def doubles(g):
    return tuple(syn.to_double(g[k]) for k in ("x", "y", "z"))


def sorted_rows(a):
    return np.sort(np.asarray(a, dtype=np.int64), axis=1)


def eigen_scale(eig_f64):
    """lambda_max per row from an eigenvalues (3, n) array."""
    return np.maximum(np.abs(eig_f64).max(axis=0), 1e-300)


def symmetric_rows(x, y, z, nbr):
    """Rows whose exact (integer) neighbourhood covariance has an off-diagonal
    entry equal to zero: lattice symmetries, where an eigensolver's sign
    choice is decided by rounding residue."""
    P = np.stack([np.asarray(v, np.int64) for v in (x, y, z)], 1)
    d = P[nbr.astype(np.int64)] - P[:, None, :]
    n = nbr.shape[1]
    S1 = d.sum(1)
    S2 = np.einsum("rki,rkj->rij", d, d)
    M = n * S2 - S1[:, :, None] * S1[:, None, :]
    return (M[:, 1, 0] == 0) | (M[:, 2, 0] == 0) | (M[:, 2, 1] == 0)


def sign_unstable_rows(port, x, y, z, nbr, scale=0.01, trials=8, rel=1e-7, seed=0):
    """Rows whose Eigen-chain eigenvector sign flips when the exact covariance
    is perturbed at the level of the reference's float narrowing (relative
    `rel` of its largest entry): exact lattice ties (equal diagonal entries,
    rational eigenvalues) send the chain down a branch that rounding residue
    decides, so the reference's sign there is not a property of the data."""
    P = np.stack([np.asarray(v, np.int64) for v in (x, y, z)], 1)
    d = P[nbr.astype(np.int64)] - P[:, None, :]
    n = nbr.shape[1]
    S1 = d.sum(1)
    S2 = np.einsum("rki,rkj->rij", d, d)
    C = (n * S2 - S1[:, :, None] * S1[:, None, :]) * (scale * scale) / (n * (n - 1))
    rng = np.random.default_rng(seed)
    out = np.zeros(len(P), bool)
    for r in range(len(P)):
        v0 = port.eigen_chain(C[r])[2][:, 0]
        sc = np.abs(C[r]).max()
        for _ in range(trials):
            E = rng.standard_normal((3, 3)) * rel * sc
            if np.dot(port.eigen_chain(C[r] + (E + E.T) / 2)[2][:, 0], v0) < 0:
                out[r] = True
                break
    return out


def viewpoint_tangent_rows(opts, X, Y, Z, want, eps=1e-6):
    """Rows whose viewpoint lies in the tangent plane ((vp - p) . n == 0 up to
    `eps` relative): the reference's orientation test leaves the eigensolver's
    sign there, which rounding residue decides on lattice inputs."""
    vp = np.asarray(list(opts.viewpoint), np.float64)
    d = np.stack([vp[0] - X, vp[1] - Y, vp[2] - Z])
    dot = (d * want[:3]).sum(0)
    return np.abs(dot) <= eps * np.abs(d).sum(0)


def compare_stage(opts, got, want, want_status, got_status, lam=None, label="", gap_min=1e-4,
                  tol=TOL, sign_eps=1e-9, sign_free=None, lam0_floor=1e-8):
    """Asserts `got` (ndims, n) matches `want` within the stated bars.

    `lam` is the (3, n) ascending eigenvalue array of the accuracy oracle
    (scale and eigen-gap of each row); rows whose relative gap is below
    `gap_min` are exempt from eigenvector-dependent dimensions.  Rows whose
    smallest eigenvalue is below `lam0_floor` times the largest are exempt
    from Omnivariance and Eigenentropy, which take the cube root or the log
    of it: a zero smallest eigenvalue (collinear neighbours) is exact here but
    rounding noise in the oracle's covariance formed from the coordinates
    (~1e-9 relative for the FP64 oracle, ~1e-7 for the reference's
    float-narrowed one)."""
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
    flat0 = (lam[0] < lam0_floor * lmax) if lam is not None else np.zeros(n, bool)
    if opts.kind == abi.STAGE_NORMAL:
        flat = np.zeros(n, bool)
        if opts.always_up and not opts.has_viewpoint:
            flat = np.abs(want[2]) < sign_eps
        if sign_free is True:
            flat = np.ones(n, bool)
        elif sign_free is not None:
            flat = flat | sign_free
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
            bar = np.where(flat0[ok], np.inf, tol * ls)
        elif name == "Eigenentropy":
            bar = np.where(flat0[ok], np.inf,
                           tol * np.maximum(np.abs(w), ls * (1.0 + np.abs(np.log(np.maximum(ls, 1e-300))))))
        elif name == "EigenvalueSum":
            bar = tol * np.abs(w)
        elif name == "SurfaceVariation":
            # lambda2 / raw sum: in normalized mode the normalized lambda2 over
            # the raw sum, which is not bounded by 1 (CovarianceFeaturesFilter.cpp:255,339)
            bar = tol * np.maximum(1.0, np.abs(w))
        elif name == "Density":
            bar = 1e-9 * np.abs(w)
        else:
            bar = tol
        err = np.abs(g - w)
        bad = fin & ~(err <= bar)
        if bad.any():
            rows = np.flatnonzero(ok)[bad][:4]
            raise AssertionError(f"{label}:{name} {bad.sum()} rows over the bar, max err "
                                 f"{err[fin].max():.3e}; first rows {rows.tolist()} got "
                                 f"{g[bad][:4].tolist()} want {w[bad][:4].tolist()}")


def status_from_exceptions(n, ex, stage=0):
    s = np.zeros(n, np.uint8)
    e = ex[ex["stage"] == stage]
    s[e["point_id"]] = e["code"]
    return s

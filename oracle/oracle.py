"""ctypes wrapper of the CPU oracle (oracle/cbct_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The CUDA product path never
imports this module.

Parity status: unpinned against the reference's own outputs (the reference
cannot be built here; it ships no golden vectors).  Pinned by closed-form
known answers and by the fixtures under tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


class Geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("W", C.c_int), ("H", C.c_int),
                ("fov_u", C.c_double), ("fov_v", C.c_double),
                ("SAD", C.c_double), ("SDD", C.c_double)]


@dataclass
class Geometry:
    """Cone-beam geometry in the units of CBCT_geometry (mm, degrees)."""
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    W: int
    H: int
    fov_u: float
    fov_v: float
    SAD: float
    SDD: float

    def c(self) -> Geom:
        return Geom(self.nx, self.ny, self.nz, self.lx, self.ly, self.lz,
                    self.W, self.H, self.fov_u, self.fov_v, self.SAD, self.SDD)


_P = np.ctypeslib.ndpointer
_f32 = _P(dtype=np.float32, flags="C_CONTIGUOUS")
_f64 = _P(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = _P(dtype=np.int32, flags="C_CONTIGUOUS")
_GP = C.POINTER(Geom)


def _declare(L):
    L.oracle_forward_f64.argtypes = [_GP, _f32, _f32, C.c_int, C.c_double, C.c_int, _f64, _f64, C.c_int]
    L.oracle_forward_f32.argtypes = [_GP, _f32, _f32, C.c_int, C.c_double, C.c_int, _f32, _f32, C.c_int]
    L.oracle_backproject_f64.argtypes = [_GP, _f32, _f32, C.c_int, C.c_int, C.c_int, _f64, _f64, C.c_int]
    L.oracle_backproject_f32.argtypes = [_GP, _f32, _f32, C.c_int, C.c_int, C.c_int, _f32, _f32, C.c_int]
    L.oracle_samples_per_ray.argtypes = [_GP, C.c_double]
    L.oracle_offset_weight.argtypes = [_GP, _f32, C.c_int, C.c_int, _f64]
    L.oracle_parker_weight.argtypes = [_GP, _f32, C.c_int, _f64]
    L.oracle_cosine_weights.argtypes = [_GP, _f64]
    L.oracle_default_filter.argtypes = [C.c_int, _f64]
    L.oracle_fdk_filter_rows.argtypes = [C.c_int, C.c_long, _f64, _f64]
    L.oracle_is_short_scan.argtypes = [_GP, _f32, C.c_int]
    L.oracle_fdk.argtypes = [_GP, _f32, _f32, C.c_int, C.c_int, C.c_int, _f64, _f64, _f64]
    L.oracle_subset_partition.argtypes = [C.c_int, _i32, C.c_int, _i32, _i32]
    L.oracle_osmom.argtypes = [_GP, _f32, _f32, _i32, _i32, C.c_int, C.c_double, C.c_int,
                               C.c_double, C.c_double, C.c_int, C.c_void_p, _f64, _f64, C.c_void_p]
    L.oracle_ossart.argtypes = L.oracle_osmom.argtypes
    L.oracle_phantom_voxelize.argtypes = [_f64, C.c_int, _GP, C.c_int, _f64]
    L.oracle_phantom_project.argtypes = [_f64, C.c_int, _GP, _f32, _f32, C.c_int, _f64]
    L.oracle_set_num_threads.argtypes = [C.c_int]
    L.oracle_set_solver_mask.argtypes = [C.c_void_p]
    L.oracle_set_solver_weights.argtypes = [C.c_void_p]
    L.oracle_set_solver_bins.argtypes = [C.c_int, C.c_void_p]
    L.oracle_set_solver_tv.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int]
    L.oracle_set_solver_snapshots.argtypes = [C.c_void_p]
    L.oracle_spacecarver.argtypes = [_GP, _f32, _f32, C.c_int, _f64, C.c_double,
                                     _P(dtype=np.uint8, flags="C_CONTIGUOUS")]


def _views(angles, offsets):
    a = np.ascontiguousarray(angles, dtype=np.float32)
    o = np.ascontiguousarray(offsets, dtype=np.float32).reshape(-1)
    assert o.size == 2 * a.size
    return a, o


def forward(g: Geometry, vol, angles, offsets, spp=1.5, mode=0, dtype=np.float64,
            out=None, accumulate=False):
    """mult_M of one set of views: returns projections of shape (P, H, W)."""
    a, o = _views(angles, offsets)
    P = a.size
    vol = np.ascontiguousarray(vol, dtype=dtype)
    if out is None:
        out = np.zeros((P, g.H, g.W), dtype=dtype)
    fn = lib().oracle_forward_f64 if dtype == np.float64 else lib().oracle_forward_f32
    fn(C.byref(g.c()), a, o, P, spp, mode, vol, out, int(accumulate))
    return out


def backproject(g: Geometry, proj, angles, offsets, fbp=False, mode=0, dtype=np.float64,
                out=None, accumulate=False):
    """mult_MH of one set of views: returns a volume of shape (nz, ny, nx)."""
    a, o = _views(angles, offsets)
    proj = np.ascontiguousarray(proj, dtype=dtype)
    if out is None:
        out = np.zeros((g.nz, g.ny, g.nx), dtype=dtype)
    fn = lib().oracle_backproject_f64 if dtype == np.float64 else lib().oracle_backproject_f32
    fn(C.byref(g.c()), a, o, a.size, int(fbp), mode, proj, out, int(accumulate))
    return out


def samples_per_ray(g: Geometry, spp=1.5) -> int:
    return lib().oracle_samples_per_ray(C.byref(g.c()), spp)


def offset_weight(g: Geometry, proj, offsets, variant: int):
    """variant 0: sin^2 weight with zeroing (BP/FDK); 1: sqrt (sin) weight."""
    p = np.ascontiguousarray(proj, dtype=np.float64).copy()
    o = np.ascontiguousarray(offsets, dtype=np.float32).reshape(-1)
    lib().oracle_offset_weight(C.byref(g.c()), o, o.size // 2, variant, p)
    return p


def parker_weight(g: Geometry, proj, angles):
    p = np.ascontiguousarray(proj, dtype=np.float64).copy()
    a = np.ascontiguousarray(angles, dtype=np.float32)
    lib().oracle_parker_weight(C.byref(g.c()), a, a.size, p)
    return p


def cosine_weights(g: Geometry):
    w = np.zeros((g.H, g.W), dtype=np.float64)
    lib().oracle_cosine_weights(C.byref(g.c()), w)
    return w


def default_filter(W: int):
    h = np.zeros(W + 1, dtype=np.float64)
    lib().oracle_default_filter(W, h)
    return h


def fdk_filter_rows(proj, filt):
    p = np.ascontiguousarray(proj, dtype=np.float64).copy()
    W = p.shape[-1]
    f = np.ascontiguousarray(filt, dtype=np.float64)
    assert f.size == W + 1
    lib().oracle_fdk_filter_rows(W, p.size // W, f, p)
    return p


def is_short_scan(g: Geometry, angles) -> bool:
    a = np.ascontiguousarray(angles, dtype=np.float32)
    return bool(lib().oracle_is_short_scan(C.byref(g.c()), a, a.size))


def fdk(g: Geometry, proj, angles, offsets, short_scan=False, offset_corr=False, filt=None):
    a, o = _views(angles, offsets)
    f = default_filter(g.W) if filt is None else np.ascontiguousarray(filt, dtype=np.float64)
    p = np.ascontiguousarray(proj, dtype=np.float64)
    out = np.zeros((g.nz, g.ny, g.nx), dtype=np.float64)
    lib().oracle_fdk(C.byref(g.c()), a, o, a.size, int(short_scan), int(offset_corr), f, p, out)
    return out


def fdk_recipe(g: Geometry, proj, angles, offsets, filt=None):
    """FDK_reconstruct_3d.cpp:152-161: FDK (hoCuConebeamProjectionOperator
    mult_MH with filtered back-projection), then x *= <A x, p> / <A x, A x>
    with A the operator's mult_M (no offset weight in FBP mode)."""
    x = fdk(g, proj, angles, offsets, filt=filt)
    ax = forward(g, x, angles, offsets)
    p = np.asarray(proj, dtype=np.float64)
    return x * (np.vdot(ax, p) / np.vdot(ax, ax))


def subset_partition(n_views: int, n_subsets: int, view_bin=None):
    vb = np.zeros(n_views, dtype=np.int32) if view_bin is None else np.ascontiguousarray(view_bin, dtype=np.int32)
    order = np.zeros(n_views, dtype=np.int32)
    sizes = np.zeros(n_subsets, dtype=np.int32)
    n = lib().oracle_subset_partition(n_views, vb, n_subsets, order, sizes)
    return order[:n], sizes


def _solver(fn, g, b, angles, offsets, sizes, offcorr, iters, beta, gamma, nonneg, x0, spp, ntrace, n_bins=1):
    a, o = _views(angles, offsets)
    sizes = np.ascontiguousarray(sizes, dtype=np.int32)
    oc = np.ascontiguousarray(offcorr, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros(((n_bins,) if n_bins > 1 else ()) + (g.nz, g.ny, g.nx), dtype=np.float64)
    trace = np.zeros(ntrace, dtype=np.float64)
    x0p = None
    if x0 is not None:
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        x0p = x0.ctypes.data
    fn(C.byref(g.c()), a, o, sizes, oc, sizes.size, spp, iters, beta, gamma, int(nonneg), x0p,
       b, out, trace.ctypes.data)
    return out, trace


def osmom(g, b, angles, offsets, sizes, offcorr, iters=10, beta=1.0, gamma=0.0, nonneg=False,
          x0=None, spp=1.5, mask=None, weights=None, view_bin=None, n_bins=1, tv_weight=0.0, tv_alpha=0.0,
          tau=1e-3, reg_steps=1, snapshots=None):
    """osMOMSolverD::solve (no regulariser); returns (z, per-step ||r||^2).
    mask: optional uint8 voxel mask applied after every mult_MH; weights:
    optional projection weights of CBSubsetWeightOperator (subset order);
    view_bin: bin of every view (subset order, each subset sorted by bin) for
    n_bins volumes (z then has shape (n_bins, nz, ny, nx)); tv_weight > 0: the
    TV-regularised solver (one cuTVPrimalDualOperator(tv_alpha) of that weight,
    the solver's tau and reg_steps); snapshots: float64 array of shape
    (iters,) + z.shape that receives z after every iteration."""
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    vb = None if view_bin is None else np.ascontiguousarray(view_bin, dtype=np.int32)
    lib().oracle_set_solver_mask(None if m is None else m.ctypes.data)
    lib().oracle_set_solver_weights(None if w is None else w.ctypes.data)
    lib().oracle_set_solver_bins(int(n_bins), None if vb is None else vb.ctypes.data)
    lib().oracle_set_solver_tv(float(tv_weight), float(tv_alpha), float(tau), int(reg_steps))
    if snapshots is not None:
        assert snapshots.dtype == np.float64 and snapshots.flags["C_CONTIGUOUS"] and snapshots.shape[0] >= iters
    lib().oracle_set_solver_snapshots(None if snapshots is None else snapshots.ctypes.data)
    try:
        return _solver(lib().oracle_osmom, g, b, angles, offsets, sizes, offcorr, iters, beta, gamma,
                       nonneg, x0, spp, iters * len(sizes), n_bins if vb is not None else 1)
    finally:
        lib().oracle_set_solver_mask(None)
        lib().oracle_set_solver_weights(None)
        lib().oracle_set_solver_bins(1, None)
        lib().oracle_set_solver_tv(0.0, 0.0, 1e-3, 1)
        lib().oracle_set_solver_snapshots(None)


def ossart(g, b, angles, offsets, sizes, offcorr, iters=10, beta=1.0, gamma=0.0, nonneg=False,
           x0=None, spp=1.5, weights=None):
    """osSARTSolver::solve; returns (x, per-iteration ||Ax-b||^2)."""
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    lib().oracle_set_solver_weights(None if w is None else w.ctypes.data)
    try:
        return _solver(lib().oracle_ossart, g, b, angles, offsets, sizes, offcorr, iters, beta, gamma,
                       nonneg, x0, spp, iters)
    finally:
        lib().oracle_set_solver_weights(None)


def phantom_voxelize(g: Geometry, ell, ss=4):
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    out = np.zeros((g.nz, g.ny, g.nx), dtype=np.float64)
    lib().oracle_phantom_voxelize(e.reshape(-1), e.shape[0], C.byref(g.c()), ss, out)
    return out


def phantom_project(g: Geometry, ell, angles, offsets):
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    a, o = _views(angles, offsets)
    out = np.zeros((a.size, g.H, g.W), dtype=np.float64)
    lib().oracle_phantom_project(e.reshape(-1), e.shape[0], C.byref(g.c()), a, o, a.size, out)
    return out


def spacecarver(g: Geometry, proj, angles, offsets, limit: float):
    """conebeam_spacecarver: uint8 mask (nz, ny, nx), 1 where fewer than 3 views
    see a nonzero value below `limit`."""
    a, o = _views(angles, offsets)
    p = np.ascontiguousarray(proj, dtype=np.float64)
    out = np.zeros((g.nz, g.ny, g.nx), dtype=np.uint8)
    lib().oracle_spacecarver(C.byref(g.c()), a, o, a.size, p, float(limit), out)
    return out


def set_num_threads(n: int):
    lib().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return lib().oracle_num_threads()


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))

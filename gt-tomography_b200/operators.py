"""Reference-shaped operator surface over the C ABI.

Mirrors gt-tomography's operator classes for the cone-beam path so that code
written against them reads the same:

  CBCT_geometry / CBCT_acquisition / CBCT_binning   xray/CBCT_acquisition.h:24-340,
                                                    xray/CBCT_binning.h:18-172
  cuConebeamProjectionOperator                      xray/cuConebeamProjectionOperator.{h,cpp}
  CBSubsetOperator                                  xray/CBSubsetOperator.{h,cpp}
  hoCuConebeamProjectionOperator                    xray/hoCuConebeamProjectionOperator.{h,cpp}
  osMOMSolverD                                      solvers/osMOMSolverD.h
  osSARTSolver                                      solvers/osSARTSolver.h
  fdk_reconstruct_3d                                xray/FDK_reconstruct_3d.cpp:135-161

Device arrays are torch CUDA tensors (torch is used for device memory and
streams only); every computation runs in libcbct.so.  Array shapes are the
reverse of Gadgetron's dimension lists: a volume of Gadgetron dims
(nx, ny, nz) is a tensor of shape (nz, ny, nx); projections (W, H, P) are
(P, H, W).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

_torch = None


def torch():
    global _torch
    if _torch is None:
        import torch as t
        _torch = t
    return _torch


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _stream(stream=None) -> int:
    if stream is not None:
        return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)
    return int(torch().cuda.current_stream().cuda_stream)


def _need_cuda_f32(t, shape, what):
    T = torch()
    if not isinstance(t, T.Tensor) or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA tensor")
    if t.dtype != T.float32:
        raise TypeError(f"{what} must be float32, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what} has shape {tuple(t.shape)}, expected {tuple(shape)}")


def _dtype_code(dtype) -> int:
    """cbct_dtype of a torch dtype (float32, float16, bfloat16)."""
    T = torch()
    codes = {T.float32: L.CBCT_F32, T.float16: L.CBCT_F16, T.bfloat16: L.CBCT_BF16}
    if dtype not in codes:
        raise TypeError(f"storage type must be float32, float16 or bfloat16, got {dtype}")
    return codes[dtype]


def _storage_of(t, shape, what) -> int:
    """Checks a contiguous CUDA tensor of the given shape; returns its cbct_dtype."""
    T = torch()
    if not isinstance(t, T.Tensor) or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA tensor")
    code = _dtype_code(t.dtype)
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return code


# ----------------------------------------------------------------- data model
@dataclass
class CBCT_geometry:
    """CBCT_geometry (xray/CBCT_acquisition.h:24-120): mm and degrees."""
    SAD: float = 0.0
    SDD: float = 0.0
    FOV: tuple = (0.0, 0.0)
    angles: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    offsets: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))

    def get_angles(self):
        return self.angles

    def set_angles(self, a):
        self.angles = np.asarray(a, dtype=np.float32).copy()

    def get_offsets(self):
        return self.offsets

    def set_offsets(self, o):
        self.offsets = np.asarray(o, dtype=np.float32).reshape(-1, 2).copy()


@dataclass
class CBCT_acquisition:
    """CBCT_acquisition: geometry plus projections of shape (P, H, W) (host, float32)."""
    geometry: CBCT_geometry
    projections: Optional[np.ndarray] = None

    def get_geometry(self):
        return self.geometry

    def get_projections(self):
        return self.projections

    def set_projections(self, p):
        self.projections = p

    def load(self, filename):
        """CBCT_acquisition::load (xray/CBCT_acquisition.h:178-303): the HDF5
        acquisition layout, geometry version 2, projection version 1."""
        from .acquisition_io import load_acquisition
        SAD, SDD, fov, angles, offsets, proj = load_acquisition(filename)
        self.geometry = CBCT_geometry(SAD, SDD, (float(fov[0]), float(fov[1])), angles, offsets)
        self.projections = proj

    def save(self, filename):
        """CBCT_acquisition::save (xray/CBCT_acquisition.h:305-322)."""
        from .acquisition_io import save_acquisition
        g = self.geometry
        save_acquisition(filename, g.SAD, g.SDD, g.FOV, g.angles, g.offsets, self.projections)

    @classmethod
    def from_file(cls, filename):
        acq = cls(CBCT_geometry())
        acq.load(filename)
        return acq


class CBCT_binning:
    """CBCT_binning (xray/CBCT_binning.h:18-172): lists of view indices per bin."""

    def __init__(self, bins: Optional[Sequence[Sequence[int]]] = None):
        self.bins = [list(map(int, b)) for b in (bins or [])]

    def set_as_default_3d_bin(self, n: int):
        self.bins = [list(range(n))]

    def get_number_of_bins(self) -> int:
        return len(self.bins)

    def get_bin(self, b: int):
        return self.bins[b]

    def get_bins(self):
        return self.bins

    def get_3d_binning(self):
        allv = sorted({v for b in self.bins for v in b})
        return CBCT_binning([allv])

    def load(self, filename):
        """CBCT_binning::load (xray/CBCT_binning.h:106-148)."""
        from .acquisition_io import load_binning
        self.bins = load_binning(filename)

    def save(self, filename):
        from .acquisition_io import save_binning
        save_binning(filename, self.bins)


# ----------------------------------------------------------------- host helpers
def _cgeom(acq_geom: CBCT_geometry, W: int, H: int, is_dims, is_dims_in_mm, spp: float) -> L.CbctGeometry:
    nx, ny, nz = (int(v) for v in is_dims)
    lx, ly, lz = (float(v) for v in is_dims_in_mm)
    return L.CbctGeometry(float(acq_geom.SAD), float(acq_geom.SDD), float(acq_geom.FOV[0]),
                          float(acq_geom.FOV[1]), int(W), int(H), nx, ny, nz, lx, ly, lz, float(spp))


def subset_partition(n_views: int, n_subsets: int, view_bin=None):
    """CBSubsetOperator::setup's subset assignment (CBSubsetOperator.cpp:66-104)."""
    vb = None if view_bin is None else np.ascontiguousarray(view_bin, dtype=np.int32)
    order = np.zeros(max(n_views, 1), np.int32)
    sizes = np.zeros(n_subsets, np.int32)
    n = C.c_int32()
    L.call("cbct_subset_partition", n_views, None if vb is None else vb.ctypes.data, n_subsets,
           order.ctypes.data, sizes.ctypes.data, C.byref(n))
    return order[:n.value], sizes


def default_frequency_filter(W: int) -> np.ndarray:
    out = np.zeros(W + 1, np.float32)
    L.call("cbct_default_frequency_filter", W, out.ctypes.data)
    return out


def cosine_weights(g: L.CbctGeometry) -> np.ndarray:
    out = np.zeros((g.height, g.width), np.float32)
    L.call("cbct_cosine_weights", C.byref(g), out.ctypes.data)
    return out


def is_short_scan(g: L.CbctGeometry, angles) -> bool:
    a = np.ascontiguousarray(angles, np.float32)
    r = C.c_int32()
    L.call("cbct_is_short_scan", C.byref(g), a.ctypes.data, a.size, C.byref(r))
    return bool(r.value)


def offset_override(g: L.CbctGeometry, offsets) -> bool:
    o = np.ascontiguousarray(offsets, np.float32).reshape(-1)
    r = C.c_int32()
    L.call("cbct_offset_override", C.byref(g), o.ctypes.data, o.size // 2, C.byref(r))
    return bool(r.value)


def hann_ramp_filter(W: int) -> np.ndarray:
    """Hann-windowed ramp on the W+1 bins of the FDK filter, normalised like the
    default filter (absolute sum W+1; hoCuConebeamProjectionOperator.cpp:59-61)."""
    k = np.arange(W + 1, dtype=np.float64)
    h = k * 0.5 * (1.0 + np.cos(np.pi * k / W))
    return (h * ((W + 1) / np.abs(h).sum())).astype(np.float32)


# ----------------------------------------------------------------- plans
class Plan:
    """A device-resident geometry (cbct_plan) for views in subset-contiguous order."""

    def __init__(self, g: L.CbctGeometry, angles, offsets, subset_sizes=None, offset_correction=None):
        self.g = g
        self.angles = np.ascontiguousarray(angles, np.float32)
        self.offsets = np.ascontiguousarray(offsets, np.float32).reshape(-1, 2)
        P = self.angles.size
        assert self.offsets.shape[0] == P
        self.subset_sizes = (np.array([P], np.int32) if subset_sizes is None
                             else np.ascontiguousarray(subset_sizes, np.int32))
        S = self.subset_sizes.size
        oc = (np.zeros(S, np.int32) if offset_correction is None
              else np.ascontiguousarray(offset_correction, np.int32))
        self.offset_correction = oc
        h = C.c_void_p()
        L.call("cbct_plan_create", C.byref(g), self.angles.ctypes.data, self.offsets.ctypes.data, P,
               self.subset_sizes.ctypes.data, S, oc.ctypes.data, C.byref(h))
        self._h = h
        self.n_views = P
        self.n_subsets = S
        self.n_bins = 1
        self.first = np.concatenate([[0], np.cumsum(self.subset_sizes)[:-1]]).astype(np.int64)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib().cbct_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def vol_shape(self):
        """(nz, ny, nx), or (bins, nz, ny, nx) for a binned plan."""
        v = (self.g.nz, self.g.ny, self.g.nx)
        return ((self.n_bins,) + v) if getattr(self, "n_bins", 1) > 1 else v

    def set_bins(self, view_bin, n_bins: int):
        """Bins of the plan's views (cbct_plan_set_bins): view_bin per view in
        plan order, the views of a bin contiguous within every subset; volumes
        then hold n_bins images.  n_bins <= 1 or None returns to one bin."""
        if view_bin is None or int(n_bins) <= 1:
            L.call("cbct_plan_set_bins", self._h, 1, None)
            self.n_bins = 1
            return
        vb = np.ascontiguousarray(view_bin, np.int32)
        if vb.size != self.n_views:
            raise ValueError("view_bin needs one entry per view")
        L.call("cbct_plan_set_bins", self._h, int(n_bins), vb.ctypes.data)
        self.n_bins = int(n_bins)
        self.view_bin = vb

    def proj_shape(self, s=-1):
        n = self.n_views if s < 0 else int(self.subset_sizes[s])
        return (n, self.g.height, self.g.width)

    def forward_variant(self) -> str:
        return L.lib().cbct_plan_forward_variant(self._h).decode()

    def set_option(self, opt: int, value: int):
        L.call("cbct_plan_set_option", self._h, opt, int(value))

    def autotune(self, stream=None) -> dict:
        """cbct_plan_autotune: times the projector variants on the largest
        subset, keeps the fastest; returns ms per launch (None: unavailable)."""
        t = np.zeros(7, np.float32)
        L.call("cbct_plan_autotune", self._h, t.ctypes.data, _stream(stream))
        names = ["forward_slab", "forward_fan", "forward_gather", "backproject_tma", "backproject_global",
                 "forward_pair", "forward_quad"]
        out = {n: (float(v) if v >= 0 else None) for n, v in zip(names, t)}
        out["forward_variant"] = self.forward_variant()
        return out

    def read_flags(self, reset=True):
        f = (C.c_int32 * 2)()
        L.call("cbct_plan_read_flags", self._h, C.cast(f, C.c_void_p), int(reset))
        return int(f[0]), int(f[1])

    def check(self, stream=None):
        """cbct_plan_check: raises CbctError (CBCT_ERR_TIMEOUT, CBCT_ERR_DEVICE_CHECK)
        when a kernel of this plan gave up a bounded wait or recorded a range
        violation since the last check; clears the flags."""
        L.call("cbct_plan_check", self._h, _stream(stream))

    # -- operators
    def forward(self, vol, out, s=-1, accumulate=False, vol_dtype=L.CBCT_F32, stream=None):
        T = torch()
        if vol_dtype == L.CBCT_F32:
            _need_cuda_f32(vol, self.vol_shape, "volume")
        else:
            want = T.float16 if vol_dtype == L.CBCT_F16 else T.bfloat16
            if vol.dtype != want or tuple(vol.shape) != self.vol_shape or not vol.is_contiguous():
                raise TypeError("volume does not match vol_dtype/shape")
        _need_cuda_f32(out, self.proj_shape(s), "projections")
        L.call("cbct_forward", self._h, s, vol_dtype, _ptr(vol), _ptr(out), int(accumulate), _stream(stream))
        return out

    def backproject(self, proj, out, s=-1, flags=0, use_plan_offset=True, accumulate=False, stream=None):
        _need_cuda_f32(proj, self.proj_shape(s), "projections")
        _need_cuda_f32(out, self.vol_shape, "volume")
        L.call("cbct_backproject", self._h, s, _ptr(proj), _ptr(out), flags, int(use_plan_offset),
               int(accumulate), _stream(stream))
        return out

    def offset_correct(self, proj, s=-1, variant=1, stream=None):
        _need_cuda_f32(proj, self.proj_shape(s), "projections")
        L.call("cbct_offset_correct", self._h, s, _ptr(proj), variant, _stream(stream))
        return proj

    def fdk_filter(self, proj_in, proj_out, s=-1, filt=None, flags=L.CBCT_FDK_RAMP | L.CBCT_FDK_COSINE,
                   stream=None):
        _need_cuda_f32(proj_in, self.proj_shape(s), "projections")
        _need_cuda_f32(proj_out, self.proj_shape(s), "projections")
        f = None if filt is None else np.ascontiguousarray(filt, np.float32)
        if f is not None and f.size != self.g.width + 1:
            raise ValueError("filter must have W+1 entries")
        L.call("cbct_fdk_filter", self._h, s, _ptr(proj_in), _ptr(proj_out),
               None if f is None else f.ctypes.data, flags, _stream(stream))
        return proj_out

    def fdk(self, proj, out, filt=None, flags=0, work=None, stream=None):
        """FDK of every view (cbct_fdk / cbct_fdk_ex): proj may be float32,
        float16 or bfloat16 (the storage type); arithmetic is FP32."""
        dt = _storage_of(proj, self.proj_shape(-1), "projections")
        _need_cuda_f32(out, self.vol_shape, "volume")
        f = None if filt is None else np.ascontiguousarray(filt, np.float32)
        L.call("cbct_fdk_ex", self._h, dt, _ptr(proj), _ptr(out), None if f is None else f.ctypes.data, flags,
               _ptr(work), _stream(stream))
        return out

    def forward_residual(self, vol, b, r, s=-1, scale=1.0, apply_offset=False, norm2=None,
                         vol_dtype=L.CBCT_F32, stream=None):
        _need_cuda_f32(b, self.proj_shape(s), "b")
        _need_cuda_f32(r, self.proj_shape(s), "r")
        L.call("cbct_forward_residual", self._h, s, vol_dtype, _ptr(vol), _ptr(b), _ptr(r), float(scale),
               int(apply_offset), _ptr(norm2), _stream(stream))
        return r

    def spacecarver(self, proj, limit, mask, s=-1, combine=False, stream=None):
        """conebeam_spacecarver over subset s: uint8 mask, 1 = keep."""
        _need_cuda_f32(proj, self.proj_shape(s), "projections")
        L.call("cbct_spacecarver", self._h, s, _ptr(proj), float(limit), _ptr(mask), int(combine), _stream(stream))
        return mask

    def set_projection_weights(self, weights):
        """Projection weights of CBSubsetWeightOperator (device tensor of the
        plan's projection shape, subset order; None clears)."""
        if weights is not None:
            _need_cuda_f32(weights, self.proj_shape(), "weights")
        self._pweights = weights
        L.call("cbct_plan_set_projection_weights", self._h, _ptr(weights))

    def set_mask(self, mask):
        """Mask applied to the output of every back-projection (None clears it).
        The plan keeps a reference so the mask stays alive while it is used."""
        self._mask = mask
        L.call("cbct_plan_set_mask", self._h, _ptr(mask))

    def phantom_project(self, ell_dev, out, s=-1, stream=None):
        _need_cuda_f32(out, self.proj_shape(s), "projections")
        n = ell_dev.numel() // 10
        L.call("cbct_phantom_project", self._h, s, _ptr(ell_dev), n, _ptr(out), _stream(stream))
        return out

    def osmom(self, b, z_out, x0=None, iterations=10, beta=1.0, gamma=0.0, nonneg=False, use_graph=False,
              storage=L.CBCT_F32, refine_every=0, resid=None, stream=None, tv_weight=0.0, tv_alpha=0.0,
              tau=1e-3, reg_steps=1):
        """osMOMSolverD::solve on the device.  storage: type of the forward
        projector's volume input (16-bit shadow of z); b may be float32,
        float16 or bfloat16 (its storage type is taken from the tensor).
        tv_weight > 0: TV regularisation (a cuTVPrimalDualOperator(tv_alpha) of
        that weight, the solver's tau and reg_steps)."""
        bt = _storage_of(b, self.proj_shape(-1), "b")
        prm = L.CbctSolverParams(int(iterations), float(beta), float(gamma), int(nonneg), int(use_graph),
                                 int(storage), int(refine_every), bt, float(tv_weight), float(tv_alpha), float(tau),
                                 int(reg_steps))
        L.call("cbct_osmom_solve", self._h, _ptr(b), _ptr(x0), _ptr(z_out), C.byref(prm), _ptr(resid),
               _stream(stream))
        return z_out

    def osmom_precon(self, out, stream=None):
        """cbct_osmom_precon: out = 1/max(A^T W A 1, 1e-6) (osMOMSolverD.h:115-120)."""
        _need_cuda_f32(out, self.vol_shape, "preconditioner")
        L.call("cbct_osmom_precon", self._h, _ptr(out), _stream(stream))
        return out

    def osmom_step(self, s, b_s, z, xold, precon, r_work, step, mom, nonneg=False, norm2=None, stream=None):
        """cbct_osmom_step: one subset step of osMOMSolverD (residual forward
        projection, then the back-projection with the fused update of z, xold)."""
        bt = _storage_of(b_s, self.proj_shape(s), "b_s")
        for t, what in ((z, "z"), (xold, "xold"), (precon, "precon")):
            _need_cuda_f32(t, self.vol_shape, what)
        _need_cuda_f32(r_work, self.proj_shape(s), "r_work")
        L.call("cbct_osmom_step", self._h, int(s), bt, _ptr(b_s), _ptr(z), _ptr(xold), _ptr(precon), _ptr(r_work),
               float(step), float(mom), int(nonneg), _ptr(norm2), _stream(stream))

    def ossart(self, b, x_out, x0=None, iterations=10, beta=1.0, gamma=0.0, nonneg=False, use_graph=False,
               cost=None, stream=None):
        prm = L.CbctSolverParams(int(iterations), float(beta), float(gamma), int(nonneg), int(use_graph),
                                 L.CBCT_F32, 0, L.CBCT_F32)
        L.call("cbct_ossart_solve", self._h, _ptr(b), _ptr(x0), _ptr(x_out), C.byref(prm), _ptr(cost),
               _stream(stream))
        return x_out


def phantom_voxelize(g: L.CbctGeometry, ell_dev, out, supersample=4, stream=None):
    _need_cuda_f32(out, (g.nz, g.ny, g.nx), "volume")
    n = ell_dev.numel() // 10
    L.call("cbct_phantom_voxelize", C.byref(g), _ptr(ell_dev), n, int(supersample), _ptr(out), _stream(stream))
    return out


def reduce_f64(kind: int, a, b=None, stream=None):
    """kind 0 = dot(a,b), 1 = sum of squares, 2 = asum; returns a CUDA float64 scalar tensor."""
    T = torch()
    out = T.zeros(1, dtype=T.float64, device=a.device)
    L.call("cbct_reduce_f64", kind, _ptr(a), _ptr(b), a.numel(), _ptr(out), _stream(stream))
    return out


def osmom_update(z, xold, precon, g, step, mom, nonneg=False, stream=None):
    L.call("cbct_osmom_update", _ptr(z), _ptr(xold), _ptr(precon), _ptr(g), z.numel(), float(step), float(mom),
           int(nonneg), _stream(stream))


def batch_osmom(jobs, n_streams=8, stream=None, fused=False):
    """Solves independent OS-MOM problems concurrently (cbct_batch_osmom).

    jobs: sequence of dicts with keys plan, b, z (outputs) and optionally x0,
    iterations, beta, gamma, nonneg, storage, refine_every, resid.  Each result
    is bitwise identical to solving that job alone.  Starts after the work on
    the current stream and returns when every job has finished.

    fused=True advances the jobs in two lockstep groups through persistent
    work-list launches captured in one graph (cbct_batch_osmom_fused; fp32
    volume storage); n_streams is then unused."""
    items = (L.CbctBatchItem * len(jobs))()
    for i, j in enumerate(jobs):
        prm = L.CbctSolverParams(int(j.get("iterations", 10)), float(j.get("beta", 1.0)), float(j.get("gamma", 0.0)),
                                 int(j.get("nonneg", False)), 1, int(j.get("storage", L.CBCT_F32)),
                                 int(j.get("refine_every", 0)),
                                 _storage_of(j["b"], j["plan"].proj_shape(-1), "b"))
        items[i] = L.CbctBatchItem(j["plan"].handle.value, _ptr(j["b"]), _ptr(j.get("x0")), _ptr(j["z"]), prm,
                                   _ptr(j.get("resid")))
    if fused:
        L.call("cbct_batch_osmom_fused", items, len(jobs), _stream(stream))
    else:
        L.call("cbct_batch_osmom", items, len(jobs), int(n_streams), _stream(stream))


def tv_step(x, P, s, D, scale, tau, tau_lambda, stream=None):
    """One primal-dual step of the TV regulariser (cbct_tv_step): x, s, D of
    shape (nz, ny, nx), P of shape (3, nz, ny, nx); x is updated in place."""
    nz, ny, nx = x.shape
    for t, shp, what in ((x, x.shape, "x"), (s, x.shape, "s"), (D, x.shape, "D"), (P, (3,) + tuple(x.shape), "P")):
        _need_cuda_f32(t, shp, what)
    L.call("cbct_tv_step", _ptr(x), _ptr(P), _ptr(s), _ptr(D), nx, ny, nz, float(scale), float(tau),
           float(tau_lambda), _stream(stream))
    return x


def apply_mask(vol, mask, stream=None):
    """apply_mask (conebeam_projection.cu:1651-1657): vol *= mask."""
    L.call("cbct_apply_mask", _ptr(vol), _ptr(mask), vol.numel(), _stream(stream))
    return vol


def convert(src, dst, dtype, stream=None):
    L.call("cbct_convert", _ptr(src), _ptr(dst), src.numel(), dtype, _stream(stream))
    return dst


# ----------------------------------------------------------------- operators
class cuConebeamProjectionOperator:
    """Device-array cone-beam operator of one bin set (cuConebeamProjectionOperator.h:21-53).

    Differences from the reference, on purpose: use_offset_correction starts
    False (the reference leaves it uninitialised unless the override fires,
    .cpp:15-21), and the default binning holds every view (the reference sizes
    it from an empty member vector, .cpp:183-187)."""

    def __init__(self):
        self.samples_per_pixel = 1.5
        self.allow_offset_correction_override = True
        self.use_offset_correction = False
        self.short_scan = False
        self.preprocessed = False
        self.domain_dims = None
        self.plans = []
        self.mask = None

    def setup(self, acquisition: CBCT_acquisition, binning: Optional[CBCT_binning] = None,
              is_dims_in_mm=None, transform_angles: bool = True, is_dims=None):
        """cuConebeamProjectionOperator::setup (.cpp:148-206)."""
        geo = acquisition.geometry
        angles = geo.angles
        if transform_angles:
            geo.set_angles(angles - angles.min())
        g0 = _cgeom(geo, 1, 1, (1, 1, 1), (1, 1, 1), self.samples_per_pixel)
        self.short_scan = is_short_scan(g0, geo.angles)
        if self.allow_offset_correction_override and offset_override(g0, geo.offsets):
            self.use_offset_correction = True
        self.binning = binning if binning is not None else CBCT_binning([list(range(geo.angles.size))])
        self.acquisition = acquisition
        self.is_dims_in_mm = tuple(float(v) for v in is_dims_in_mm)
        self.bin_angles = [geo.angles[np.asarray(b, np.int64)] for b in self.binning.bins]
        self.bin_offsets = [geo.offsets[np.asarray(b, np.int64)] for b in self.binning.bins]
        proj = acquisition.projections
        if proj is not None:
            order = np.asarray([v for b in self.binning.bins for v in b], np.int64)
            acquisition.set_projections(np.ascontiguousarray(proj[order]))
        self.preprocessed = True
        if is_dims is not None:
            self.set_domain_dimensions(is_dims)

    def set_domain_dimensions(self, dims):
        """dims in Gadgetron order: (nx, ny, nz[, bins])."""
        self.domain_dims = tuple(int(d) for d in dims)
        self._make_plans()

    def _make_plans(self):
        if not self.preprocessed or self.domain_dims is None:
            return
        for p in self.plans:
            p.close()
        self.plans = []
        proj = self.acquisition.projections
        H, W = (proj.shape[1], proj.shape[2]) if proj is not None else self._detector
        for a, o in zip(self.bin_angles, self.bin_offsets):
            g = _cgeom(self.acquisition.geometry, W, H, self.domain_dims[:3], self.is_dims_in_mm,
                       self.samples_per_pixel)
            self.plans.append(Plan(g, a, o, None, [int(self.use_offset_correction)]) if a.size else None)

    def set_detector(self, W: int, H: int):
        self._detector = (H, W)

    def set_use_offset_correction(self, use: bool):
        self.use_offset_correction = bool(use)
        self.allow_offset_correction_override = False
        self._make_plans()

    def get_use_offset_correction(self) -> bool:
        return self.use_offset_correction

    def set_mask(self, mask):
        """cuConebeamProjectionOperator::set_mask: mult_MH applies it (.cpp:113-114)."""
        self.mask = mask
        for pl in self.plans:
            if pl is not None:
                pl.set_mask(mask if mask is None or mask.dim() == 3 else None)

    def calculate_mask(self, projections, limit: float):
        """cuConebeamProjectionOperator::calculate_mask (.cpp:118-147): one space
        carve per bin; returns a uint8 mask of the domain's shape."""
        T = torch()
        masks = []
        for pl, p in zip(self.plans, self._views(projections, True, False)):
            m = T.ones(pl.vol_shape, dtype=T.uint8, device=projections.device)
            if pl is not None:
                pl.spacecarver(p, limit, m)
            masks.append(m)
        return masks[0] if len(masks) == 1 else T.stack(masks)

    def _views(self, arr, per_bin, is_volume):
        out, off = [], 0
        for b, pl in enumerate(self.plans):
            if is_volume:
                out.append(arr[b] if arr.dim() == 4 else arr)
            else:
                n = len(self.binning.bins[b])
                out.append(arr[off:off + n])
                off += n
        return out

    def mult_M(self, x, out, accumulate=False, vol_dtype=L.CBCT_F32):
        """cuConebeamProjectionOperator::mult_M (.cpp:38-80): no offset weight."""
        vols = self._views(x, True, True)
        projs = self._views(out, True, False)
        for pl, v, p in zip(self.plans, vols, projs):
            if pl is not None:
                pl.forward(v, p, -1, accumulate, vol_dtype)
        return out

    def mult_MH(self, proj, out, accumulate=False):
        """cuConebeamProjectionOperator::mult_MH (.cpp:82-116): sin^2 offset weight on a copy."""
        vols = self._views(out, True, True)
        projs = self._views(proj, True, False)
        for pl, v, p in zip(self.plans, vols, projs):
            if pl is not None:
                pl.backproject(p, v, -1, 0, True, accumulate)
        return out

    def offset_correct(self, proj):
        """apply_offset_correct: sqrt (sin) weight in place (conebeam_projection.cu:394-404)."""
        for pl, p in zip(self.plans, self._views(proj, True, False)):
            if pl is not None:
                pl.offset_correct(p, -1, 1)
        return proj


class CBSubsetOperator:
    """Ordered-subset cone-beam operator (CBSubsetOperator.h:30-72) on device arrays."""

    def __init__(self, subsets: int = 1):
        self.number_of_subsets = int(subsets)
        self.samples_per_pixel = 1.5
        self.domain_dims = None
        self.plan: Optional[Plan] = None
        self.use_offset_override = None

    def setup(self, acq: CBCT_acquisition, binning: Optional[CBCT_binning] = None, is_dims_in_mm=None,
              is_dims=None):
        """CBSubsetOperator::setup (.cpp:52-158): permutes the acquisition in place."""
        geo = acq.geometry
        P = geo.angles.size
        if binning is None:
            binning = CBCT_binning([list(range(P))])
        self.n_bins = binning.get_number_of_bins()
        all_angles = geo.angles - geo.angles.min()
        view_bin = np.full(P, -1, np.int32)
        for b, views in enumerate(binning.bins):
            view_bin[np.asarray(views, np.int64)] = b
        order, sizes = subset_partition(P, self.number_of_subsets, view_bin)
        self.permutation = order
        self.subset_sizes = sizes
        self.view_bin = view_bin[order]   # bin of each view in subset order
        if acq.projections is not None:
            acq.set_projections(np.ascontiguousarray(acq.projections[order]))
        geo.set_angles(all_angles[order])
        geo.set_offsets(geo.offsets[order])
        self.acq = acq
        self.is_dims_in_mm = tuple(float(v) for v in is_dims_in_mm)
        # Per-subset offset-correction override (cuConebeamProjectionOperator.cpp:176-181).
        g0 = _cgeom(geo, 1, 1, (1, 1, 1), (1, 1, 1), self.samples_per_pixel)
        first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        self.offcorr = np.array([
            int(offset_override(g0, geo.offsets[f:f + n])) if n else 0 for f, n in zip(first, sizes)], np.int32)
        if self.use_offset_override is not None:
            self.offcorr[:] = int(self.use_offset_override)
        self.first = first
        if is_dims is not None:
            self.set_domain_dimensions(is_dims)

    def set_domain_dimensions(self, dims):
        self.domain_dims = tuple(int(d) for d in dims)
        self._make_plan()

    def _make_plan(self):
        if self.plan is not None:
            self.plan.close()
        proj = self.acq.projections
        H, W = proj.shape[1], proj.shape[2]
        g = _cgeom(self.acq.geometry, W, H, self.domain_dims[:3], self.is_dims_in_mm, self.samples_per_pixel)
        self.plan = Plan(g, self.acq.geometry.angles, self.acq.geometry.offsets, self.subset_sizes, self.offcorr)
        if self.n_bins > 1:
            self.plan.set_bins(self.view_bin, self.n_bins)

    def set_use_offset_correction(self, use: bool):
        self.use_offset_override = bool(use)
        if hasattr(self, "offcorr"):
            self.offcorr[:] = int(use)
            if self.domain_dims is not None:
                self._make_plan()

    def get_number_of_subsets(self):
        return self.number_of_subsets

    def get_codomain_dimensions(self, subset: int):
        return (self.plan.g.width, self.plan.g.height, int(self.subset_sizes[subset]))

    def projection_subsets(self, projections):
        """Contiguous views of each subset's projections (subsetOperator::projection_subsets)."""
        return [projections[f:f + n] for f, n in zip(self.first, self.subset_sizes)]

    def mult_M(self, x, out, subset: int = -1, accumulate=False):
        if subset < 0:
            for s, o in enumerate(self.projection_subsets(out)):
                self.plan.forward(x, o, s, accumulate)
            return out
        return self.plan.forward(x, out, subset, accumulate)

    def mult_MH(self, proj, out, subset: int = -1, accumulate=False):
        if subset < 0:
            if not accumulate:
                out.zero_()
            for s, p in enumerate(self.projection_subsets(proj)):
                self.plan.backproject(p, out, s, 0, True, True)
            return out
        return self.plan.backproject(proj, out, subset, 0, True, accumulate)

    def mult_MH_M(self, x, out, subset: int, accumulate=False):
        T = torch()
        tmp = T.empty(self.plan.proj_shape(subset), dtype=T.float32, device=x.device)
        self.mult_M(x, tmp, subset, False)
        return self.mult_MH(tmp, out, subset, accumulate)

    def calculate_mask(self, projections, limit: float):
        """CBSubsetOperator::calculate_mask (.cpp:179-190): the AND of every
        subset's space-carved mask."""
        T = torch()
        mask = T.ones(self.plan.vol_shape, dtype=T.uint8, device=projections.device)
        for s, p in enumerate(self.projection_subsets(projections)):
            self.plan.spacecarver(p, limit, mask, s, combine=True)
        return mask

    def set_mask(self, mask):
        """CBSubsetOperator::set_mask: every subset's mult_MH applies the mask."""
        self.plan.set_mask(mask)

    def offset_correct(self, projections):
        """CBSubsetOperator::offset_correct (.cpp:44-50): sqrt weight on subsets with correction."""
        for s, p in enumerate(self.projection_subsets(projections)):
            if self.offcorr[s]:
                self.plan.offset_correct(p, s, 1)
        return projections


class CBSubsetWeightOperator(CBSubsetOperator):
    """CBSubsetOperator with per-pixel projection weights
    (xray/CBSubsetWeightOperator.h:11-63): setup multiplies the acquisition's
    projections by the weights, mult_M returns w * (A x) and mult_MH
    back-projects w * input."""

    def setup(self, acq: CBCT_acquisition, binning: Optional[CBCT_binning] = None, is_dims_in_mm=None,
              projection_weights=None, is_dims=None):
        w = np.ascontiguousarray(projection_weights, np.float32)
        if acq.projections is not None:
            acq.set_projections(np.ascontiguousarray(acq.projections * w))
        self._host_weights = w
        super().setup(acq, binning, is_dims_in_mm, is_dims=None)
        self.weights = torch().from_numpy(np.ascontiguousarray(w[self.permutation])).cuda()
        if is_dims is not None:
            self.set_domain_dimensions(is_dims)

    def _make_plan(self):
        super()._make_plan()
        self.plan.set_projection_weights(self.weights)


def _host_f32(a, what):
    """Pointer of a C-contiguous float32 host array (numpy or CPU torch tensor)."""
    T = torch()
    if isinstance(a, np.ndarray):
        if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
            raise TypeError(f"{what} must be a C-contiguous float32 array")
        return a.ctypes.data
    if isinstance(a, T.Tensor) and not a.is_cuda:
        if a.dtype != T.float32 or not a.is_contiguous():
            raise TypeError(f"{what} must be a contiguous float32 tensor")
        return a.data_ptr()
    raise TypeError(f"{what} must be a host array")


class hoCuConebeamProjectionOperator:
    """Host-array operator with optional FDK (hoCuConebeamProjectionOperator.h:17-156).

    Host arrays are float32 numpy arrays (or CPU torch tensors, page-locked for
    overlapped copies) of shape (P, H, W) for projections and (nz, ny, nx) or
    (bins, nz, ny, nx) for images.  Each bin's volume stays on the device while
    its projections stream through two device buffers of
    `projections_per_batch` views (default 20, .h:23), as the reference's
    host-array projectors do (conebeam_projection.cu:640-819, :1300-1649);
    cbct_host_forward / cbct_host_backproject do the streaming."""

    def __init__(self):
        self.samples_per_pixel = 1.5
        self.projections_per_batch = 20
        self.use_fbp = False
        self.short_scan = False
        self.preprocessed = False
        self.use_offset_correction = False
        self.allow_offset_correction_override = True
        self.frequency_filter = None
        self.domain_dims = None
        self._cache = None

    def setup(self, acquisition: CBCT_acquisition, binning: Optional[CBCT_binning] = None, is_dims_in_mm=None,
              transform_angles=True, is_dims=None):
        geo = acquisition.geometry
        if transform_angles:
            geo.set_angles(geo.angles - geo.angles.min())
        g0 = _cgeom(geo, 1, 1, (1, 1, 1), (1, 1, 1), self.samples_per_pixel)
        self.short_scan = is_short_scan(g0, geo.angles)
        if self.allow_offset_correction_override and offset_override(g0, geo.offsets):
            self.use_offset_correction = True
        self.acquisition = acquisition
        self.binning = binning if binning is not None else CBCT_binning([list(range(geo.angles.size))])
        self.is_dims_in_mm = tuple(float(v) for v in is_dims_in_mm)
        self.preprocessed = True
        self._cache = None
        if is_dims is not None:
            self.domain_dims = tuple(int(d) for d in is_dims)

    def set_domain_dimensions(self, dims):
        self.domain_dims = tuple(int(d) for d in dims)
        self._cache = None

    def set_use_filtered_backprojection(self, use: bool):
        self.use_fbp = bool(use)

    def set_use_offset_correction(self, use: bool):
        self.use_offset_correction = bool(use)
        self.allow_offset_correction_override = False

    def get_use_offset_correction(self):
        return self.use_offset_correction

    def set_num_projections_per_batch(self, n: int):
        if int(n) < 1:
            raise ValueError("projections_per_batch must be >= 1")
        self.projections_per_batch = int(n)
        self._cache = None

    def set_num_samples_per_pixel(self, spp: float):
        self.samples_per_pixel = float(spp)
        self._cache = None

    def set_frequency_filter(self, filt):
        self.frequency_filter = np.ascontiguousarray(filt, np.float32)

    def _stream_plan(self, W, H):
        """Plan whose views are the bins' views in bin order, cut into batches
        of projections_per_batch views (the plan's subsets)."""
        key = (W, H, self.domain_dims[:3], self.projections_per_batch, self.samples_per_pixel)
        if self._cache is not None and self._cache[0] == key:
            return self._cache[1]
        if not self.preprocessed:
            raise RuntimeError("hoCuConebeamProjectionOperator: setup not performed")
        geo = self.acquisition.geometry
        g = _cgeom(geo, W, H, self.domain_dims[:3], self.is_dims_in_mm, self.samples_per_pixel)
        order, sizes, bins = [], [], []
        B = self.projections_per_batch
        for views in self.binning.bins:
            v = [int(i) for i in views]
            for i in v:
                if not 0 <= i < geo.angles.size:
                    raise ValueError("illegal index in bin")
            first = len(sizes)
            for k in range(0, len(v), B):
                sizes.append(len(v[k:k + B]))
            bins.append((first, len(sizes) - first, len(v)))
            order += v
        idx = np.asarray(order, np.int64)
        plan = Plan(g, geo.angles[idx], geo.offsets[idx], np.asarray(sizes if sizes else [0], np.int32))
        st = dict(plan=plan, view_index=np.ascontiguousarray(idx, np.int32), bins=bins)
        self._cache = (key, st)
        return st

    def _bin_image(self, image, b):
        if image.ndim == 4:
            return image[b]
        if len(self.binning.bins) != 1:
            raise ValueError("several bins need a 4-D image (bins, nz, ny, nx)")
        return image

    def mult_M(self, image, projections, accumulate=False):
        """hoCuConebeamProjectionOperator::mult_M (.cpp:104-176)."""
        P, H, W = projections.shape
        if P != self.acquisition.geometry.angles.size:
            raise ValueError("inconsistent sizes of input arrays/vectors")
        st = self._stream_plan(W, H)
        result = np.zeros(projections.shape, np.float32) if accumulate else projections
        offset = int(self.use_offset_correction and not self.use_fbp)
        for b, (first, nb, n) in enumerate(st["bins"]):
            if n == 0:
                continue
            vol = self._bin_image(image, b)
            L.call("cbct_host_forward", st["plan"].handle, first, nb, _host_f32(vol, "image"),
                   _host_f32(result, "projections"), st["view_index"].ctypes.data, offset, None)
        if accumulate:
            projections += result
        return projections

    def mult_MH(self, projections, image, accumulate=False):
        """hoCuConebeamProjectionOperator::mult_MH (.cpp:178-265), FDK when FBP is on."""
        P, H, W = projections.shape
        if P != self.acquisition.geometry.angles.size:
            raise ValueError("inconsistent sizes of input arrays/vectors")
        st = self._stream_plan(W, H)
        filt = None if self.frequency_filter is None else self.frequency_filter
        if filt is not None and filt.size != W + 1:
            raise ValueError("frequency filter must have W+1 entries")
        for b, (first, nb, n) in enumerate(st["bins"]):
            tgt = self._bin_image(image, b)
            if self.use_fbp:
                flags = (L.CBCT_FDK_PARKER if self.short_scan else 0) | \
                        (L.CBCT_FDK_OFFSET if self.use_offset_correction else 0)
                scale = 2.0 / float(n) if n else 1.0
                L.call("cbct_host_backproject", st["plan"].handle, first, nb, _host_f32(projections, "projections"),
                       _host_f32(tgt, "image"), st["view_index"].ctypes.data, 1,
                       None if filt is None else filt.ctypes.data, flags, 0, scale, int(accumulate), None)
            else:
                L.call("cbct_host_backproject", st["plan"].handle, first, nb, _host_f32(projections, "projections"),
                       _host_f32(tgt, "image"), st["view_index"].ctypes.data, 0, None, 0,
                       int(self.use_offset_correction), 1.0, int(accumulate), None)
        return image


# ----------------------------------------------------------------- solvers
class cuTVPrimalDualOperator:
    """Total-variation regulariser of osMOMSolverD
    (operators/cuTVPrimalDualOperator.{h,cu}): periodic forward differences
    projected onto the unit ball; alpha as the reference's constructor
    argument, the weight via set_weight.  Evaluated on the device inside
    cbct_osmom_solve."""

    def __init__(self, alpha: float = 0.0):
        self.alpha = float(alpha)
        self.weight = 1.0

    def set_weight(self, w: float):
        self.weight = float(w)

    def get_weight(self) -> float:
        return self.weight


class osMOMSolverD:
    """osMOMSolverD<cuNDArray<float>> (solvers/osMOMSolverD.h:19-329), unregularised
    or with one cuTVPrimalDualOperator.

    solve() runs the whole loop on the device (cbct_osmom_solve).  The
    per-iteration dump files of the reference (:184-189) are not written;
    set_dump is accepted for interface compatibility."""

    def __init__(self):
        self._iterations = 10
        self._beta = 1.0
        self._gamma = 0.0
        self.non_negativity = False
        self.x0 = None
        self.E: Optional[CBSubsetOperator] = None
        self.use_graph = False
        self.storage = L.CBCT_F32
        self.refine_every = 0
        self.residual_norms = None
        self.regularizers = []
        self.tau = 1e-3          # osMOMSolverD.h:33
        self.reg_steps = 1       # :29
        self.huber = 0.0

    def set_tau(self, tau):
        self.tau = float(tau)

    def set_reg_steps(self, n):
        self.reg_steps = int(n)

    def set_huber(self, h):
        """denoise_alpha of the solver's linear-operator regularisers; the TV
        operator takes its own alpha."""
        self.huber = float(h)

    def set_max_iterations(self, i):
        self._iterations = int(i)

    def get_max_iterations(self):
        return self._iterations

    def set_non_negativity_constraint(self, v=True):
        self.non_negativity = bool(v)

    def set_beta(self, b):
        self._beta = float(b)

    def set_gamma(self, g):
        self._gamma = float(g)

    def set_dump(self, d):
        pass

    def set_x0(self, x0):
        self.x0 = x0

    def set_encoding_operator(self, E):
        self.E = E

    def add_regularization_operator(self, op):
        """osMOMSolverD::add_regularization_operator (.h:48-54); this build
        takes one cuTVPrimalDualOperator."""
        if not isinstance(op, cuTVPrimalDualOperator):
            raise NotImplementedError("only cuTVPrimalDualOperator regularisation is built")
        if self.regularizers:
            raise NotImplementedError("one regulariser per solver in this build")
        self.regularizers.append(op)

    def solve(self, projections):
        T = torch()
        E = self.E
        if E is None:
            raise RuntimeError("osMOMSolverD: no encoding operator is set")
        if E.domain_dims is None:
            raise RuntimeError("osMOMSolverD: encoding operator has not set domain dimension")
        z = T.empty(E.plan.vol_shape, dtype=T.float32, device=projections.device)
        S = E.get_number_of_subsets()
        self.residual_norms = T.zeros(self._iterations * S, dtype=T.float64, device=projections.device)
        tv = self.regularizers[0] if self.regularizers else None
        if tv is not None:
            self.residual_norms = None   # the regularised solve keeps no residual trace
        E.plan.osmom(projections, z, self.x0, self._iterations, self._beta, self._gamma, self.non_negativity,
                     self.use_graph, self.storage, self.refine_every, self.residual_norms,
                     tv_weight=0.0 if tv is None else tv.weight, tv_alpha=0.0 if tv is None else tv.alpha,
                     tau=self.tau, reg_steps=self.reg_steps)
        return z


class osSARTSolver:
    """osSARTSolver<cuNDArray<float>> (solvers/osSARTSolver.h:11-137); the per-iteration
    .real files of the reference (:117-121) are not written."""

    def __init__(self):
        self._iterations = 10
        self._beta = 1.0
        self._gamma = 0.0
        self.non_negativity = False
        self.x0 = None
        self.E = None
        self.use_graph = False
        self.costs = None

    def set_max_iterations(self, i):
        self._iterations = int(i)

    def set_non_negativity_constraint(self, v=True):
        self.non_negativity = bool(v)

    def set_beta(self, b):
        self._beta = float(b)

    def set_gamma(self, g):
        self._gamma = float(g)

    def set_x0(self, x0):
        self.x0 = x0

    def set_encoding_operator(self, E):
        self.E = E

    def solve(self, projections):
        T = torch()
        E = self.E
        x = T.empty(E.plan.vol_shape, dtype=T.float32, device=projections.device)
        self.costs = T.zeros(self._iterations, dtype=T.float64, device=projections.device)
        E.plan.ossart(projections, x, self.x0, self._iterations, self._beta, self._gamma, self.non_negativity,
                      self.use_graph, self.costs)
        return x


def fdk_reconstruct_3d(acquisition: CBCT_acquisition, is_dims, is_dims_in_mm, filt=None, binning=None,
                       projections_per_batch=20):
    """The FDK recipe of FDK_reconstruct_3d.cpp:135-161 over the host-array
    operator: FDK (mult_MH with filtered back-projection, streamed in batches of
    views), the forward projection of the result (mult_M), then the
    least-squares rescale s = <A x, p> / <A x, A x> (dot products in FP64).
    Returns the host volume (nz, ny, nx)."""
    T = torch()
    E = hoCuConebeamProjectionOperator()
    E.set_num_projections_per_batch(projections_per_batch)
    if binning is not None and binning.get_number_of_bins() > 1:
        binning = binning.get_3d_binning()
    E.setup(acquisition, binning, is_dims_in_mm, is_dims=is_dims)
    E.set_use_filtered_backprojection(True)
    if filt is not None:
        E.set_frequency_filter(filt)
    p = T.from_numpy(np.ascontiguousarray(acquisition.projections, np.float32)).pin_memory()
    nx, ny, nz = (int(v) for v in is_dims)
    x = T.zeros((nz, ny, nx), dtype=T.float32).pin_memory()
    E.mult_MH(p, x)
    tmp = T.zeros_like(p).pin_memory()
    E.mult_M(x, tmp)
    a = tmp.numpy().astype(np.float64).ravel()
    s = float(np.dot(a, p.numpy().astype(np.float64).ravel()) / np.dot(a, a))
    return (x.numpy() * np.float32(s)).astype(np.float32)

"""FDK filter and full FDK on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.mark.parametrize("W", [40, 48, 100, 129, 256, 300, 512, 513])
def test_ramp_filter_rows(gtb, O, cuda, W):
    """The FFT convolution equals pad(2W)/FFT/filter/IFFT/crop: the radix-2
    shared-memory kernel (W <= 128, W > 512) and the register four-step FFT
    (512-point transforms for W = 129..256, 1024-point for W = 257..512)."""
    import torch
    case = make("cube")
    case.W = W
    case.fov_u = 1.5 * W
    rng = np.random.default_rng(W)
    p = rng.normal(0, 1, (case.angles.size, case.H, W))
    filt = O.default_filter(W)
    ref = O.fdk_filter_rows(p, filt)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.empty_like(pt)
    plan.fdk_filter(pt, out, -1, None, gtb._lib.CBCT_FDK_RAMP)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("W,H", [(300, 41), (200, 7)])
def test_register_fft_odd_rows_in_place(gtb, O, cuda, W, H):
    """Odd row counts (the last pair has no second row), in place, custom filter."""
    import torch
    case = make("cube")
    case.W, case.H, case.fov_u, case.fov_v = W, H, 1.5 * W, 1.5 * H
    rng = np.random.default_rng(W + H)
    p = rng.normal(0, 1, (3, H, W))
    case.angles = case.angles[:3].copy()
    case.offsets = case.offsets[:3].copy()
    filt = gtb.hann_ramp_filter(W).astype(np.float64)
    ref = O.fdk_filter_rows(p, filt)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    plan.fdk_filter(pt, pt, -1, filt.astype(np.float32), gtb._lib.CBCT_FDK_RAMP)
    assert O.rel_l2(pt.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("dtype", ["float16", "bfloat16"])
def test_register_fft_16bit_input(gtb, O, cuda, dtype):
    import torch
    td = getattr(torch, dtype)
    case = make("cube")
    W = 300
    case.W, case.fov_u = W, 1.5 * W
    p = np.random.default_rng(8).uniform(0, 1, (case.angles.size, case.H, W))
    stored = torch.from_numpy(p.astype(np.float32)).to(td)
    ref = O.fdk_filter_rows(stored.double().numpy(), O.default_filter(W))
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    out = torch.empty((case.angles.size, case.H, W), dtype=torch.float32, device=cuda)
    L = gtb._lib
    sd = stored.to(cuda)
    code = L.CBCT_F16 if dtype == "float16" else L.CBCT_BF16
    L.call("cbct_fdk_filter_ex", plan._h, -1, code, sd.data_ptr(), out.data_ptr(), None, L.CBCT_FDK_RAMP, None)
    torch.cuda.synchronize()
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


def test_filter_in_place_and_custom(gtb, O, cuda):
    import torch
    case = make("cube")
    rng = np.random.default_rng(4)
    p = rng.normal(0, 1, (case.angles.size, case.H, case.W))
    filt = gtb.hann_ramp_filter(case.W).astype(np.float64)
    ref = O.fdk_filter_rows(p, filt)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    plan.fdk_filter(pt, pt, -1, filt.astype(np.float32), gtb._lib.CBCT_FDK_RAMP)
    assert O.rel_l2(pt.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("flags", ["cos", "cos+offset", "cos+parker", "cos+offset+parker"])
@pytest.mark.parametrize("W", [None, 300])
def test_fdk_weights(gtb, O, cuda, flags, W):
    import torch
    case = make("offset")
    if W is not None:   # the register FFT path (1024-point transforms)
        case.fov_u *= W / case.W
        case.offsets = case.offsets * np.float32(W / case.W)
        case.W = W
    if "parker" in flags:
        case.angles = (np.arange(case.angles.size) * (220.0 / case.angles.size)).astype(np.float32)
    g = case.oracle_geom(O)
    rng = np.random.default_rng(5)
    p = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    q = p * O.cosine_weights(g)[None]
    F = gtb._lib
    fl = F.CBCT_FDK_RAMP | F.CBCT_FDK_COSINE
    if "parker" in flags:
        q = O.parker_weight(g, q, case.angles)
        fl |= F.CBCT_FDK_PARKER
    filt = O.default_filter(case.W)
    q = O.fdk_filter_rows(q, filt)
    if "offset" in flags:
        q = O.offset_weight(g, q, case.offsets, 0)
        fl |= F.CBCT_FDK_OFFSET
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.empty_like(pt)
    plan.fdk_filter(pt, out, -1, None, fl)
    assert O.rel_l2(out.cpu().numpy(), q) < TOL


@pytest.mark.parametrize("name", ["cube", "offset"])
def test_fdk_full(gtb, O, cuda, name):
    import torch
    case = make(name)
    g = case.oracle_geom(O)
    rng = np.random.default_rng(6)
    p = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    off = name == "offset"
    ref = O.fdk(g, p, case.angles, case.offsets, short_scan=False, offset_corr=off)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(pt, out, None, gtb._lib.CBCT_FDK_OFFSET if off else 0)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


def test_fdk_recipe_reconstructs_phantom(gtb, O, cuda):
    """FDK_reconstruct_3d recipe (FDK + least-squares rescale) of exact line
    integrals reproduces the phantom (known answer, loose bound)."""
    case = make("c1small")
    from gt_tomography_b200 import phantom
    ell = phantom.ellipsoids(21, (case.lx, case.ly, case.lz), n=5)
    g = case.oracle_geom(O)
    proj = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets).astype(np.float32)
    truth = O.phantom_voxelize(g, ell.astype(np.float64), ss=2)
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, proj.copy())
    x = gtb.fdk_reconstruct_3d(acq, (case.nx, case.ny, case.nz), (case.lx, case.ly, case.lz),
                               filt=gtb.hann_ramp_filter(case.W))
    c = np.corrcoef(x.ravel(), truth.ravel())[0, 1]
    assert c > 0.9, c

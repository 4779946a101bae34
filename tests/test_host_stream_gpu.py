"""Host-array operators streamed in batches of views (cbct_host_forward,
cbct_host_backproject; hoCuConebeamProjectionOperator over
conebeam_projection.cu:640-819 and :1300-1649).

The forward result of a ray does not depend on how views are batched, so the
streamed mult_M equals the device operator bitwise; the streamed mult_MH and
FDK add the batches one after another and agree with the single-launch device
operators to rounding and with the FP64 oracle within 1e-4."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _operator(gtb, case, batch, fbp=False, bins=None, offset=None):
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, None)
    op = gtb.hoCuConebeamProjectionOperator()
    op.set_num_projections_per_batch(batch)
    if offset is not None:
        op.set_use_offset_correction(offset)
    op.setup(acq, None if bins is None else gtb.CBCT_binning(bins), (case.lx, case.ly, case.lz),
             transform_angles=False, is_dims=(case.nx, case.ny, case.nz))
    op.set_use_filtered_backprojection(fbp)
    return op


def _vol(gtb, case, O, seed=3):
    ell = gtb.phantom.ellipsoids(seed, (case.lx, case.ly, case.lz), n=6).astype(np.float64)
    return O.phantom_voxelize(case.oracle_geom(O), ell, ss=2).astype(np.float32)


@pytest.mark.parametrize("name,batch,offset", [("cube", 5, False), ("offset", 7, True), ("short", 4, False)])
def test_streamed_forward_equals_device(gtb, O, cuda, name, batch, offset):
    import torch
    case = make(name)
    vol = _vol(gtb, case, O)
    op = _operator(gtb, case, batch, offset=offset)
    proj = np.full((case.angles.size, case.H, case.W), -1.0, np.float32)
    op.mult_M(vol, proj)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    ref = torch.empty(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(torch.from_numpy(vol).to(cuda), ref)
    if offset:
        plan.offset_correct(ref, -1, 1)
    assert np.array_equal(proj, ref.cpu().numpy())
    oracle = O.forward(case.oracle_geom(O), vol.astype(np.float64), case.angles, case.offsets)
    if offset:
        oracle = O.offset_weight(case.oracle_geom(O), oracle, case.offsets, 1)
    assert O.rel_l2(proj, oracle) < TOL


@pytest.mark.parametrize("name,batch", [("cube", 5), ("aniso", 3)])
def test_streamed_backproject(gtb, O, cuda, name, batch):
    import torch
    case = make(name)
    p = np.random.default_rng(2).uniform(0, 1, (case.angles.size, case.H, case.W)).astype(np.float32)
    op = _operator(gtb, case, batch)
    vol = np.zeros((case.nz, case.ny, case.nx), np.float32)
    op.mult_MH(p, vol)
    ref = O.backproject(case.oracle_geom(O), p.astype(np.float64), case.angles, case.offsets)
    assert O.rel_l2(vol, ref) < TOL
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    dev = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(torch.from_numpy(p).to(cuda), dev, -1, 0, False)
    assert O.rel_l2(vol, dev.cpu().numpy()) < 1e-6
    # accumulate: vol + A^T p
    acc = vol.copy()
    op.mult_MH(p, acc, accumulate=True)
    assert O.rel_l2(acc, 2 * vol) < 1e-6


@pytest.mark.parametrize("name,batch", [("cube", 4), ("offset", 6)])
def test_streamed_fdk(gtb, O, cuda, name, batch):
    import torch
    case = make(name)
    p = np.random.default_rng(6).uniform(0, 1, (case.angles.size, case.H, case.W)).astype(np.float32)
    off = name == "offset"
    op = _operator(gtb, case, batch, fbp=True)
    assert op.get_use_offset_correction() == off   # the override rule of setup
    vol = np.zeros((case.nz, case.ny, case.nx), np.float32)
    op.mult_MH(p, vol)
    ref = O.fdk(case.oracle_geom(O), p.astype(np.float64), case.angles, case.offsets, offset_corr=off)
    assert O.rel_l2(vol, ref) < TOL
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    dev = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(torch.from_numpy(p).to(cuda), dev, None, gtb._lib.CBCT_FDK_OFFSET if off else 0)
    assert O.rel_l2(vol, dev.cpu().numpy()) < 1e-6
    # accumulate: the bin's 2/P scales the incoming image too (.cpp:253)
    acc = vol.copy()
    op.mult_MH(p, acc, accumulate=True)
    P = case.angles.size
    assert O.rel_l2(acc, vol * (2.0 / P) + vol) < 1e-6


def test_streamed_bins_and_pinned_arrays(gtb, O, cuda):
    """Two bins of interleaved views, a 4-D image, page-locked host tensors."""
    import torch
    case = make("cube")
    P = case.angles.size
    bins = [list(range(0, P, 2)), list(range(1, P, 2))]
    v0, v1 = _vol(gtb, case, O, 3), _vol(gtb, case, O, 5)
    img = torch.from_numpy(np.stack([v0, v1])).pin_memory()
    op = _operator(gtb, case, 4, bins=bins)
    proj = torch.zeros((P, case.H, case.W), dtype=torch.float32).pin_memory()
    op.mult_M(img, proj)
    g = case.oracle_geom(O)
    for b, vb in enumerate((v0, v1)):
        idx = np.asarray(bins[b])
        ref = O.forward(g, vb.astype(np.float64), case.angles[idx], case.offsets[idx])
        assert O.rel_l2(proj.numpy()[idx], ref) < TOL
    back = torch.zeros_like(img).pin_memory()
    op.mult_MH(proj, back)
    for b in range(2):
        idx = np.asarray(bins[b])
        ref = O.backproject(g, proj.numpy()[idx].astype(np.float64), case.angles[idx], case.offsets[idx])
        assert O.rel_l2(back.numpy()[b], ref) < TOL
    with pytest.raises(ValueError):
        op.mult_M(v0, proj)      # several bins need a 4-D image

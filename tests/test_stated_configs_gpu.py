"""Parity at the stated workload sizes against the FP64 oracle.

C1 at full size: a 128^3 phantom of 10 seeded ellipsoids at 1 mm, 180 views
over 360 degrees, a 256x192 detector at 1.5 mm, SAD 1000 mm, SDD 1500 mm, no
offset: the forward projection (mult_M), FDK with a Hann-windowed ramp
(hoCuConebeamProjectionOperator::mult_MH with filtered back-projection), the
FDK_reconstruct_3d recipe (FDK, mult_M of the result, least-squares rescale;
FDK_reconstruct_3d.cpp:152-161) and the OS-MOM preconditioner
(osMOMSolverD.h:115-120).

C2 at full size, one subset: a 256^3 volume, 360 views of 512x384 at 0.8 mm
with an 80 mm half-fan offset, 10 subsets; subset 0 (36 views) takes one
OS-MOM step (osMOMSolverD.h:142-175): the residual forward projection with
its offset weight and FP64 norm, then the back-projection with the update of
z and xold fused into its epilogue.

Inputs are made on the device (supersampled voxelisation, exact chord
integrals of the ellipsoids) and copied to the host, so the oracle and the
device path see the same float32 values.  Tolerance: 1e-4 relative L2, the
FP32 path's bound against FP64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _c1(gtb, O, cuda):
    import torch
    nx = 128
    P, W, H, pitch = 180, 256, 192, 1.5
    ang = gtb.phantom.circular_orbit(P)
    off = np.zeros((P, 2), np.float32)
    g = gtb._lib.CbctGeometry(1000.0, 1500.0, W * pitch, H * pitch, W, H, nx, nx, nx, 128.0, 128.0, 128.0, 1.5)
    og = O.Geometry(nx, nx, nx, 128.0, 128.0, 128.0, W, H, W * pitch, H * pitch, 1000.0, 1500.0)
    ell = torch.from_numpy(gtb.phantom.ellipsoids(1234, (128.0, 128.0, 128.0), n=10).reshape(-1)).to(cuda)
    plan = gtb.Plan(g, ang, off)
    vol = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    gtb.phantom_voxelize(g, ell, vol, 4)
    proj = torch.empty(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.phantom_project(ell, proj)
    torch.cuda.synchronize()
    return plan, g, og, ang, off, vol, proj


@pytest.fixture(scope="module")
def c1(gtb, O, cuda):
    return _c1(gtb, O, cuda)


def test_c1_forward_full_size(gtb, O, cuda, c1):
    import torch
    plan, g, og, ang, off, vol, proj = c1
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(vol, out)
    plan.check()
    ref = O.forward(og, vol.cpu().numpy().astype(np.float64), ang, off)
    e = O.rel_l2(out.cpu().numpy(), ref)
    print(f"C1 forward ({plan.forward_variant()}) vs FP64: {e:.2e}")
    assert e < TOL


def test_c1_fdk_full_size(gtb, O, cuda, c1):
    import torch
    plan, g, og, ang, off, vol, proj = c1
    filt = gtb.hann_ramp_filter(g.width)
    x = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(proj, x, filt, 0)
    ref = O.fdk(og, proj.cpu().numpy().astype(np.float64), ang, off, filt=filt)
    e = O.rel_l2(x.cpu().numpy(), ref)
    print(f"C1 FDK (Hann ramp) vs FP64: {e:.2e}")
    assert e < TOL


def test_c1_fdk_recipe_full_size(gtb, O, cuda, c1):
    """fdk_reconstruct_3d (host arrays, views streamed in batches of 20) against
    the oracle's recipe: FDK, A x, s = <A x, p> / <A x, A x>, x s."""
    plan, g, og, ang, off, vol, proj = c1
    filt = gtb.hann_ramp_filter(g.width)
    p = proj.cpu().numpy()
    geo = gtb.CBCT_geometry(1000.0, 1500.0, (g.fov_u, g.fov_v), ang.copy(), off.copy())
    acq = gtb.CBCT_acquisition(geo, p.copy())
    x = gtb.fdk_reconstruct_3d(acq, (g.nx, g.ny, g.nz), (g.lx, g.ly, g.lz), filt=filt)
    ref = O.fdk_recipe(og, p.astype(np.float64), ang, off, filt=filt)
    e = O.rel_l2(x, ref)
    print(f"C1 FDK_reconstruct_3d recipe vs FP64: {e:.2e}")
    assert e < TOL


def test_c1_osmom_preconditioner_full_size(gtb, O, cuda, c1):
    import torch
    plan, g, og, ang, off, vol, proj = c1
    D = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom_precon(D)
    plan.check()
    ones = np.ones((g.nz, g.ny, g.nx))
    ref = 1.0 / np.maximum(O.backproject(og, O.forward(og, ones, ang, off), ang, off), 1e-6)
    e = O.rel_l2(D.cpu().numpy(), ref)
    print(f"C1 OS-MOM preconditioner vs FP64: {e:.2e}")
    assert e < TOL


def test_c2_subset_step_full_size(gtb, O, cuda):
    """One full 36-view subset of C2: residual forward projection (Wang offset
    weight, FP64 norm) and the back-projection with the fused OS-MOM update."""
    import torch
    nx, P, W, H, pitch, S = 256, 360, 512, 384, 0.8, 10
    ang = gtb.phantom.circular_orbit(P)
    off = np.tile(np.array([[80.0, 0.0]], np.float32), (P, 1))
    order, sizes = gtb.subset_partition(P, S)
    a, o = ang[order] - ang.min(), off[order]
    g = gtb._lib.CbctGeometry(1000.0, 1500.0, W * pitch, H * pitch, W, H, nx, nx, nx, 256.0, 256.0, 256.0, 1.5)
    og = O.Geometry(nx, nx, nx, 256.0, 256.0, 256.0, W, H, W * pitch, H * pitch, 1000.0, 1500.0)
    oc = [1] * S          # |mean offset| 80 mm > 0.1 * 409.6 mm: offset correction on every subset
    plan = gtb.Plan(g, a, o, sizes, oc)
    n0 = int(sizes[0])
    ell = torch.from_numpy(gtb.phantom.ellipsoids(1234, (256.0, 256.0, 256.0), n=10).reshape(-1)).to(cuda)
    truth = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    gtb.phantom_voxelize(g, ell, truth, 2)
    b = torch.empty(plan.proj_shape(0), dtype=torch.float32, device=cuda)
    plan.phantom_project(ell, b, 0)
    gen = torch.Generator(device=cuda).manual_seed(5)
    z = (0.7 * truth + 0.002 * torch.rand(truth.shape, device=cuda, generator=gen)).contiguous()
    xold = (0.6 * truth).contiguous()
    D = (0.001 + 0.002 * torch.rand(truth.shape, device=cuda, generator=gen)).contiguous()
    zh, xh, Dh, bh = (t.cpu().numpy().astype(np.float64) for t in (z, xold, D, b))
    r = torch.empty(plan.proj_shape(0), dtype=torch.float32, device=cuda)
    n2 = torch.zeros(1, dtype=torch.float64, device=cuda)
    step, mom = 1.0 * S, 0.38
    plan.osmom_step(0, b, z, xold, D, r, step, mom, nonneg=True, norm2=n2)
    plan.check()
    a0, o0 = a[:n0], o[:n0]
    resid = O.forward(og, zh, a0, o0) - bh
    r_ref = O.offset_weight(og, resid, o0, 0)
    grad = O.backproject(og, r_ref, a0, o0)
    x_ref = np.maximum(zh - step * Dh * grad, 0.0)
    z_ref = x_ref * (1 + mom) - mom * xh
    e_r = O.rel_l2(r.cpu().numpy(), r_ref)
    e_z = O.rel_l2(z.cpu().numpy(), z_ref)
    e_x = O.rel_l2(xold.cpu().numpy(), x_ref)
    e_n = abs(float(n2.item()) - float(np.sum(resid * resid))) / float(np.sum(resid * resid))
    print(f"C2 subset step ({plan.forward_variant()}): residual {e_r:.2e}, z {e_z:.2e}, xold {e_x:.2e}, "
          f"norm {e_n:.2e} vs FP64")
    assert e_r < TOL and e_z < TOL and e_x < TOL and e_n < TOL

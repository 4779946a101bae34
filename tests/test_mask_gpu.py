"""Space carver, apply_mask and masked back-projection / OS-MOM on the GPU
against the FP64 oracle (conebeam_projection.cu:822-921, :1651-1657)."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu


def _proj(case, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, (case.angles.size, case.H, case.W))
    p[rng.uniform(size=p.shape) < 0.2] = 0.0          # zeros are ignored by the carver
    return p


@pytest.mark.parametrize("name", ["cube", "offset", "aniso"])
def test_spacecarver_matches_oracle(gtb, O, cuda, name):
    import torch
    case = make(name)
    p = _proj(case, 1)
    ref = O.spacecarver(case.oracle_geom(O), p, case.angles, case.offsets, 0.35)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    m = torch.zeros(plan.vol_shape, dtype=torch.uint8, device=cuda)
    plan.spacecarver(torch.from_numpy(p.astype(np.float32)).to(cuda), 0.35, m)
    got = m.cpu().numpy()
    # point sampling: a voxel may flip where u*W lands within float rounding of a texel edge
    assert np.mean(got != ref) < 2e-3, np.mean(got != ref)
    assert 0.0 < ref.mean() < 1.0


def test_subset_mask_is_and_of_subsets(gtb, O, cuda):
    import torch
    case = make("cube")
    p = _proj(case, 2)
    sizes = [4, 4, 4]
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, sizes)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    m = torch.ones(plan.vol_shape, dtype=torch.uint8, device=cuda)
    for s, f in enumerate((0, 4, 8)):
        plan.spacecarver(pt[f:f + 4], 0.35, m, s, combine=True)
    g = case.oracle_geom(O)
    ref = np.ones((case.nz, case.ny, case.nx), np.uint8)
    for f in (0, 4, 8):
        ref &= O.spacecarver(g, p[f:f + 4], case.angles[f:f + 4], case.offsets[f:f + 4], 0.35)
    assert np.mean(m.cpu().numpy() != ref) < 2e-3


def test_masked_backprojection_and_apply_mask(gtb, O, cuda):
    import torch
    case = make("offset")
    rng = np.random.default_rng(3)
    p = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    mask = (rng.uniform(size=(case.nz, case.ny, case.nx)) < 0.7).astype(np.uint8)
    g = case.oracle_geom(O)
    ref = O.backproject(g, p, case.angles, case.offsets) * mask
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    mt = torch.from_numpy(mask).to(cuda)
    plan.set_mask(mt)
    out = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(torch.from_numpy(p.astype(np.float32)).to(cuda), out)
    assert O.rel_l2(out.cpu().numpy(), ref) < 1e-4
    v = torch.ones(plan.vol_shape, dtype=torch.float32, device=cuda)
    gtb.operators.apply_mask(v, mt)
    assert torch.equal(v.cpu(), torch.from_numpy(mask.astype(np.float32)))


def test_masked_osmom_matches_oracle(gtb, O, cuda):
    import torch
    case = make("cube")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(9, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, bp = case.angles[order], case.offsets[order], b[order]
    mask = O.spacecarver(g, bp, a, o, 0.05)
    zr, _ = O.osmom(g, bp, a, o, sizes, np.zeros(S, np.int32), iters=2, nonneg=True, mask=mask)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes)
    plan.set_mask(torch.from_numpy(mask).to(cuda))
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(torch.from_numpy(bp.astype(np.float32)).to(cuda), z, None, 2, nonneg=True, use_graph=True)
    assert O.rel_l2(z.cpu().numpy(), zr) < 1e-4


def test_masked_accumulating_backprojection(gtb, O, cuda):
    """mult_MH with accumulate and a mask: the reference applies the mask to
    the whole output after accumulating (cuConebeamProjectionOperator.cpp:113-114,
    apply_mask on `output`), so voxels outside the mask lose the caller's
    earlier contents too: out = mask * (incoming + A^T p)."""
    import torch
    case = make("offset")
    rng = np.random.default_rng(4)
    p = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    mask = (rng.uniform(size=(case.nz, case.ny, case.nx)) < 0.6).astype(np.uint8)
    incoming = rng.uniform(0.5, 1.5, (case.nz, case.ny, case.nx))
    g = case.oracle_geom(O)
    ref = (incoming + O.backproject(g, p, case.angles, case.offsets)) * mask
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    plan.set_mask(torch.from_numpy(mask).to(cuda))
    out = torch.from_numpy(incoming.astype(np.float32)).to(cuda)
    plan.backproject(torch.from_numpy(p.astype(np.float32)).to(cuda), out, accumulate=True)
    got = out.cpu().numpy()
    assert O.rel_l2(got, ref) < 1e-4
    assert np.all(got[mask == 0] == 0.0)

"""Back-projector (mult_MH) on the GPU against the FP64 oracle (rel L2 <= 1e-4)."""
import numpy as np
import pytest

from cases import ALL, make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _proj(case, O, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, (case.angles.size, case.H, case.W))


@pytest.mark.parametrize("name", ALL)
@pytest.mark.parametrize("fdk", [False, True])
def test_backproject_matches_oracle(gtb, O, cuda, name, fdk):
    import torch
    case = make(name)
    p = _proj(case, O)
    ref = O.backproject(case.oracle_geom(O), p, case.angles, case.offsets, fbp=fdk)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(pt, out, -1, gtb._lib.CBCT_BP_FDK_WEIGHT if fdk else 0)
    err = O.rel_l2(out.cpu().numpy(), ref)
    assert err < TOL, (name, fdk, err)


def test_backproject_offset_weight_copy(gtb, O, cuda):
    """mult_MH with offset correction weights a copy (input unchanged)."""
    import torch
    case = make("offset")
    p = _proj(case, O, 2)
    g = case.oracle_geom(O)
    ref = O.backproject(g, O.offset_weight(g, p, case.offsets, 0), case.angles, case.offsets)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, None, [1])
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    keep = pt.clone()
    out = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(pt, out, -1, 0, True)
    assert torch.equal(pt, keep)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


def test_backproject_accumulate(gtb, O, cuda):
    import torch
    case = make("cube")
    p = _proj(case, O, 3)
    ref = O.backproject(case.oracle_geom(O), p, case.angles, case.offsets)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, [6, 6])
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.full(plan.vol_shape, 2.0, dtype=torch.float32, device=cuda)
    plan.backproject(pt[:6], out, 0, 0, False, True)
    plan.backproject(pt[6:], out, 1, 0, False, True)
    assert O.rel_l2(out.cpu().numpy() - 2.0, ref) < TOL


@pytest.mark.parametrize("variant", [0, 1])
def test_offset_correct_kernel(gtb, O, cuda, variant):
    import torch
    case = make("offset")
    p = _proj(case, O, 4)
    ref = O.offset_weight(case.oracle_geom(O), p, case.offsets, variant)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    plan.offset_correct(pt, -1, variant)
    assert O.rel_l2(pt.cpu().numpy(), ref) < 1e-6


def test_adjoint_mismatch_recorded(gtb, O, cuda):
    """The pair is unmatched (no ray-length weight in mult_MH): <Ax,y>/<x,A^T y>
    is reported, not asserted to be 1; GPU and oracle agree on it."""
    import torch
    case = make("cube")
    rng = np.random.default_rng(9)
    x = rng.uniform(0, 1, (case.nz, case.ny, case.nx))
    y = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    g = case.oracle_geom(O)
    r_or = float((O.forward(g, x, case.angles, case.offsets) * y).sum() /
                 (x * O.backproject(g, y, case.angles, case.offsets)).sum())
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    xt = torch.from_numpy(x.astype(np.float32)).to(cuda)
    yt = torch.from_numpy(y.astype(np.float32)).to(cuda)
    ax = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    aty = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.forward(xt, ax)
    plan.backproject(yt, aty)
    r_gpu = float((ax.double() * yt.double()).sum() / (xt.double() * aty.double()).sum())
    assert abs(r_gpu - r_or) / r_or < 1e-5

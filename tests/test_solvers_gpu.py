"""OS-MOM and OS-SART on the GPU against the FP64 oracle's restatement of
osMOMSolverD.h:82-196 and osSARTSolver.h:33-126 (rel L2 <= 1e-4)."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _setup(gtb, O, name, S, seed=13, noise=0.0):
    case = make(name)
    from gt_tomography_b200 import phantom
    ell = phantom.ellipsoids(seed, (case.lx, case.ly, case.lz), n=5)
    g = case.oracle_geom(O)
    b = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets)
    if noise:
        b = b + np.random.default_rng(seed).normal(0, noise, b.shape)
    order, sizes = O.subset_partition(case.angles.size, S)
    a = case.angles[order] - case.angles.min()
    o = case.offsets[order]
    bp = b[order]
    return case, g, a, o, sizes, bp


@pytest.mark.parametrize("name,S,nonneg,off", [("cube", 3, True, 0), ("offset", 4, True, 1),
                                               ("aniso", 2, False, 0)])
def test_osmom_matches_oracle(gtb, O, cuda, name, S, nonneg, off):
    import torch
    case, g, a, o, sizes, b = _setup(gtb, O, name, S)
    oc = np.full(S, off, np.int32)
    iters = 3
    zr, rr = O.osmom(g, b, a, o, sizes, oc, iters=iters, nonneg=nonneg)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes, oc)
    bt = torch.from_numpy(b.astype(np.float32)).to(cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    res = torch.zeros(iters * S, dtype=torch.float64, device=cuda)
    plan.osmom(bt, z, None, iters, nonneg=nonneg, resid=res)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL
    assert np.allclose(res.cpu().numpy(), rr, rtol=1e-4)


def test_osmom_graph_equals_eager_and_is_deterministic(gtb, O, cuda):
    import torch
    case, g, a, o, sizes, b = _setup(gtb, O, "cube", 4, noise=0.01)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes)
    bt = torch.from_numpy(b.astype(np.float32)).to(cuda)
    z1 = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    z2 = torch.empty_like(z1)
    z3 = torch.empty_like(z1)
    plan.osmom(bt, z1, None, 2, nonneg=True)
    plan.osmom(bt, z2, None, 2, nonneg=True, use_graph=True)
    plan.osmom(bt, z3, None, 2, nonneg=True, use_graph=True)  # replay
    assert torch.equal(z1, z2) and torch.equal(z2, z3)


def test_osmom_x0(gtb, O, cuda):
    import torch
    case, g, a, o, sizes, b = _setup(gtb, O, "cube", 2)
    rng = np.random.default_rng(2)
    x0 = rng.uniform(0, 0.01, (case.nz, case.ny, case.nx))
    zr, _ = O.osmom(g, b, a, o, sizes, np.zeros(2, np.int32), iters=2, x0=x0)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes)
    bt = torch.from_numpy(b.astype(np.float32)).to(cuda)
    x0t = torch.from_numpy(x0.astype(np.float32)).to(cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(bt, z, x0t, 2)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL


@pytest.mark.parametrize("name,S,off", [("cube", 3, 0), ("offset", 2, 1)])
def test_ossart_matches_oracle(gtb, O, cuda, name, S, off):
    import torch
    case, g, a, o, sizes, b = _setup(gtb, O, name, S)
    oc = np.full(S, off, np.int32)
    xr, cr = O.ossart(g, b, a, o, sizes, oc, iters=3, nonneg=True)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes, oc)
    bt = torch.from_numpy(b.astype(np.float32)).to(cuda)
    x = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    cost = torch.zeros(3, dtype=torch.float64, device=cuda)
    plan.ossart(bt, x, None, 3, nonneg=True, cost=cost)
    assert O.rel_l2(x.cpu().numpy(), xr) < TOL
    assert np.allclose(cost.cpu().numpy(), cr, rtol=1e-4)


def test_subset_operator_surface(gtb, O, cuda):
    """CBSubsetOperator + osMOMSolverD used the way cuCBOS_reconstruct.cpp does."""
    import torch
    case = make("offset")
    from gt_tomography_b200 import phantom
    ell = phantom.ellipsoids(17, (case.lx, case.ly, case.lz), n=4)
    g = case.oracle_geom(O)
    b = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets).astype(np.float32)
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, b.copy())
    E = gtb.CBSubsetOperator(4)
    E.setup(acq, None, (case.lx, case.ly, case.lz))
    E.set_domain_dimensions((case.nx, case.ny, case.nz))
    assert E.offcorr.tolist() == [1, 1, 1, 1]          # mean offset 14 > 0.1*64
    solver = gtb.osMOMSolverD()
    solver.set_max_iterations(2)
    solver.set_non_negativity_constraint(True)
    solver.set_encoding_operator(E)
    z = solver.solve(torch.from_numpy(acq.projections).to(cuda))
    order, sizes = O.subset_partition(case.angles.size, 4)
    zr, _ = O.osmom(g, b[order].astype(np.float64), geo.angles, geo.offsets, sizes,
                    np.ones(4, np.int32), iters=2, nonneg=True)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL
    # all-subset mult_M / mult_MH
    x = torch.rand(E.plan.vol_shape, device=cuda)
    p = torch.empty(E.plan.proj_shape(), device=cuda)
    E.mult_M(x, p)
    y = torch.empty_like(x)
    E.mult_MH(p, y)
    ax = O.forward(g, x.cpu().numpy().astype(np.float64), geo.angles, geo.offsets)
    assert O.rel_l2(p.cpu().numpy(), ax) < TOL

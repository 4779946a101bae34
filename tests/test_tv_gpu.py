"""TV-regularised OS-MOM (osMOMSolverD with a cuTVPrimalDualOperator) on the
GPU against the FP64 oracle (rel L2 <= 1e-4)."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.mark.parametrize("name,S,lam,alpha,steps", [("cube", 3, 0.05, 0.0, 2), ("offset", 4, 0.2, 0.5, 1)])
def test_tv_osmom_matches_oracle(gtb, O, cuda, name, S, lam, alpha, steps):
    import torch
    case = make(name)
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(17, (case.lx, case.ly, case.lz), n=5)
    b = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets)
    b = b + np.random.default_rng(3).normal(0, 0.01, b.shape)
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, b = case.angles[order] - case.angles.min(), case.offsets[order], b[order]
    oc = np.full(S, int(name == "offset"), np.int32)
    zr, _ = O.osmom(g, b, a, o, sizes, oc, iters=3, nonneg=True, tv_weight=lam, tv_alpha=alpha, tau=1e-3,
                    reg_steps=steps)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes, oc)
    bt = torch.from_numpy(b.astype(np.float32)).to(cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(bt, z, None, 3, nonneg=True, tv_weight=lam, tv_alpha=alpha, tau=1e-3, reg_steps=steps)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL
    # the prior smooths: lower total variation than the unregularised solve
    zu = torch.empty_like(z)
    plan.osmom(bt, zu, None, 3, nonneg=True)
    tv = lambda v: float(sum(np.abs(np.diff(v, axis=ax)).sum() for ax in range(3)))
    assert tv(z.cpu().numpy()) < tv(zu.cpu().numpy())


def test_tv_through_solver_class_and_bins(gtb, O, cuda):
    """The reference's solver API (add_regularization_operator, set_tau,
    set_reg_steps) with a binned subset operator: each bin regularised in 3-D."""
    import torch
    case = make("cube")
    P = case.angles.size
    bins = [list(range(0, P, 2)), list(range(1, P, 2))]
    g = case.oracle_geom(O)
    proj = np.zeros((P, case.H, case.W))
    for bi, vb in enumerate(bins):
        ell = gtb.phantom.ellipsoids(30 + bi, (case.lx, case.ly, case.lz), n=4).astype(np.float64)
        proj[vb] = O.phantom_project(g, ell, case.angles[vb], case.offsets[vb])
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, proj.astype(np.float32))
    E = gtb.CBSubsetOperator(3)
    E.setup(acq, gtb.CBCT_binning(bins), (case.lx, case.ly, case.lz), is_dims=(case.nx, case.ny, case.nz))
    solver = gtb.osMOMSolverD()
    solver.set_encoding_operator(E)
    solver.set_max_iterations(2)
    solver.set_non_negativity_constraint(True)
    tv = gtb.cuTVPrimalDualOperator(0.0)
    tv.set_weight(0.1)
    solver.add_regularization_operator(tv)
    solver.set_tau(1e-3)
    solver.set_reg_steps(2)
    z = solver.solve(torch.from_numpy(np.ascontiguousarray(acq.projections)).to(cuda))
    zr, _ = O.osmom(g, acq.projections.astype(np.float64), acq.geometry.angles, acq.geometry.offsets,
                    E.subset_sizes, E.offcorr, iters=2, nonneg=True, view_bin=E.view_bin, n_bins=2,
                    tv_weight=0.1, tau=1e-3, reg_steps=2)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL


def test_tv_step_matches_numpy(gtb, cuda):
    """cbct_tv_step against its restatement in numpy (np.roll for the periodic
    neighbours), FP64 reference, FP32 kernel."""
    import torch
    rng = np.random.default_rng(9)
    shp = (12, 10, 14)
    x = rng.uniform(0, 1, shp)
    s = rng.uniform(0, 1, shp)
    D = rng.uniform(0.01, 0.1, shp)
    scale, tau, tl = 3.0, 1e-3, 0.02
    d = np.stack([(np.roll(x, -1, axis=ax) - x) * scale for ax in (2, 1, 0)])
    P = d / np.maximum(1.0, np.sqrt((d * d).sum(axis=0)))
    gv = sum(np.roll(P[i], 1, axis=ax) - P[i] for i, ax in enumerate((2, 1, 0)))
    ref = ((x - tau * gv) + tl * (s / D)) / ((1.0 / D) * tl + 1.0)
    t = lambda a: torch.from_numpy(a.astype(np.float32)).to(cuda)
    xt, Pt = t(x), torch.empty((3,) + shp, dtype=torch.float32, device=cuda)
    gtb.operators.tv_step(xt, Pt, t(s), t(D), scale, tau, tl)
    assert np.max(np.abs(Pt.cpu().numpy() - P)) < 1e-5
    assert np.linalg.norm(xt.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-6

"""CBSubsetWeightOperator (projection weights) on the GPU against the FP64
oracle: weighted mult_M / mult_MH and the device-resident OS-MOM and OS-SART."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _weighted_problem(gtb, O, S=3):
    case = make("offset")
    g = case.oracle_geom(O)
    rng = np.random.default_rng(8)
    ell = gtb.phantom.ellipsoids(19, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets).astype(np.float32)
    w = rng.uniform(0.5, 1.5, b.shape).astype(np.float32)
    return case, g, b, w


def test_weighted_operator_matches_oracle(gtb, O, cuda):
    import torch
    case, g, b, w = _weighted_problem(gtb, O)
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, b.copy())
    E = gtb.CBSubsetWeightOperator(3)
    E.setup(acq, None, (case.lx, case.ly, case.lz), w, is_dims=(case.nx, case.ny, case.nz))
    order = E.permutation
    # the acquisition now holds w*b in subset order
    assert np.allclose(acq.projections, (b * w)[order])
    x = torch.rand(E.plan.vol_shape, device=cuda) * 0.02
    p = torch.empty(E.plan.proj_shape(), device=cuda)
    E.mult_M(x, p)
    wp = w[order].astype(np.float64)
    ax = O.forward(g, x.cpu().numpy().astype(np.float64), geo.angles, geo.offsets) * wp
    assert O.rel_l2(p.cpu().numpy(), ax) < TOL
    y = torch.empty_like(x)
    E.mult_MH(p, y)
    ref = O.backproject(g, O.offset_weight(g, ax * wp, geo.offsets, 0), geo.angles, geo.offsets)
    assert O.rel_l2(y.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("solver", ["osmom", "ossart"])
def test_weighted_solvers_match_oracle(gtb, O, cuda, solver):
    import torch
    case, g, b, w = _weighted_problem(gtb, O)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o = case.angles[order], case.offsets[order]
    bw = (b * w)[order].astype(np.float64)
    wp = w[order].astype(np.float64)
    oc = np.ones(S, np.int32)
    if solver == "osmom":
        zr, _ = O.osmom(g, bw, a, o, sizes, oc, iters=2, nonneg=True, weights=wp)
    else:
        zr, _ = O.ossart(g, bw, a, o, sizes, oc, iters=2, nonneg=True, weights=wp)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes, oc)
    wt = torch.from_numpy(w[order]).to(cuda)
    plan.set_projection_weights(wt)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    bt = torch.from_numpy(bw.astype(np.float32)).to(cuda)
    if solver == "osmom":
        plan.osmom(bt, z, None, 2, nonneg=True, use_graph=True)
    else:
        plan.ossart(bt, z, None, 2, nonneg=True)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL

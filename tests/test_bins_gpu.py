"""4-D bins (CBCT_binning) in the subset operator and the OS-MOM solver, against
the FP64 oracle's binned restatement (each bin's views project and
back-project that bin's volume; bins without views in a subset step take the
momentum update with a zero gradient)."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _binned(gtb, O, name, S, nbins=2, seed=21):
    case = make(name)
    P = case.angles.size
    # respiratory-like bins: consecutive runs of views cycle through the bins
    bins = [[v for v in range(P) if (v // 3) % nbins == b] for b in range(nbins)]
    g = case.oracle_geom(O)
    vols = [O.phantom_voxelize(g, gtb.phantom.ellipsoids(seed + b, (case.lx, case.ly, case.lz), n=5)
                               .astype(np.float64), ss=2) for b in range(nbins)]
    proj = np.zeros((P, case.H, case.W))
    for b, vb in enumerate(bins):
        idx = np.asarray(vb)
        proj[idx] = O.forward(g, vols[b], case.angles[idx], case.offsets[idx])
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, proj.astype(np.float32))
    op = gtb.CBSubsetOperator(S)
    op.setup(acq, gtb.CBCT_binning(bins), (case.lx, case.ly, case.lz), is_dims=(case.nx, case.ny, case.nz))
    return case, g, op, acq, np.stack(vols)


def test_binned_subset_operator(gtb, O, cuda):
    import torch
    case, g, op, acq, vols = _binned(gtb, O, "cube", 3)
    assert op.plan.vol_shape == (2, case.nz, case.ny, case.nx)
    a, o, vb = acq.geometry.angles, acq.geometry.offsets, op.view_bin
    x = torch.from_numpy(vols.astype(np.float32)).to(cuda)
    for s in range(3):
        f, n = int(op.first[s]), int(op.subset_sizes[s])
        out = torch.empty(op.plan.proj_shape(s), dtype=torch.float32, device=cuda)
        op.mult_M(x, out, s)
        ref = np.zeros((n, case.H, case.W))
        for b in range(2):
            m = vb[f:f + n] == b
            if m.any():
                ref[m] = O.forward(g, vols[b], a[f:f + n][m], o[f:f + n][m])
        assert O.rel_l2(out.cpu().numpy(), ref) < TOL
        back = torch.full(op.plan.vol_shape, 7.0, dtype=torch.float32, device=cuda)
        op.mult_MH(out, back, s)
        for b in range(2):
            m = vb[f:f + n] == b
            refb = (O.backproject(g, out.cpu().numpy()[m].astype(np.float64), a[f:f + n][m], o[f:f + n][m])
                    if m.any() else np.zeros((case.nz, case.ny, case.nx)))
            got = back[b].cpu().numpy()
            assert (O.rel_l2(got, refb) < TOL) if m.any() else not got.any()


@pytest.mark.parametrize("graph", [False, True])
def test_binned_osmom_matches_oracle(gtb, O, cuda, graph):
    import torch
    case, g, op, acq, vols = _binned(gtb, O, "offset", 4)
    b = torch.from_numpy(np.ascontiguousarray(acq.projections)).to(cuda)
    z = torch.empty(op.plan.vol_shape, dtype=torch.float32, device=cuda)
    op.plan.osmom(b, z, None, 3, nonneg=True, use_graph=graph)
    zr, _ = O.osmom(g, acq.projections.astype(np.float64), acq.geometry.angles, acq.geometry.offsets,
                    op.subset_sizes, op.offcorr, iters=3, nonneg=True, view_bin=op.view_bin, n_bins=2)
    assert zr.shape == (2, case.nz, case.ny, case.nx)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL


def test_bins_must_be_contiguous_in_subsets(gtb, cuda):
    case = make("cube")
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, [6, 6])
    with pytest.raises(gtb.CbctError, match="contiguous"):
        plan.set_bins(np.array([0, 1, 0, 1, 0, 1] * 2, np.int32), 2)
    plan.set_bins(np.array([0, 0, 0, 1, 1, 1, 1, 1, 0, 0, 0, 0], np.int32), 2)
    assert plan.vol_shape[0] == 2
    plan.set_bins(None, 1)
    assert plan.vol_shape == (case.nz, case.ny, case.nx)

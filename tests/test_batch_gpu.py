"""Batched reconstruction of uneven scans (cbct_batch_osmom): each result is
bitwise identical to the scan solved alone, and matches the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_equals_alone(gtb, O, cuda):
    import torch
    specs = gtb.phantom.uneven_scans(5, seed0=77, vol_range=(32, 64), z_range=(24, 48), view_range=(20, 60),
                                     width_range=(40, 80))
    for sp in specs:          # a detector that covers the whole volume in every view
        sp["pitch"] *= 1.6
    scans = [gtb.phantom.make_osmom_scan(sp, 3, 1e5, cuda) for sp in specs]
    alone, jobs = [], []
    for plan, b, _ in scans:
        z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
        plan.osmom(b, z, None, 3, nonneg=True, use_graph=True)
        alone.append(z)
    torch.cuda.synchronize()
    outs = []
    for plan, b, _ in scans:
        z = torch.full(plan.vol_shape, -1.0, dtype=torch.float32, device=cuda)
        outs.append(z)
        jobs.append(dict(plan=plan, b=b, z=z, iterations=3, nonneg=True))
    gtb.batch_osmom(jobs, n_streams=3)
    for a, z in zip(alone, outs):
        assert torch.equal(a, z)
    # one of them against the FP64 oracle
    (plan, b, (ang, off, sizes, oc)), sp = scans[1], specs[1]
    nx, ny, nz = sp["n"]
    g = O.Geometry(nx, ny, nz, float(nx), float(ny), float(nz), sp["W"], sp["H"], sp["W"] * sp["pitch"],
                   sp["H"] * sp["pitch"], 1000.0, 1500.0)
    zr, _ = O.osmom(g, b.double().cpu().numpy(), ang, off, sizes, np.asarray(oc, np.int32), iters=3, nonneg=True)
    # Voxels that only grazing rays reach have A^T A 1 near 0, where the solver's
    # preconditioner 1/max(A^T A 1, 1e-6) magnifies any rounding difference; the
    # comparison covers the voxels the scan actually measures.
    pre = O.backproject(g, O.forward(g, np.ones((nz, ny, nx)), ang, off), ang, off)
    seen = pre > 1e-2 * pre.max()
    assert seen.mean() > 0.5
    assert O.rel_l2(outs[1].cpu().numpy()[seen], zr[seen]) < 1e-4


def test_batch_rejects_shared_plans(gtb, cuda):
    import torch
    sp = gtb.phantom.uneven_scans(1, seed0=5, vol_range=(32, 32), z_range=(24, 24), view_range=(20, 20),
                                  width_range=(40, 40))[0]
    plan, b, _ = gtb.phantom.make_osmom_scan(sp, 2, 0, cuda)
    z1 = torch.empty(plan.vol_shape, device=cuda)
    z2 = torch.empty(plan.vol_shape, device=cuda)
    with pytest.raises(gtb.CbctError):
        gtb.batch_osmom([dict(plan=plan, b=b, z=z1), dict(plan=plan, b=b, z=z2)])

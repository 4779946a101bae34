"""Fused batch OS-MOM (cbct_batch_osmom_fused): scans of uneven volume,
detector, view count, subset count and iteration count advanced in lockstep
through persistent work-list launches captured in one graph.  Every result
(and residual trace) is bitwise the scan solved alone through its plan."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-4

# CBCT_OPT_FORWARD_KERNEL per scan: automatic, slab, row pairs, row quads,
# column fan and gather (the last two run as one-scan launches in the graph).
KERNELS = [0, 1, 4, 5, 3, 2]


def _scans(gtb, cuda, n, seed0):
    specs = gtb.phantom.uneven_scans(n, seed0=seed0, vol_range=(32, 64), z_range=(24, 48), view_range=(20, 60),
                                     width_range=(40, 80))
    out = []
    for i, sp in enumerate(specs):
        sp["pitch"] *= 1.6        # a detector that covers the whole volume in every view
        S = 2 + i % 3
        off = 0.25 * sp["W"] * sp["pitch"] if i % 4 == 2 else 0.0   # half-fan offset on some scans
        plan, b, meta = gtb.phantom.make_osmom_scan(sp, S, 1e5, cuda, offset_mm=off)
        out.append((sp, S, plan, b, meta))
    return out


def test_fused_equals_alone(gtb, O, cuda):
    import torch
    L = gtb._lib
    scans = _scans(gtb, cuda, 8, 301)
    iters = [3, 2, 3, 1, 2, 3, 2, 3]
    jobs, alone, alone_res, outs, res = [], [], [], [], []
    for i, (sp, S, plan, b, _) in enumerate(scans):
        plan.set_option(L.CBCT_OPT_FORWARD_KERNEL, KERNELS[i % len(KERNELS)])
        if i == 5:
            b = b.to(torch.bfloat16)      # 16-bit measurements (fp32 volume)
        x0 = torch.full(plan.vol_shape, 0.01, dtype=torch.float32, device=cuda) if i == 3 else None
        beta, gamma = 1.0 - 0.1 * (i % 3), 0.05 * (i % 2)
        za = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
        ra = torch.zeros(iters[i] * S, dtype=torch.float64, device=cuda)
        plan.osmom(b, za, x0, iters[i], beta=beta, gamma=gamma, nonneg=True, use_graph=True, resid=ra)
        alone.append(za)
        alone_res.append(ra)
        z = torch.full(plan.vol_shape, -1.0, dtype=torch.float32, device=cuda)
        r = torch.full((iters[i] * S,), -1.0, dtype=torch.float64, device=cuda)
        outs.append(z)
        res.append(r)
        jobs.append(dict(plan=plan, b=b, z=z, x0=x0, iterations=iters[i], beta=beta, gamma=gamma, nonneg=True,
                         resid=r))
    torch.cuda.synchronize()
    variants = {s[2].forward_variant() for s in scans}
    assert {"tma-slab", "tma-pair", "tma-quad"} <= variants, variants
    gtb.batch_osmom(jobs, fused=True)
    for i in range(len(jobs)):
        assert torch.equal(alone[i], outs[i]), i
        assert torch.equal(alone_res[i], res[i]), i
    # one of them against the FP64 oracle (fp32 measurements, automatic kernel)
    sp, S, plan, b, (ang, off, sizes, oc) = scans[0]
    nx, ny, nz = sp["n"]
    g = O.Geometry(nx, ny, nz, float(nx), float(ny), float(nz), sp["W"], sp["H"], sp["W"] * sp["pitch"],
                   sp["H"] * sp["pitch"], 1000.0, 1500.0)
    zr, _ = O.osmom(g, b.double().cpu().numpy(), ang, off, sizes, np.asarray(oc, np.int32), iters=iters[0],
                    nonneg=True)
    pre = O.backproject(g, O.forward(g, np.ones((nz, ny, nx)), ang, off), ang, off)
    seen = pre > 1e-2 * pre.max()     # voxels the scan measures (see test_batch_gpu.py)
    assert seen.mean() > 0.5
    assert O.rel_l2(outs[0].cpu().numpy()[seen], zr[seen]) < TOL


def test_fused_many_scans_repeat(gtb, cuda):
    """Twenty scans in one fused call, twice: the same bits both times and the
    same as the stream-pool executor."""
    import torch
    scans = _scans(gtb, cuda, 20, 401)
    outs = [[torch.empty(s[2].vol_shape, dtype=torch.float32, device=cuda) for s in scans] for _ in range(3)]
    for k, fused in enumerate([True, True, False]):
        jobs = [dict(plan=s[2], b=s[3], z=outs[k][i], iterations=2, nonneg=True) for i, s in enumerate(scans)]
        gtb.batch_osmom(jobs, n_streams=4, fused=fused)
    for i in range(len(scans)):
        assert torch.equal(outs[0][i], outs[1][i]), i
        assert torch.equal(outs[0][i], outs[2][i]), i


def test_fused_reports_the_failing_item(gtb, O, cuda):
    """One item's bounded waits give up at once (limit 0): the fused batch
    returns CBCT_ERR_TIMEOUT, and the other item, which shares its work-list
    launches, is still exact."""
    import torch
    L = gtb._lib
    scans = _scans(gtb, cuda, 2, 501)
    scans[1][2].set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    ref = torch.empty(scans[0][2].vol_shape, dtype=torch.float32, device=cuda)
    scans[0][2].osmom(scans[0][3], ref, None, 2, nonneg=True)
    zs = [torch.empty(s[2].vol_shape, dtype=torch.float32, device=cuda) for s in scans]
    jobs = [dict(plan=s[2], b=s[3], z=zs[i], iterations=2, nonneg=True) for i, s in enumerate(scans)]
    with pytest.raises(L.CbctError) as ei:
        gtb.batch_osmom(jobs, fused=True)
    assert ei.value.status == L.CBCT_ERR_TIMEOUT, str(ei.value)
    assert "batch item 1" in str(ei.value)
    assert torch.equal(zs[0], ref)
    assert scans[1][2].read_flags() == (0, 0)    # read and cleared by the batch
    scans[1][2].set_option(L.CBCT_OPT_WAIT_LIMIT, 1 << 22)
    gtb.batch_osmom(jobs, fused=True)
    ref1 = torch.empty_like(zs[1])
    scans[1][2].osmom(scans[1][3], ref1, None, 2, nonneg=True)
    assert torch.equal(zs[1], ref1)


def test_fused_rejects(gtb, cuda):
    import torch
    L = gtb._lib
    sp, S, plan, b, _ = _scans(gtb, cuda, 1, 601)[0]
    z1 = torch.empty(plan.vol_shape, device=cuda)
    z2 = torch.empty(plan.vol_shape, device=cuda)
    with pytest.raises(L.CbctError) as ei:
        gtb.batch_osmom([dict(plan=plan, b=b, z=z1), dict(plan=plan, b=b, z=z2)], fused=True)
    assert ei.value.status == L.CBCT_ERR_INVALID_ARGUMENT
    with pytest.raises(L.CbctError) as ei:
        gtb.batch_osmom([dict(plan=plan, b=b, z=z1, storage=L.CBCT_BF16)], fused=True)
    assert ei.value.status == L.CBCT_ERR_UNSUPPORTED


def test_fused_splits_large_groups(gtb, cuda):
    """More scans of one kernel and box width than one work-list launch holds
    (64): the group is split over several launches, results unchanged."""
    import torch
    sp = gtb.phantom.uneven_scans(1, seed0=701, vol_range=(32, 32), z_range=(24, 24), view_range=(24, 24),
                                  width_range=(40, 40))[0]
    sp["pitch"] *= 1.6
    plan0, b, (a, o, sizes, oc) = gtb.phantom.make_osmom_scan(sp, 2, 1e5, cuda)
    ref = torch.empty(plan0.vol_shape, dtype=torch.float32, device=cuda)
    plan0.osmom(b, ref, None, 2, nonneg=True)
    plans = [gtb.Plan(plan0.g, a, o, sizes, oc) for _ in range(130)]
    zs = [torch.empty(plan0.vol_shape, dtype=torch.float32, device=cuda) for _ in plans]
    variants = {p.forward_variant() for p in plans}
    assert len(variants) == 1 and variants <= {"tma-slab", "tma-pair", "tma-quad"}, variants
    gtb.batch_osmom([dict(plan=p, b=b, z=z, iterations=2, nonneg=True) for p, z in zip(plans, zs)], fused=True)
    for z in zs:
        assert torch.equal(z, ref)


def test_fused_mixes_filling_and_small_scans(gtb, cuda):
    """A scan whose forward launches fill the GPU for several waves keeps its
    one-scan launches inside the fused graph; the small scans beside it go
    through the work lists.  Both results are bitwise the solves alone."""
    import torch
    big = dict(seed=811, n=(128, 128, 96), P=144, W=256, H=192, pitch=1.2 * 1.5 * 128 / 256)
    small = gtb.phantom.uneven_scans(2, seed0=812, vol_range=(32, 48), z_range=(24, 32), view_range=(20, 30),
                                     width_range=(40, 56))
    for sp in small:
        sp["pitch"] *= 1.6
    scans = [gtb.phantom.make_osmom_scan(sp, 2, 1e5, cuda) for sp in [big] + small]
    refs, outs = [], []
    for plan, b, _ in scans:
        r = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
        plan.osmom(b, r, None, 2, nonneg=True)
        refs.append(r)
        outs.append(torch.empty_like(r))
    gtb.batch_osmom([dict(plan=s[0], b=s[1], z=z, iterations=2, nonneg=True) for s, z in zip(scans, outs)],
                    fused=True)
    for r, z in zip(refs, outs):
        assert torch.equal(r, z)


def test_fused_graph_is_reused_and_rebuilt_on_plan_change(gtb, cuda):
    """The last fused schedule is replayed for an identical call, and rebuilt
    when a plan changes state (here: a voxel mask set between the calls)."""
    import torch
    scans = _scans(gtb, cuda, 3, 901)
    outs = [torch.empty(s[2].vol_shape, dtype=torch.float32, device=cuda) for s in scans]
    jobs = [dict(plan=s[2], b=s[3], z=z, iterations=2, nonneg=True) for s, z in zip(scans, outs)]
    gtb.batch_osmom(jobs, fused=True)
    first = [z.clone() for z in outs]
    for z in outs:
        z.fill_(-1.0)
    gtb.batch_osmom(jobs, fused=True)            # replayed
    for a, z in zip(first, outs):
        assert torch.equal(a, z)
    plan = scans[1][2]
    mask = torch.ones(plan.vol_shape, dtype=torch.uint8, device=cuda)
    mask[:, :, : plan.vol_shape[2] // 2] = 0
    plan.set_mask(mask)
    gtb.batch_osmom(jobs, fused=True)            # rebuilt: the mask applies
    ref = torch.empty_like(outs[1])
    plan.osmom(scans[1][3], ref, None, 2, nonneg=True)
    assert torch.equal(outs[1], ref)
    assert not torch.equal(outs[1], first[1])
    assert torch.equal(outs[0], first[0]) and torch.equal(outs[2], first[2])

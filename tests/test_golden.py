"""Committed golden vectors (tests/golden/oracle_small.npz, made by
tests/golden/make_golden.py).  CPU: the oracle reproduces them (regression
pin).  GPU: the product path matches them within 1e-4 relative L2."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "oracle_small.npz")
GEOM = dict(nx=24, ny=20, nz=16, lx=24.0, ly=20.0, lz=16.0, W=32, H=24, fov_u=48.0, fov_v=36.0,
            SAD=600.0, SDD=900.0)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def test_oracle_reproduces_golden(O, gold):
    g = O.Geometry(**GEOM)
    a, o, vol, proj = gold["angles"], gold["offsets"], gold["vol"], gold["proj"]
    assert _rel(O.forward(g, vol.astype(np.float64), a, o), gold["forward"]) < 1e-12
    assert _rel(O.backproject(g, proj.astype(np.float64), a, o), gold["backproject"]) < 1e-12
    assert _rel(O.backproject(g, proj.astype(np.float64), a, o, fbp=True), gold["backproject_fdk"]) < 1e-12
    assert _rel(O.fdk(g, proj, a, o, offset_corr=True), gold["fdk"]) < 1e-12
    assert _rel(O.offset_weight(g, proj, o, 0), gold["offset_full"]) < 1e-12
    assert _rel(O.fdk_filter_rows(proj, gold["filter"]), gold["filter_rows"]) < 1e-12
    order, sizes = O.subset_partition(a.size, 3)
    assert np.array_equal(order, gold["order"]) and np.array_equal(sizes, gold["sizes"])
    z, _ = O.osmom(g, gold["b"].astype(np.float64), a[order], o[order], sizes, np.ones(3, np.int32), iters=2,
                   nonneg=True)
    assert _rel(z, gold["osmom"]) < 1e-12
    assert np.array_equal(O.spacecarver(g, proj, a, o, 0.3), gold["spacecarver"])


@pytest.mark.gpu
def test_gpu_matches_golden(gtb, cuda, gold):
    import torch
    G = GEOM
    a, o, vol, proj = gold["angles"], gold["offsets"], gold["vol"], gold["proj"]
    cg = gtb._lib.CbctGeometry(G["SAD"], G["SDD"], G["fov_u"], G["fov_v"], G["W"], G["H"], G["nx"], G["ny"], G["nz"],
                               G["lx"], G["ly"], G["lz"], 1.5)
    plan = gtb.Plan(cg, a, o)
    v = torch.from_numpy(vol).to(cuda)
    p = torch.from_numpy(proj).to(cuda)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(v, out)
    assert _rel(out.cpu().numpy(), gold["forward"]) < 1e-4
    bp = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(p, bp, -1, 0, False)
    assert _rel(bp.cpu().numpy(), gold["backproject"]) < 1e-4
    plan.backproject(p, bp, -1, gtb._lib.CBCT_BP_FDK_WEIGHT, False)
    assert _rel(bp.cpu().numpy(), gold["backproject_fdk"]) < 1e-4
    x = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(p, x, None, gtb._lib.CBCT_FDK_OFFSET)
    assert _rel(x.cpu().numpy(), gold["fdk"]) < 1e-4
    order, sizes = gold["order"], gold["sizes"]
    plan_s = gtb.Plan(cg, a[order], o[order], sizes, [1, 1, 1])
    z = torch.empty(plan_s.vol_shape, dtype=torch.float32, device=cuda)
    plan_s.osmom(torch.from_numpy(gold["b"]).to(cuda), z, None, 2, nonneg=True)
    assert _rel(z.cpu().numpy(), gold["osmom"]) < 1e-4
    xs = torch.empty(plan_s.vol_shape, dtype=torch.float32, device=cuda)
    plan_s.ossart(torch.from_numpy(gold["b"]).to(cuda), xs, None, 2, nonneg=True)
    assert _rel(xs.cpu().numpy(), gold["ossart"]) < 1e-4
    m = torch.zeros(plan.vol_shape, dtype=torch.uint8, device=cuda)
    plan.spacecarver(p, 0.3, m)
    assert np.mean(m.cpu().numpy() != gold["spacecarver"]) < 2e-3

"""Serving loop (cbct_server_*) and 16-bit projection storage on the GPU.

- FDK and OS-MOM with projections stored as float16/bfloat16 match the FP64
  oracle run on the same stored values (rel L2 <= 1e-4);
- a served request equals the same reconstruction through a Plan (bitwise);
- each result is bitwise the same served alone and served in a mix of
  concurrent requests of uneven sizes, kinds and storage types;
- admission keeps the admitted footprints within the budget, and a request
  that fails does not disturb the others."""
import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _stored(x, dtype):
    """x rounded to a torch storage dtype, back in float64."""
    import torch
    return torch.from_numpy(np.asarray(x, np.float32)).to(dtype).double().numpy()


@pytest.mark.parametrize("dtype", ["float16", "bfloat16"])
def test_fdk_16bit_projections(gtb, O, cuda, dtype):
    import torch
    td = getattr(torch, dtype)
    case = make("offset")
    g = case.oracle_geom(O)
    p = np.random.default_rng(11).uniform(0, 1, (case.angles.size, case.H, case.W))
    ref = O.fdk(g, _stored(p, td), case.angles, case.offsets, offset_corr=True)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(td).to(cuda)
    out = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(pt, out, None, gtb._lib.CBCT_FDK_OFFSET)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL
    # the storage rounding itself, against the FP32 input (reported bound)
    full = O.fdk(g, p.astype(np.float32).astype(np.float64), case.angles, case.offsets, offset_corr=True)
    assert O.rel_l2(out.cpu().numpy(), full) < (2e-3 if dtype == "float16" else 1.5e-2)


@pytest.mark.parametrize("dtype", ["float16", "bfloat16"])
def test_osmom_16bit_measurements(gtb, O, cuda, dtype):
    import torch
    td = getattr(torch, dtype)
    case = make("cube")
    ell = gtb.phantom.ellipsoids(13, (case.lx, case.ly, case.lz), n=5)
    g = case.oracle_geom(O)
    b = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, b = case.angles[order] - case.angles.min(), case.offsets[order], b[order]
    oc = np.zeros(S, np.int32)
    zr, _ = O.osmom(g, _stored(b, td), a, o, sizes, oc, iters=3, nonneg=True)
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes, oc)
    bt = torch.from_numpy(b.astype(np.float32)).to(td).to(cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(bt, z, None, 3, nonneg=True)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL


def _scan(gtb, spec, cuda, offset_mm=0.0):
    """Geometry, acquisition-order angles/offsets and exact line integrals
    (host float32) of one seeded scan shape."""
    import torch
    L = gtb._lib
    nx, ny, nz = spec["n"]
    P, W, H, pitch = spec["P"], spec["W"], spec["H"], spec["pitch"]
    g = L.CbctGeometry(1000.0, 1500.0, W * pitch, H * pitch, W, H, nx, ny, nz, float(nx), float(ny), float(nz), 1.5)
    ang = gtb.phantom.circular_orbit(P)
    off = np.tile(np.array([[offset_mm, 0.0]], np.float32), (P, 1))
    plan = gtb.Plan(g, ang, off)
    ell = torch.from_numpy(gtb.phantom.ellipsoids(spec["seed"], (nx, ny, nz), n=6).reshape(-1)).to(cuda)
    proj = torch.empty(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.phantom_project(ell, proj)
    return g, ang, off, proj.cpu()


def test_served_fdk_equals_plan(gtb, cuda):
    import torch
    spec = dict(seed=3, n=(48, 40, 32), P=60, W=96, H=72, pitch=1.2 * 1.5 * 48 / 96 * 1.3)
    g, ang, off, proj = _scan(gtb, spec, cuda, offset_mm=12.0)
    vol = torch.empty((32, 40, 48), dtype=torch.float32)
    with gtb.Server(4e9, 2) as srv:
        t = srv.submit(srv.fdk_request(g, ang, off, proj, vol, filt=gtb.hann_ramp_filter(96)))
        rec = srv.wait(t)
    assert rec["bytes_peak"] <= rec["bytes_reserved"]
    plan = gtb.Plan(g, ang, off)
    flags = gtb._lib.CBCT_FDK_OFFSET if gtb.operators.offset_override(g, off) else 0
    assert flags  # 12 mm > 0.1 * detector width
    ref = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(proj.to(cuda), ref, gtb.hann_ramp_filter(96), flags)
    assert torch.equal(vol, ref.cpu())


def test_served_osmom_equals_plan_and_oracle(gtb, O, cuda):
    import torch
    spec = dict(seed=4, n=(40, 40, 24), P=48, W=80, H=60, pitch=1.2 * 1.5 * 40 / 80 * 1.6)
    g, ang, off, proj = _scan(gtb, spec, cuda)
    vol = torch.full((24, 40, 40), -1.0, dtype=torch.float32).pin_memory()
    S = 4
    with gtb.Server(4e9, 2) as srv:
        rec = srv.wait(srv.submit(srv.osmom_request(g, ang, off, proj.pin_memory(), vol, S, iterations=3)))
    assert rec["status"] == 0 and rec["bytes_peak"] <= rec["bytes_reserved"]
    order, sizes = gtb.subset_partition(ang.size, S)
    a, o = ang[order] - ang.min(), off[order]
    plan = gtb.Plan(g, a, o, sizes)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(proj[order].contiguous().to(cuda), z, None, 3, nonneg=True)
    assert torch.equal(vol, z.cpu())
    og = O.Geometry(40, 40, 24, 40.0, 40.0, 24.0, 80, 60, g.fov_u, g.fov_v, 1000.0, 1500.0)
    zr, _ = O.osmom(og, proj[order].double().numpy(), a, o, sizes, np.zeros(S, np.int32), iters=3, nonneg=True)
    assert O.rel_l2(vol.numpy(), zr) < TOL


def _mix(gtb, cuda):
    """Uneven requests: FDK and OS-MOM, float32 / bfloat16 / float16 storage."""
    import torch
    specs = gtb.phantom.uneven_scans(6, seed0=300, vol_range=(32, 72), z_range=(24, 48), view_range=(30, 90),
                                     width_range=(48, 112))
    kinds = ["fdk", "osmom", "fdk", "osmom", "fdk", "osmom"]
    dts = [torch.float32, torch.bfloat16, torch.float16, torch.float32, torch.bfloat16, torch.float16]
    out = []
    for sp, k, dt in zip(specs, kinds, dts):
        sp["pitch"] *= 1.6
        g, ang, off, proj = _scan(gtb, sp, cuda, offset_mm=0.0)
        out.append((k, g, ang, off, proj.to(dt).pin_memory()))
    return out


def _request(gtb, item, vol):
    k, g, ang, off, proj = item
    if k == "fdk":
        return gtb.Server.fdk_request(g, ang, off, proj, vol)
    return gtb.Server.osmom_request(g, ang, off, proj, vol, 4, iterations=3, use_graph=True)


def test_alone_equals_mix(gtb, cuda):
    import torch
    items = _mix(gtb, cuda)
    shape = lambda it: (it[1].nz, it[1].ny, it[1].nx)
    alone = [torch.full(shape(it), -1.0).pin_memory() for it in items]
    with gtb.Server(8e9, 1) as srv:
        for it, v in zip(items, alone):
            srv.wait(srv.submit(_request(gtb, it, v)))
    mixed = [torch.full(shape(it), -2.0).pin_memory() for it in items]
    with gtb.Server(8e9, 4) as srv:
        tickets = [srv.submit(_request(gtb, it, v)) for it, v in zip(items, mixed)]
        recs = [srv.wait(t) for t in tickets]
    for a, m in zip(alone, mixed):
        assert torch.equal(a, m)
    # the mix did run requests at the same time
    spans = sorted((r["t_admit"], r["t_done"]) for r in recs)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    assert len({r["slot"] for r in recs}) > 1


def test_budget_admission(gtb, cuda):
    import torch
    item = _mix(gtb, cuda)[1]
    vols = [torch.empty((item[1].nz, item[1].ny, item[1].nx)) for _ in range(3)]
    reqs = [_request(gtb, item, v) for v in vols]
    need = gtb.Server.request_bytes(reqs[0])
    with gtb.Server(int(need * 1.5), 4) as srv:     # room for one request at a time
        recs = [srv.wait(t) for t in [srv.submit(r) for r in reqs]]
    spans = sorted((r["t_admit"], r["t_done"]) for r in recs)
    assert all(spans[i + 1][0] >= spans[i][1] for i in range(len(spans) - 1))
    assert all(r["bytes_peak"] <= r["bytes_reserved"] == need for r in recs)
    assert torch.equal(vols[0], vols[1]) and torch.equal(vols[0], vols[2])
    with gtb.Server(need // 2, 1) as srv:
        with pytest.raises(gtb.CbctError, match="budget"):
            srv.submit(reqs[0])


def test_failed_request_is_isolated(gtb, cuda):
    import torch
    L = gtb._lib
    items = _mix(gtb, cuda)[:2]
    good_vol = torch.empty((items[0][1].nz, items[0][1].ny, items[0][1].nx))
    # A detector wider than the FDK filter's shared-memory transform supports.
    W = 4100
    g = L.CbctGeometry(1000.0, 1500.0, W * 0.1, 0.2, W, 2, 16, 16, 16, 16.0, 16.0, 16.0, 1.5)
    bad_proj = torch.zeros((2, 2, W))
    bad_vol = torch.empty((16, 16, 16))
    with gtb.Server(8e9, 2) as srv:
        tb = srv.submit(srv.fdk_request(g, np.array([0.0, 90.0], np.float32), None, bad_proj, bad_vol))
        tg = srv.submit(_request(gtb, items[0], good_vol))
        rb = srv.wait(tb, check=False)
        rg = srv.wait(tg)
        with pytest.raises(gtb.CbctError):
            srv.wait(tb)          # collected already
    assert rb["status"] == 4 and "FDK filter" in rb["message"]
    assert rg["status"] == 0 and torch.isfinite(good_vol).all()

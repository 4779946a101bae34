"""Device-side failure path: a bounded wait that runs out becomes a status.

Every TMA-staged projector kernel waits for its next shared-memory stage with
a bounded number of polls (CBCT_OPT_WAIT_LIMIT).  A thread block that gives
up records the event in the plan's flag word, waits with the default limit for
the loads it still has in flight, and exits with its rays or voxels
unfinished; nothing hangs and nothing faults.  With the limit set to 0 every
such wait gives up at once, so these tests make the failure happen on purpose
and check that the host sees it: cbct_plan_check (and the solve, FDK,
host-streaming and batch entry points on their own) return CBCT_ERR_TIMEOUT,
the flag word counts the events, and the same plan, with the default limit
restored, computes correct results again (the CUDA context is still usable).
"""
import ctypes as C

import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu
TOL = 1e-4
DEFAULT_POLLS = 1 << 22


def _phantom(gtb, case, O, seed=3):
    ell = gtb.phantom.ellipsoids(seed, (case.lx, case.ly, case.lz), n=6).astype(np.float64)
    return O.phantom_voxelize(case.oracle_geom(O), ell, ss=2)


def _expect_timeout(gtb, fn):
    with pytest.raises(gtb._lib.CbctError) as ei:
        fn()
    assert ei.value.status == gtb._lib.CBCT_ERR_TIMEOUT, str(ei.value)


@pytest.mark.parametrize("kernel", [1, 3, 4, 5])   # slab, fan, row pairs, row quads
def test_forward_wait_expiry(gtb, O, cuda, kernel):
    import torch
    L = gtb._lib
    case = make("cube")
    vol = _phantom(gtb, case, O)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    plan.set_option(L.CBCT_OPT_FORWARD_KERNEL, kernel)
    assert plan.forward_variant().startswith("tma-")
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    plan.forward(v, out)                       # asynchronous: returns CBCT_OK
    flags = plan.read_flags(reset=False)
    assert flags[1] > 0, flags
    _expect_timeout(gtb, plan.check)
    assert plan.read_flags() == (0, 0)         # the check cleared them
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, DEFAULT_POLLS)
    plan.forward(v, out)
    plan.check()
    ref = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


def test_backproject_wait_expiry(gtb, O, cuda):
    import torch
    L = gtb._lib
    case = make("cube")
    p = np.random.default_rng(1).uniform(0, 1, (case.angles.size, case.H, case.W))
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    plan.backproject(pt, out)
    assert plan.read_flags(reset=False)[1] > 0
    _expect_timeout(gtb, plan.check)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, DEFAULT_POLLS)
    plan.backproject(pt, out)
    plan.check()
    ref = O.backproject(case.oracle_geom(O), p, case.angles, case.offsets)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("use_graph", [False, True])
def test_solve_returns_timeout(gtb, O, cuda, use_graph):
    """cbct_osmom_solve reads the flag words on return and fails; a captured
    graph made with the short limit is dropped when the limit changes."""
    import torch
    L = gtb._lib
    case = make("cube")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(13, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, bp = case.angles[order], case.offsets[order], b[order]
    plan = gtb.Plan(case.cgeom(gtb), a, o, sizes)
    bt = torch.from_numpy(bp.astype(np.float32)).to(cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    _expect_timeout(gtb, lambda: plan.osmom(bt, z, None, 2, nonneg=True, use_graph=use_graph))
    assert plan.read_flags() == (0, 0)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, DEFAULT_POLLS)
    plan.osmom(bt, z, None, 2, nonneg=True, use_graph=use_graph)
    zr, _ = O.osmom(g, bp, a, o, sizes, np.zeros(S, np.int32), iters=2, nonneg=True)
    assert O.rel_l2(z.cpu().numpy(), zr) < TOL


def test_status_check_off_leaves_it_to_the_caller(gtb, O, cuda):
    import torch
    L = gtb._lib
    case = make("cube")
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    plan.set_option(L.CBCT_OPT_STATUS_CHECK, 0)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    b = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.osmom(b, z, None, 1)                  # asynchronous, returns CBCT_OK
    _expect_timeout(gtb, plan.check)


def test_fdk_returns_timeout(gtb, O, cuda):
    import torch
    L = gtb._lib
    case = make("cube")
    p = np.random.default_rng(8).uniform(0, 1, (case.angles.size, case.H, case.W))
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    pt = torch.from_numpy(p.astype(np.float32)).to(cuda)
    out = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    _expect_timeout(gtb, lambda: plan.fdk(pt, out))
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, DEFAULT_POLLS)
    plan.fdk(pt, out)
    ref = O.fdk(case.oracle_geom(O), p, case.angles, case.offsets)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL


def test_host_stream_returns_timeout(gtb, O, cuda):
    """cbct_host_forward synchronises anyway and reports the flags itself."""
    L = gtb._lib
    case = make("cube")
    vol = _phantom(gtb, case, O).astype(np.float32)
    P = case.angles.size
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, [4, 4, P - 8])
    plan.set_option(L.CBCT_OPT_FORWARD_KERNEL, 1)
    proj = np.zeros((P, case.H, case.W), np.float32)
    vi = np.arange(P, dtype=np.int32)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    st = L.lib().cbct_host_forward(plan.handle, 0, 3, vol.ctypes.data, proj.ctypes.data, vi.ctypes.data, 0, None)
    assert st == L.CBCT_ERR_TIMEOUT, L.status_string(st)
    plan.set_option(L.CBCT_OPT_WAIT_LIMIT, DEFAULT_POLLS)
    L.call("cbct_host_forward", plan.handle, 0, 3, vol.ctypes.data, proj.ctypes.data, vi.ctypes.data, 0, None)
    ref = O.forward(case.oracle_geom(O), vol.astype(np.float64), case.angles, case.offsets)
    assert O.rel_l2(proj, ref) < TOL


def test_batch_reports_the_failing_item(gtb, O, cuda):
    """One item of a batch fails on the device: the batch returns its status,
    and the other item's result is still exact."""
    import torch
    L = gtb._lib
    case = make("cube")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(5, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, bp = case.angles[order], case.offsets[order], b[order]
    plans = [gtb.Plan(case.cgeom(gtb), a, o, sizes) for _ in range(2)]
    plans[1].set_option(L.CBCT_OPT_WAIT_LIMIT, 0)
    bt = torch.from_numpy(bp.astype(np.float32)).to(cuda)
    zs = [torch.empty(plans[0].vol_shape, dtype=torch.float32, device=cuda) for _ in range(2)]
    jobs = [dict(plan=plans[i], b=bt, z=zs[i], iterations=2, nonneg=True) for i in range(2)]
    _expect_timeout(gtb, lambda: gtb.batch_osmom(jobs, n_streams=2))
    zr, _ = O.osmom(g, bp, a, o, sizes, np.zeros(S, np.int32), iters=2, nonneg=True)
    assert O.rel_l2(zs[0].cpu().numpy(), zr) < TOL
    assert plans[1].read_flags() == (0, 0)

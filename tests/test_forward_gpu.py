"""Forward projector (mult_M) on the GPU against the FP64 oracle.

Tolerance: relative L2 <= 1e-4 against the FP64 oracle of the same projector
geometry (the FP32 path's bound); the kernels typically land near 1e-6.
"""
import numpy as np
import pytest

from cases import ALL, make

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _phantom(case, O, seed=3):
    from gt_tomography_b200 import phantom
    ell = phantom.ellipsoids(seed, (case.lx, case.ly, case.lz), n=6)
    return ell, O.phantom_voxelize(case.oracle_geom(O), ell.astype(np.float64), ss=2)


@pytest.mark.parametrize("name", ALL)
@pytest.mark.parametrize("variant", ["auto", "gather", "fan", "pair", "quad"])
def test_forward_matches_oracle(gtb, O, cuda, name, variant):
    import torch
    case = make(name)
    _, vol = _phantom(case, O)
    ref = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets, spp=case.spp)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    if variant == "gather":
        plan.set_option(gtb._lib.CBCT_OPT_FORCE_GATHER, 1)
    elif variant == "fan":
        plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 3)
    elif variant == "pair":
        plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 4)
    elif variant == "quad":
        plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 5)
    plan.set_option(gtb._lib.CBCT_OPT_DEBUG_CHECKS, 1)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(v, out)
    got = out.cpu().numpy()
    assert plan.read_flags() == (0, 0)
    err = O.rel_l2(got, ref)
    assert err < TOL, (name, variant, plan.forward_variant(), err)


def test_variant_selection(gtb, cuda):
    """Automatic choice: row pairs where adjacent detector rows stay within one
    z texel of each other ("offset": 0.88 texel), else per-ray slabs ("cube":
    1.02 texel); every variant can be forced."""
    plan = gtb.Plan(make("offset").cgeom(gtb), make("offset").angles, make("offset").offsets)
    assert plan.forward_variant() == "tma-pair"
    case = make("cube")
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    assert plan.forward_variant() == "tma-slab"
    plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 3)
    assert plan.forward_variant() == "tma-fan"
    plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 4)
    assert plan.forward_variant() == "tma-pair"
    plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 5)
    assert plan.forward_variant() == "tma-quad"
    plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, 2)
    assert plan.forward_variant() == "gather"


@pytest.mark.parametrize("name", ["short", "cube", "offset", "aniso"])
def test_kernels_bitwise_equal(gtb, O, cuda, name):
    """Slab, row-pair, row-quad, fan and gather kernels evaluate the same
    samples in the same order."""
    import torch
    case = make(name)
    _, vol = _phantom(case, O, seed=9)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    plan.set_option(gtb._lib.CBCT_OPT_DEBUG_CHECKS, 1)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    outs = {}
    for k in (1, 4, 5, 3, 2):
        plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, k)
        out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
        plan.forward(v, out)
        outs[plan.forward_variant()] = out
        assert plan.read_flags() == (0, 0)
    assert set(outs) == {"tma-slab", "tma-pair", "tma-quad", "tma-fan", "gather"}
    assert torch.equal(outs["tma-slab"], outs["tma-fan"])
    assert torch.equal(outs["tma-slab"], outs["tma-pair"])
    assert torch.equal(outs["tma-slab"], outs["tma-quad"])
    # the gather kernel interpolates with another FMA arrangement: equal to rounding
    a, b = outs["tma-slab"].double(), outs["gather"].double()
    assert float((a - b).norm() / b.norm()) < 1e-6


def test_forward_accumulate_and_subsets(gtb, O, cuda):
    import torch
    case = make("offset")
    _, vol = _phantom(case, O, seed=5)
    ref = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets)
    sizes = [5, 6, 5]
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, sizes)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    full = torch.ones(plan.proj_shape(), dtype=torch.float32, device=cuda)
    first = 0
    for s, n in enumerate(sizes):
        plan.forward(v, full[first:first + n], s, accumulate=True)
        first += n
    err = O.rel_l2(full.cpu().numpy() - 1.0, ref)
    assert err < TOL


def test_forward_residual_fused(gtb, O, cuda):
    """r = w_off * (A x - b) and ||A x - b||^2 in FP64 (osMOMSolverD.h:144-149 +
    the weighted copy of cuConebeamProjectionOperator.cpp:101-102)."""
    import torch
    case = make("offset")
    _, vol = _phantom(case, O, seed=7)
    g = case.oracle_geom(O)
    ax = O.forward(g, vol, case.angles, case.offsets)
    rng = np.random.default_rng(1)
    b = (ax + rng.normal(0, 0.05, ax.shape)).astype(np.float32)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    bt = torch.from_numpy(b).to(cuda)
    r = torch.empty_like(bt)
    n2 = torch.zeros(1, dtype=torch.float64, device=cuda)
    plan.forward_residual(v, bt, r, -1, 1.0, True, n2)
    d = ax - b.astype(np.float64)
    ref = O.offset_weight(g, d, case.offsets, 0)
    assert O.rel_l2(r.cpu().numpy(), ref) < TOL
    assert abs(n2.item() - float((d * d).sum())) / float((d * d).sum()) < 1e-4


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
def test_forward_16bit_storage(gtb, O, cuda, dtype):
    """16-bit volume storage, FP32 interpolation: error is the storage rounding."""
    import torch
    case = make("cube")
    _, vol = _phantom(case, O)
    ref = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    plan.set_option(gtb._lib.CBCT_OPT_DEBUG_CHECKS, 1)
    td = torch.float16 if dtype == "f16" else torch.bfloat16
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda).to(td)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(v, out, vol_dtype=gtb.CBCT_F16 if dtype == "f16" else gtb.CBCT_BF16)
    assert plan.read_flags() == (0, 0)
    err = O.rel_l2(out.cpu().numpy(), ref)
    assert err < (1e-3 if dtype == "f16" else 8e-3), err


def test_forward_analytic_kat(gtb, O, cuda):
    """Known answer: the discrete line integral of a supersampled ellipsoid
    phantom approaches the exact chord integral (loose bound: voxelisation)."""
    import torch
    case = make("c1small")
    ell, vol = _phantom(case, O, seed=11)
    exact = O.phantom_project(case.oracle_geom(O), ell.astype(np.float64), case.angles, case.offsets)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(v, out)
    assert O.rel_l2(out.cpu().numpy(), exact) < 0.03


def test_forward_deterministic(gtb, O, cuda):
    import torch
    case = make("aniso")
    _, vol = _phantom(case, O)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    a = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    b = torch.zeros_like(a)
    plan.forward(v, a)
    plan.forward(v, b)
    assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
def test_forward_16bit_full_size_offset(gtb, cuda, dtype):
    """The benchmark geometry (256^3, 512x384 at 0.8 mm, 80 mm offset) with a
    16-bit volume: the wider 16-bit box needs the opt-in shared-memory limit
    (static + dynamic above 48 KB).  The 16-bit kernel reads the stored values
    exactly and interpolates in FP32, so it equals the fp32 kernel on the
    rounded volume bitwise."""
    import torch
    L = gtb._lib
    g = L.CbctGeometry(1000.0, 1500.0, 512 * 0.8, 384 * 0.8, 512, 384, 256, 256, 256, 256.0, 256.0, 256.0, 1.5)
    ang = gtb.phantom.circular_orbit(360)[::10].copy()
    off = np.tile(np.array([[80.0, 0.0]], np.float32), (ang.size, 1))
    plan = gtb.Plan(g, ang, off)
    ell = torch.from_numpy(gtb.phantom.ellipsoids(4, (256.0, 256.0, 256.0)).reshape(-1)).to(cuda)
    vol = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    gtb.phantom_voxelize(g, ell, vol, 1)
    td = torch.float16 if dtype == "f16" else torch.bfloat16
    v16 = vol.to(td).contiguous()
    a = torch.empty(plan.proj_shape(), dtype=torch.float32, device=cuda)
    b = torch.empty_like(a)
    plan.forward(v16, a, vol_dtype=gtb.CBCT_F16 if dtype == "f16" else gtb.CBCT_BF16)
    plan.forward(v16.float().contiguous(), b)
    assert plan.forward_variant() == "tma-quad"
    assert torch.equal(a, b)
    for k, name in ((1, "tma-slab"), (4, "tma-pair")):
        plan.set_option(L.CBCT_OPT_FORWARD_KERNEL, k)
        plan.forward(v16, b, vol_dtype=gtb.CBCT_F16 if dtype == "f16" else gtb.CBCT_BF16)
        assert plan.forward_variant() == name
        assert torch.equal(a, b)


@pytest.mark.parametrize("name", ["cube", "short"])
def test_autotune_keeps_results(gtb, O, cuda, name):
    """The autotuner times the variants, keeps the fastest, and the plan's
    results stay within the FP32 tolerance of the FP64 oracle."""
    import torch
    case = make(name)
    _, vol = _phantom(case, O)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets, [7, case.angles.size - 7])
    t = plan.autotune()
    assert t["forward_slab"] is not None and t["forward_gather"] is not None and t["backproject_global"] is not None
    fastest = min((v, k) for k, v in t.items() if k.startswith("forward_") and k != "forward_variant"
                  and v is not None)[1]
    assert t["forward_variant"] == {"forward_slab": "tma-slab", "forward_fan": "tma-fan",
                                    "forward_gather": "gather", "forward_pair": "tma-pair",
                                    "forward_quad": "tma-quad"}[fastest]
    plan.set_option(gtb._lib.CBCT_OPT_DEBUG_CHECKS, 1)
    v = torch.from_numpy(vol.astype(np.float32)).to(cuda)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(v, out)
    assert plan.read_flags() == (0, 0)
    ref = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets)
    assert O.rel_l2(out.cpu().numpy(), ref) < TOL
    back = torch.zeros(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.backproject(out, back)
    refb = O.backproject(case.oracle_geom(O), out.cpu().numpy().astype(np.float64), case.angles, case.offsets)
    assert O.rel_l2(back.cpu().numpy(), refb) < TOL

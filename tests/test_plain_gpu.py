"""The plain reference-replica GPU path (include/cbct_plain.h).

It restates the reference's CUDA kernels with hardware texture filtering, so
it stands in for "the reference's CUDA projector outputs".  The bounds below
are about twice the values measured on a B200 (printed by each test):

  forward, plain vs the oracle's texture-emulating mode  2.1e-4 .. 2.6e-4
  forward, plain vs exact FP64                            2.4e-4 .. 2.9e-4
  back-projection, plain vs texture mode / exact          4.3e-4 / 5.6e-4
  product vs plain (64^3 from 45 views)                   1.2e-4 (product vs FP64: 2.7e-6)
  OS-MOM, 2 iterations, plain vs FP64                     3.7e-4
  FDK (cuFFT row filter, texture back-projection) vs FP64 2.1e-3 .. 2.3e-3

The texture unit interpolates with 9-bit weights (8 fractional bits): each
tap's weight is the fraction rounded to a multiple of 1/256.  The
texture-emulating oracle quantises its FP64 fractions the same way, but the
replica's fractions come from FP32 fast-math coordinates that differ from the
FP64 ones by about 1e-6 relative (1e-4 texel at 128 texels), enough to move a
few per cent of the taps across a 1/256 step.  Those flipped steps leave the
emulation about 2e-4 from the hardware, close to the whole quantisation
error, so the emulation does not pin the replica much tighter than exact FP64
does; the ramp filter's high frequencies make the FDK's share ten times
larger.  The product's FP32 software interpolation has none of this: it is
within 3e-6 of FP64."""
import ctypes as C

import numpy as np
import pytest

from cases import make

pytestmark = pytest.mark.gpu


def _plain_forward(gtb, case, vol):
    import torch
    L = gtb._lib
    g = case.cgeom(gtb)
    v = torch.from_numpy(vol.astype(np.float32)).cuda()
    out = torch.zeros((case.angles.size, case.H, case.W), dtype=torch.float32, device="cuda")
    a = np.ascontiguousarray(case.angles, np.float32)
    o = np.ascontiguousarray(case.offsets, np.float32)
    L.call("cbct_plain_forward", C.byref(g), a.ctypes.data, o.ctypes.data, a.size, v.data_ptr(), out.data_ptr(), 0)
    return out.cpu().numpy()


def _plain_bp(gtb, case, proj, offcorr=0):
    import torch
    L = gtb._lib
    g = case.cgeom(gtb)
    p = torch.from_numpy(proj.astype(np.float32)).cuda()
    out = torch.zeros((case.nz, case.ny, case.nx), dtype=torch.float32, device="cuda")
    a = np.ascontiguousarray(case.angles, np.float32)
    o = np.ascontiguousarray(case.offsets, np.float32)
    L.call("cbct_plain_backproject", C.byref(g), a.ctypes.data, o.ctypes.data, a.size, p.data_ptr(), out.data_ptr(),
           offcorr, 0)
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["cube", "aniso", "offset"])
def test_plain_forward_vs_oracle_modes(gtb, O, cuda, name):
    case = make(name)
    ell = gtb.phantom.ellipsoids(3, (case.lx, case.ly, case.lz), n=6).astype(np.float64)
    g = case.oracle_geom(O)
    vol = O.phantom_voxelize(g, ell, ss=2)
    plain = _plain_forward(gtb, case, vol)
    tex = O.forward(g, vol, case.angles, case.offsets, mode=1)
    exact = O.forward(g, vol, case.angles, case.offsets, mode=0)
    e_tex, e_exact = O.rel_l2(plain, tex), O.rel_l2(plain, exact)
    print(f"{name}: plain vs texture-emulating oracle {e_tex:.2e}, vs exact FP64 {e_exact:.2e}")
    assert e_tex < 5e-4 and e_exact < 6e-4


def test_plain_backproject_vs_oracle(gtb, O, cuda):
    case = make("offset")
    rng = np.random.default_rng(0)
    p = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    g = case.oracle_geom(O)
    plain = _plain_bp(gtb, case, p, offcorr=1)
    pw = O.offset_weight(g, p, case.offsets, 0)
    tex = O.backproject(g, pw, case.angles, case.offsets, mode=1)
    exact = O.backproject(g, pw, case.angles, case.offsets, mode=0)
    e_tex, e_exact = O.rel_l2(plain, tex), O.rel_l2(plain, exact)
    print(f"plain BP vs texture-emulating oracle {e_tex:.2e}, vs exact FP64 {e_exact:.2e}")
    assert e_tex < 9e-4 and e_exact < 1.2e-3


def test_product_path_vs_plain_path(gtb, O, cuda):
    """The product's FP32 software interpolation against the reference-style
    texture path on identical geometry: they differ by the texture unit's
    weight quantisation, while the product tracks the FP64 oracle to ~1e-6."""
    import torch
    case = make("c1small")
    ell = gtb.phantom.ellipsoids(5, (case.lx, case.ly, case.lz), n=8).astype(np.float64)
    g = case.oracle_geom(O)
    vol = O.phantom_voxelize(g, ell, ss=2)
    plain = _plain_forward(gtb, case, vol)
    plan = gtb.Plan(case.cgeom(gtb), case.angles, case.offsets)
    out = torch.zeros(plan.proj_shape(), dtype=torch.float32, device=cuda)
    plan.forward(torch.from_numpy(vol.astype(np.float32)).to(cuda), out)
    ours = out.cpu().numpy()
    exact = O.forward(g, vol, case.angles, case.offsets)
    d_plain, d_ours = O.rel_l2(ours, plain), O.rel_l2(ours, exact)
    print(f"product vs plain texture path {d_plain:.2e}; product vs FP64 {d_ours:.2e}; "
          f"plain vs FP64 {O.rel_l2(plain, exact):.2e}")
    assert d_ours < 1e-5 and d_plain < 2.5e-4


def test_plain_osmom_vs_oracle(gtb, O, cuda):
    import torch
    case = make("cube")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(13, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets)
    S = 3
    order, sizes = O.subset_partition(case.angles.size, S)
    a, o, bp = case.angles[order], case.offsets[order], b[order]
    zr, rr = O.osmom(g, bp, a, o, sizes, np.zeros(S, np.int32), iters=2, nonneg=True)
    L = gtb._lib
    cg = case.cgeom(gtb)
    bt = torch.from_numpy(bp.astype(np.float32)).to(cuda)
    z = torch.empty((case.nz, case.ny, case.nx), dtype=torch.float32, device=cuda)
    resid = np.zeros(2 * S)
    sz = np.ascontiguousarray(sizes, np.int32)
    oc = np.zeros(S, np.int32)
    aa, oo = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(o, np.float32)
    L.call("cbct_plain_osmom_solve", C.byref(cg), aa.ctypes.data, oo.ctypes.data, aa.size, sz.ctypes.data, S,
           oc.ctypes.data, bt.data_ptr(), z.data_ptr(), 2, 1, resid.ctypes.data)
    e = O.rel_l2(z.cpu().numpy(), zr)
    print(f"plain OS-MOM vs FP64 oracle {e:.2e}")
    assert e < 8e-4
    r_rel = float(np.max(np.abs(resid - rr) / np.abs(rr)))
    print(f"plain OS-MOM residual norms vs FP64: max relative difference {r_rel:.2e}")
    assert r_rel < 2e-2


@pytest.mark.parametrize("name,batch", [("cube", 20), ("offset", 7)])
def test_plain_fdk_vs_oracle_and_product(gtb, O, cuda, name, batch):
    """The plain FDK (host arrays, batches of views, cuFFT row filter,
    texture back-projection) against the FP64 oracle's FDK and the product's."""
    import torch
    L = gtb._lib
    case = make(name)
    g = case.oracle_geom(O)
    p = np.random.default_rng(8).uniform(0, 1, (case.angles.size, case.H, case.W))
    off = name == "offset"
    ref = O.fdk(g, p, case.angles, case.offsets, offset_corr=off)
    ph = torch.from_numpy(p.astype(np.float32)).pin_memory()
    vol = torch.zeros((case.nz, case.ny, case.nx), dtype=torch.float32).pin_memory()
    a = np.ascontiguousarray(case.angles, np.float32)
    o = np.ascontiguousarray(case.offsets, np.float32)
    cg = case.cgeom(gtb)
    L.call("cbct_plain_fdk", C.byref(cg), a.ctypes.data, o.ctypes.data, a.size, ph.data_ptr(), vol.data_ptr(), None,
           int(off), batch)
    e_ref = O.rel_l2(vol.numpy(), ref)
    plan = gtb.Plan(cg, case.angles, case.offsets)
    prod = torch.empty(plan.vol_shape, dtype=torch.float32, device=cuda)
    plan.fdk(ph.to(cuda), prod, None, L.CBCT_FDK_OFFSET if off else 0)
    e_prod = O.rel_l2(vol.numpy(), prod.cpu().numpy())
    print(f"{name}: plain FDK vs FP64 {e_ref:.2e}, vs product {e_prod:.2e}")
    assert e_ref < 4.5e-3 and e_prod < 4.5e-3

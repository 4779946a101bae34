"""The C++ drop-in for gt-tomography (include/cbct_gadgetron.hpp).

CPU: the header compiles against the Gadgetron interfaces (stand-ins under
tests/gadgetron_stub).  GPU: a C++ program drives CBSubsetOperatorB200 the way
cuCBOS_reconstruct.cpp drives CBSubsetOperator, and its outputs match the FP64
oracle (rel L2 <= 1e-4)."""
import os
import subprocess

import numpy as np
import pytest

from cases import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


PROGRAMS = ["dropin_main", "fdk_main", "bins_main"]


def _compile(out_path, program="dropin_main"):
    lib_dir = os.path.join(ROOT, "gt-tomography_b200", "_build")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wno-unused-function",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "gadgetron_stub"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", program + ".cpp"),
           "-o", out_path, "-L", lib_dir, "-lcbct", f"-Wl,-rpath,{lib_dir}",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("program", PROGRAMS)
def test_dropin_header_compiles(gtb, tmp_path, program):
    _compile(str(tmp_path / program), program)


def _geom_args(case):
    return [str(case.nx), str(case.ny), str(case.nz), str(case.lx), str(case.ly), str(case.lz),
            str(case.W), str(case.H), str(case.fov_u), str(case.fov_v), str(case.SAD), str(case.SDD),
            str(case.angles.size)]


@pytest.mark.gpu
def test_dropin_matches_oracle(gtb, O, cuda, tmp_path):
    case = make("offset")
    g = case.oracle_geom(O)
    exe = str(tmp_path / "dropin_main")
    _compile(exe)
    ell = gtb.phantom.ellipsoids(31, (case.lx, case.ly, case.lz), n=4).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets).astype(np.float32)
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 0.02, (case.nz, case.ny, case.nx)).astype(np.float32)
    d = str(tmp_path)
    case.angles.astype(np.float32).tofile(os.path.join(d, "angles.f32"))
    case.offsets.astype(np.float32).tofile(os.path.join(d, "offsets.f32"))
    b.tofile(os.path.join(d, "b.f32"))
    x.tofile(os.path.join(d, "x.f32"))
    S = 4
    args = [exe, d, str(case.nx), str(case.ny), str(case.nz), str(case.lx), str(case.ly), str(case.lz),
            str(case.W), str(case.H), str(case.fov_u), str(case.fov_v), str(case.SAD), str(case.SDD),
            str(case.angles.size), str(S)]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    P = case.angles.size
    a = np.fromfile(os.path.join(d, "angles_perm.f32"), np.float32)
    o = np.fromfile(os.path.join(d, "offsets_perm.f32"), np.float32).reshape(P, 2)
    order, sizes = O.subset_partition(P, S)
    assert np.array_equal(a, case.angles[order] - case.angles.min())
    ax = np.fromfile(os.path.join(d, "ax.f32"), np.float32).reshape(P, case.H, case.W)
    ref_ax = O.forward(g, x.astype(np.float64), a, o)
    assert O.rel_l2(ax, ref_ax) < 1e-4
    # mult_MH over all subsets with the per-subset sin^2 weight (mean offset 14 > 0.1*64)
    atax = np.fromfile(os.path.join(d, "atax.f32"), np.float32).reshape(case.nz, case.ny, case.nx)
    ref_atax = O.backproject(g, O.offset_weight(g, ax.astype(np.float64), o, 0), a, o)
    assert O.rel_l2(atax, ref_atax) < 1e-4
    z = np.fromfile(os.path.join(d, "z.f32"), np.float32).reshape(case.nz, case.ny, case.nx)
    zr, _ = O.osmom(g, b[order].astype(np.float64), a, o, sizes, np.ones(S, np.int32), iters=2, nonneg=True)
    assert O.rel_l2(z, zr) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("name,batch,custom", [("cube", 5, False), ("offset", 7, True), ("c1small", 20, True)])
def test_fdk_recipe_dropin_matches_oracle(gtb, O, cuda, tmp_path, name, batch, custom):
    """xray/FDK_reconstruct_3d.cpp:124-161 call for call with
    hoCuConebeamProjectionOperatorB200: the FDK volume and the rescaled result
    against the oracle's FDK and recipe.  "offset": the setup's override turns
    offset correction on (mean offset 14 mm > 0.1 x 64 mm), so FDK applies the
    sin^2 weight."""
    case = make(name)
    g = case.oracle_geom(O)
    exe = str(tmp_path / "fdk_main")
    _compile(exe, "fdk_main")
    ell = gtb.phantom.ellipsoids(41, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    b = O.phantom_project(g, ell, case.angles, case.offsets).astype(np.float32)
    d = str(tmp_path)
    case.angles.astype(np.float32).tofile(os.path.join(d, "angles.f32"))
    case.offsets.astype(np.float32).tofile(os.path.join(d, "offsets.f32"))
    b.tofile(os.path.join(d, "b.f32"))
    filt = gtb.hann_ramp_filter(case.W) if custom else None
    if custom:
        filt.tofile(os.path.join(d, "filter.f32"))
    args = [exe, d] + _geom_args(case) + [str(batch)] + (["1"] if custom else [])
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    off = name == "offset"
    a = case.angles - case.angles.min()
    raw = np.fromfile(os.path.join(d, "fdk_raw.f32"), np.float32).reshape(case.nz, case.ny, case.nx)
    ref_raw = O.fdk(g, b.astype(np.float64), a, case.offsets, offset_corr=off, filt=filt)
    assert O.rel_l2(raw, ref_raw) < 1e-4
    x = np.fromfile(os.path.join(d, "fdk.f32"), np.float32).reshape(case.nz, case.ny, case.nx)
    ax = O.forward(g, ref_raw, a, case.offsets)
    ref = ref_raw * (np.vdot(ax, b.astype(np.float64)) / np.vdot(ax, ax))
    assert O.rel_l2(x, ref) < 1e-4


@pytest.mark.gpu
def test_binned_dropins_match_oracle(gtb, O, cuda, tmp_path):
    """cuConebeamProjectionOperatorB200 and CBSubsetOperatorB200 with two bins
    (4-D images): forward and back-projection per bin, the acquisition
    permuted into bin order, the subset operator's permutation and its binned
    OS-MOM solve."""
    case = make("cube")
    g = case.oracle_geom(O)
    P = case.angles.size
    S = 3
    vb = np.array([(v // 3) % 2 for v in range(P)], np.int32)
    exe = str(tmp_path / "bins_main")
    _compile(exe, "bins_main")
    vols = np.stack([O.phantom_voxelize(g, gtb.phantom.ellipsoids(60 + k, (case.lx, case.ly, case.lz), n=5)
                                        .astype(np.float64), ss=2) for k in range(2)])
    b = np.zeros((P, case.H, case.W))
    for k in range(2):
        idx = np.nonzero(vb == k)[0]
        b[idx] = O.forward(g, vols[k], case.angles[idx], case.offsets[idx])
    d = str(tmp_path)
    case.angles.astype(np.float32).tofile(os.path.join(d, "angles.f32"))
    case.offsets.astype(np.float32).tofile(os.path.join(d, "offsets.f32"))
    b.astype(np.float32).tofile(os.path.join(d, "b.f32"))
    vols.astype(np.float32).tofile(os.path.join(d, "x.f32"))
    vb.tofile(os.path.join(d, "view_bin.i32"))
    r = subprocess.run([exe, d] + _geom_args(case) + [str(S)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    x32 = vols.astype(np.float32).astype(np.float64)
    # 1. the device-array operator: projections in bin order
    order = np.concatenate([np.nonzero(vb == k)[0] for k in range(2)])
    ax = np.fromfile(os.path.join(d, "op_ax.f32"), np.float32).reshape(P, case.H, case.W)
    ref_ax = np.concatenate([O.forward(g, x32[k], case.angles[vb == k], case.offsets[vb == k]) for k in range(2)])
    assert O.rel_l2(ax, ref_ax) < 1e-4
    atax = np.fromfile(os.path.join(d, "op_atax.f32"), np.float32).reshape(2, case.nz, case.ny, case.nx)
    n0 = int((vb == 0).sum())
    for k, sl in enumerate((slice(0, n0), slice(n0, P))):
        ref = O.backproject(g, ax[sl].astype(np.float64), case.angles[order][sl], case.offsets[order][sl])
        assert O.rel_l2(atax[k], ref) < 1e-4
    perm = np.fromfile(os.path.join(d, "op_b_perm.f32"), np.float32).reshape(P, case.H, case.W)
    assert np.array_equal(perm, b.astype(np.float32)[order])
    # 2. the subset operator
    order2, sizes = O.subset_partition(P, S, vb)
    a2 = np.fromfile(os.path.join(d, "sub_angles.f32"), np.float32)
    assert np.array_equal(a2, (case.angles - case.angles.min())[order2])
    o2 = np.fromfile(os.path.join(d, "sub_offsets.f32"), np.float32).reshape(P, 2)
    ax0 = np.fromfile(os.path.join(d, "sub_ax0.f32"), np.float32).reshape(int(sizes[0]), case.H, case.W)
    v0 = order2[:sizes[0]]
    ref0 = np.stack([O.forward(g, x32[vb[v]], a2[i:i + 1], o2[i:i + 1])[0] for i, v in enumerate(v0)])
    assert O.rel_l2(ax0, ref0) < 1e-4
    z = np.fromfile(os.path.join(d, "sub_z.f32"), np.float32).reshape(2, case.nz, case.ny, case.nx)
    zr, _ = O.osmom(g, b[order2], a2, o2, sizes, np.zeros(S, np.int32), iters=2, nonneg=True,
                    view_bin=vb[order2], n_bins=2)
    assert O.rel_l2(z, zr) < 1e-4

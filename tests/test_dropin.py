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


def _compile(out_path):
    lib_dir = os.path.join(ROOT, "gt-tomography_b200", "_build")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wno-unused-function",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "gadgetron_stub"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"),
           "-o", out_path, "-L", lib_dir, "-lcbct", f"-Wl,-rpath,{lib_dir}",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_dropin_header_compiles(gtb, tmp_path):
    _compile(str(tmp_path / "dropin_main"))


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

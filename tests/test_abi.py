"""CPU checks of the C ABI: the library loads, exports every entry point that
include/cbct.h declares, and its pure-host helpers agree with the oracle.
No device work is issued here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from cases import make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header="cbct.h"):
    txt = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"CBCT_API\s+[\w\s\*]*?\b(cbct_\w+)\s*\(", txt)))


def test_header_symbols_exported(gtb):
    lib = gtb.lib()
    names = _declared()
    assert len(names) >= 27
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", gtb._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (cbct_\w+)", out))
    assert set(names) <= exported
    assert set(gtb._lib.EXPORTED) == set(names)
    plain = _declared("cbct_plain.h")
    assert set(plain) == set(gtb._lib.EXPORTED_PLAIN) and set(plain) <= exported


def test_status_strings(gtb):
    lib = gtb.lib()
    assert lib.cbct_status_string(0) == b"CBCT_OK"
    assert lib.cbct_status_string(1) == b"CBCT_ERR_INVALID_ARGUMENT"
    assert b"sm_100a" in lib.cbct_version()
    # the binding's status constants are the header's enum
    txt = open(os.path.join(ROOT, "include", "cbct.h")).read()
    enum = dict((k, int(v)) for k, v in re.findall(r"\b(CBCT_(?:OK|ERR_\w+))\s*=\s*(\d+)", txt))
    assert len(enum) == 10
    for k, v in enum.items():
        if k != "CBCT_OK":
            assert getattr(gtb._lib, k) == v, k
        assert lib.cbct_status_string(v) == k.encode()


def test_subset_partition_matches_oracle(gtb, O):
    for P, S in [(360, 10), (180, 7), (17, 4), (720, 10), (5, 8)]:
        o1, s1 = O.subset_partition(P, S)
        o2, s2 = gtb.subset_partition(P, S)
        assert np.array_equal(o1, o2) and np.array_equal(s1, s2)
    rng = np.random.default_rng(0)
    vb = rng.integers(-1, 4, 200).astype(np.int32)
    o1, s1 = O.subset_partition(200, 6, vb)
    o2, s2 = gtb.subset_partition(200, 6, vb)
    assert np.array_equal(o1, o2) and np.array_equal(s1, s2)
    # each subset is sorted by bin (CBSubsetOperator.cpp:86-87)
    first = np.concatenate([[0], np.cumsum(s2)[:-1]])
    for f, n in zip(first, s2):
        bins = vb[o2[f:f + n]]
        assert np.all(np.diff(bins) >= 0)


def test_default_filter_matches_oracle(gtb, O):
    for W in (48, 256, 512, 1024):
        assert np.allclose(gtb.default_frequency_filter(W), O.default_filter(W), rtol=2e-6, atol=1e-9)


def test_cosine_weights_match_oracle(gtb, O):
    case = make("offset")
    got = gtb.operators.cosine_weights(case.cgeom(gtb))
    assert np.array_equal(got.astype(np.float64), O.cosine_weights(case.oracle_geom(O)))


def test_short_scan_and_offset_override(gtb, O):
    case = make("cube")
    g = case.cgeom(gtb)
    assert not gtb.operators.is_short_scan(g, case.angles)
    short = np.linspace(0, 190, 50, dtype=np.float32)
    assert gtb.operators.is_short_scan(g, short) == O.is_short_scan(case.oracle_geom(O), short)
    assert gtb.operators.offset_override(g, np.tile([[8.0, 0.0]], (4, 1)))       # 8 > 0.1*72
    assert not gtb.operators.offset_override(g, np.tile([[7.0, 3.0]], (4, 1)))


def test_invalid_arguments_are_reported(gtb):
    lib = gtb.lib()
    L = gtb._lib
    bad = L.CbctGeometry(1000.0, 900.0, 10.0, 10.0, 8, 8, 8, 8, 8, 8.0, 8.0, 8.0, 1.5)   # SDD < SAD
    h = C.c_void_p()
    a = np.zeros(4, np.float32)
    o = np.zeros(8, np.float32)
    st = lib.cbct_plan_create(C.byref(bad), a.ctypes.data, o.ctypes.data, 4, None, 1, None, C.byref(h))
    assert st == 1 and b"SAD" in lib.cbct_last_error()
    good = L.CbctGeometry(1000.0, 1500.0, 10.0, 10.0, 8, 8, 8, 8, 8, 8.0, 8.0, 8.0, 1.5)
    sizes = np.array([3, 3], np.int32)   # sums to 6, not 4
    st = lib.cbct_plan_create(C.byref(good), a.ctypes.data, o.ctypes.data, 4, sizes.ctypes.data, 2, None, C.byref(h))
    assert st == 1
    with pytest.raises(gtb.CbctError):
        L.call("cbct_default_frequency_filter", 0, None)


def test_missing_library_fails_loudly(gtb, monkeypatch, tmp_path):
    """No CPU fallback: a missing libcbct.so is an error, not a silent path."""
    import importlib
    L = gtb._lib
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libcbct.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.lib()


_LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "cbct.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
#define S(T) printf(#T " %zu\n", sizeof(T));
int main(void) {
  S(cbct_geometry) S(cbct_solver_params) S(cbct_batch_item) S(cbct_server_config) S(cbct_request)
  S(cbct_request_info)
  F(cbct_solver_params, proj_storage) F(cbct_solver_params, reg_steps) F(cbct_batch_item, params)
  F(cbct_batch_item, resid_norm2_out)
  F(cbct_server_config, device) F(cbct_request, geometry) F(cbct_request, angles_deg)
  F(cbct_request, proj_host) F(cbct_request, params) F(cbct_request, filter) F(cbct_request, offset_correction)
  F(cbct_request_info, t_submit) F(cbct_request_info, bytes_peak) F(cbct_request_info, message)
  return 0;
}
"""


def test_struct_layouts_match_ctypes(gtb, tmp_path):
    """Every struct the ABI passes has the same size and field offsets in C
    (gcc on include/cbct.h) and in the ctypes binding."""
    src = tmp_path / "probe.c"
    src.write_text(_LAYOUT_PROBE)
    exe = tmp_path / "probe"
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, str(src), "-o",
                    str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    L = gtb._lib
    types = {"cbct_geometry": L.CbctGeometry, "cbct_solver_params": L.CbctSolverParams,
             "cbct_batch_item": L.CbctBatchItem, "cbct_server_config": L.CbctServerConfig,
             "cbct_request": L.CbctRequest, "cbct_request_info": L.CbctRequestInfo}
    for key, val in got.items():
        if "." in key:
            t, m = key.split(".")
            assert getattr(types[t], m).offset == int(val), key
        else:
            assert C.sizeof(types[key]) == int(val), key


def test_server_request_validation(gtb):
    """Host-side checks of the serving API: footprint estimate, rejected
    requests (no device work is issued)."""
    L = gtb._lib
    g = L.CbctGeometry(1000.0, 1500.0, 300.0, 225.0, 256, 192, 128, 128, 128, 128.0, 128.0, 128.0, 1.5)
    ang = np.arange(90, dtype=np.float32) * 4.0
    proj = np.zeros((90, 192, 256), np.float32)
    vol = np.zeros((128, 128, 128), np.float32)
    fdk = gtb.Server.fdk_request(g, ang, None, proj, vol)
    nb = gtb.Server.request_bytes(fdk)
    # projections + volume + FDK tables, no FP32 copy for float storage
    lower = 90 * 192 * 256 * 4 + 128 ** 3 * 4
    assert lower < nb < lower * 1.05
    mom = gtb.Server.osmom_request(g, ang, None, proj, vol, n_subsets=9)
    nm = gtb.Server.request_bytes(mom)
    assert nm > 2 * 90 * 192 * 256 * 4 + 4 * 128 ** 3 * 4
    half = gtb.Server.fdk_request(g, ang, None, proj.astype(np.float16), vol)
    assert gtb.Server.request_bytes(half) > nb  # 16-bit projections + an FP32 filtered copy
    with pytest.raises(gtb.CbctError, match="n_subsets"):
        gtb.Server.request_bytes(gtb.Server.osmom_request(g, ang, None, proj, vol, n_subsets=0))
    with pytest.raises(ValueError):
        gtb.Server.fdk_request(g, ang, None, proj[:10], vol)
    with pytest.raises(TypeError):
        gtb.Server.fdk_request(g, ang, None, proj, vol.astype(np.float16))

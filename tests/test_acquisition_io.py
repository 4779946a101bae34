"""Acquisition and binning files (xray/CBCT_acquisition.h:178-333,
xray/CBCT_binning.h:106-157, python/readReal.py:41-76) on the CPU: .real
round trips, the HDF5 layout written byte for byte as the format
specification lays it out, round trips of acquisitions and binnings, and the
reference's version checks and /spacing fallback."""
import struct

import numpy as np
import pytest


def _acq(gtb, P=7, H=5, W=6, seed=0):
    rng = np.random.default_rng(seed)
    geo = gtb.CBCT_geometry(1000.0, 1500.0, (76.8, 64.0), (np.arange(P) * 51.4).astype(np.float32),
                            rng.uniform(-9, 9, (P, 2)).astype(np.float32))
    return gtb.CBCT_acquisition(geo, rng.uniform(0, 3, (P, H, W)).astype(np.float32))


def test_real_round_trip(gtb, tmp_path):
    a = np.random.default_rng(1).standard_normal((3, 4, 5)).astype(np.float32)
    p = tmp_path / "a.real"
    gtb.save_real(a, p)
    raw = p.read_bytes()
    assert struct.unpack_from("<4I", raw, 0) == (3, 5, 4, 3)      # rank, then dims fastest first
    assert len(raw) == 16 + a.nbytes
    assert np.array_equal(gtb.read_real(p), a)
    c = (a + 1j * a).astype(np.complex64)
    gtb.save_real(c, p, dtype=np.complex64)
    assert np.array_equal(gtb.read_real(p), c)


def test_h5_layout(gtb, tmp_path):
    """Superblock version 0 and the root group's B-tree, symbol-table node and
    local heap where the superblock's root entry points."""
    io = gtb.acquisition_io
    p = tmp_path / "x.h5"
    io.write_h5(p, {"b": np.arange(3, dtype=np.uint32), "a": np.ones((2, 2), np.float32)})
    raw = p.read_bytes()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n"
    assert raw[8] == 0 and raw[13] == 8 and raw[14] == 8
    eof = struct.unpack_from("<Q", raw, 40)[0]
    assert eof == len(raw)
    _, root, cache, _ = struct.unpack_from("<QQII", raw, 56)
    tree, heap = struct.unpack_from("<QQ", raw, 80)
    assert cache == 1 and raw[tree:tree + 4] == b"TREE" and raw[heap:heap + 4] == b"HEAP"
    assert raw[root] == 1                                            # version-1 object header
    used = struct.unpack_from("<H", raw, tree + 6)[0]
    snod = struct.unpack_from("<Q", raw, tree + 32)[0]
    assert used == 1 and raw[snod:snod + 4] == b"SNOD"
    assert struct.unpack_from("<H", raw, snod + 6)[0] == 2
    d = io.read_h5(p)
    assert list(d) == ["a", "b"]                                     # sorted, as the group B-tree needs
    assert d["a"].dtype == np.float32 and d["b"].dtype == np.uint32
    assert np.array_equal(d["b"], np.arange(3)) and np.array_equal(d["a"], np.ones((2, 2)))


def test_h5_many_datasets_and_types(gtb, tmp_path):
    io = gtb.acquisition_io
    rng = np.random.default_rng(2)
    data = {f"d{i:03d}": rng.standard_normal(i + 1).astype([np.float32, np.float64, np.int32, np.uint16][i % 4])
            for i in range(70)}                                      # three symbol-table nodes
    data["be"] = np.arange(4, dtype=">f4")
    p = tmp_path / "m.h5"
    io.write_h5(p, data)
    d = io.read_h5(p)
    assert set(d) == set(data)
    for k, v in data.items():
        assert np.array_equal(d[k], v) and d[k].dtype == v.dtype.newbyteorder("=")


def test_acquisition_round_trip(gtb, tmp_path):
    acq = _acq(gtb)
    p = tmp_path / "acq.h5"
    acq.save(p)
    back = gtb.CBCT_acquisition.from_file(p)
    assert np.array_equal(back.projections, acq.projections)
    g, h = back.geometry, acq.geometry
    assert (g.SAD, g.SDD) == (h.SAD, h.SDD) and tuple(np.float32(g.FOV)) == tuple(np.float32(h.FOV))
    assert np.array_equal(g.angles, h.angles) and np.array_equal(g.offsets, h.offsets)
    d = gtb.acquisition_io.read_h5(p)
    assert d["projections"].shape == (7, 5, 6)                       # [P][H][W]
    assert int(d["geometry_dataformat_version"][0]) == 2 and int(d["projection_dataformat_version"][0]) == 1


def test_acquisition_version_checks_and_spacing(gtb, tmp_path):
    io = gtb.acquisition_io
    acq = _acq(gtb)
    base = {"projection_dataformat_version": np.array([1], np.uint32), "projections": acq.projections,
            "geometry_dataformat_version": np.array([2], np.uint32), "SAD": np.array([1000.0], np.float32),
            "SDD": np.array([1500.0], np.float32), "angles": acq.geometry.angles,
            "offsetx": acq.geometry.offsets[:, 0].copy(), "offsety": acq.geometry.offsets[:, 1].copy(),
            "spacing": np.array([0.5, 0.25], np.float32)}
    p = tmp_path / "s.h5"
    io.write_h5(p, base)
    back = gtb.CBCT_acquisition.from_file(p)
    assert back.geometry.FOV == (0.5 * 6, 0.25 * 5)                  # spacing x (W, H)
    io.write_h5(p, dict(base, geometry_dataformat_version=np.array([1], np.uint32)))
    with pytest.raises(RuntimeError, match="wrong geometry data version"):
        gtb.CBCT_acquisition.from_file(p)
    io.write_h5(p, dict(base, projection_dataformat_version=np.array([3], np.uint32)))
    with pytest.raises(RuntimeError, match="wrong projection data format version"):
        gtb.CBCT_acquisition.from_file(p)
    bad = dict(base)
    del bad["spacing"]
    io.write_h5(p, bad)
    with pytest.raises(RuntimeError, match="/FOV"):
        gtb.CBCT_acquisition.from_file(p)


def test_binning_round_trip(gtb, tmp_path):
    bins = [[0, 3, 6], [1, 4], [2, 5, 7, 8]]
    p = tmp_path / "bins.h5"
    b = gtb.CBCT_binning(bins)
    b.save(p)
    c = gtb.CBCT_binning()
    c.load(p)
    assert c.bins == bins
    d = gtb.acquisition_io.read_h5(p)
    assert int(d["numBins"][0]) == 3 and d["bin_2"].dtype == np.uint32
    gtb.acquisition_io.write_h5(p, {"binning_dataformat_version": np.array([2], np.uint32),
                                    "numBins": np.array([0], np.uint32)})
    with pytest.raises(RuntimeError, match="wrong format of binning file"):
        c.load(p)


@pytest.mark.gpu
def test_loaded_acquisition_reconstructs_identically(gtb, O, cuda, tmp_path):
    """An acquisition and binning written to HDF5 and read back reconstruct
    bitwise the same as the in-memory ones (FDK recipe; binned OS-MOM)."""
    import torch
    from cases import make
    case = make("offset")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(77, (case.lx, case.ly, case.lz), n=5).astype(np.float64)
    proj = O.phantom_project(g, ell, case.angles, case.offsets).astype(np.float32)
    geo = gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v), case.angles.copy(), case.offsets.copy())
    acq = gtb.CBCT_acquisition(geo, proj.copy())
    p = tmp_path / "acq.h5"
    acq.save(p)
    loaded = gtb.CBCT_acquisition.from_file(p)
    dims, mm = (case.nx, case.ny, case.nz), (case.lx, case.ly, case.lz)
    x_mem = gtb.fdk_reconstruct_3d(acq, dims, mm)
    x_file = gtb.fdk_reconstruct_3d(loaded, dims, mm)
    assert np.array_equal(x_mem, x_file)
    # binned OS-MOM through the subset operator
    P = case.angles.size
    bins = [[v for v in range(P) if (v // 3) % 2 == b] for b in range(2)]
    gtb.CBCT_binning(bins).save(tmp_path / "bins.h5")
    lb = gtb.CBCT_binning()
    lb.load(tmp_path / "bins.h5")
    outs = []
    for a, bn in ((gtb.CBCT_acquisition(gtb.CBCT_geometry(case.SAD, case.SDD, (case.fov_u, case.fov_v),
                                                          case.angles.copy(), case.offsets.copy()), proj.copy()),
                   gtb.CBCT_binning(bins)),
                  (gtb.CBCT_acquisition.from_file(p), lb)):
        op = gtb.CBSubsetOperator(3)
        op.setup(a, bn, mm, is_dims=dims)
        b = torch.from_numpy(np.ascontiguousarray(a.projections)).to(cuda)
        z = torch.empty(op.plan.vol_shape, dtype=torch.float32, device=cuda)
        op.plan.osmom(b, z, None, 2, nonneg=True)
        outs.append(z.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])

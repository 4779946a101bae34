"""Acquisition and binning files: the reference's on-disk formats, without libraries.

Two formats carry gt-tomography's data:

* ``.real`` arrays (python/readReal.py:41-76): a uint32 rank, the dimensions
  as uint32 fastest first, then float32 (or complex64) samples.
* HDF5 acquisition files (xray/CBCT_acquisition.h:178-333) with root-group
  datasets ``/projections`` [P][H][W] float, ``/angles``, ``/offsetx``,
  ``/offsety`` float [P], ``/SAD``, ``/SDD`` float [1], ``/FOV`` float [2]
  (or ``/spacing`` [2], then FOV = spacing x detector size),
  ``/geometry_dataformat_version`` = 2 and ``/projection_dataformat_version`` = 1
  (uint32 [1]); binning files (xray/CBCT_binning.h:106-157) with
  ``/binning_dataformat_version`` = 1, ``/numBins`` and ``/bin_1`` ..
  ``/bin_N`` (uint32 view indices).

The HDF5 library is not available here, so this module reads and writes the
subset of the HDF5 format (File Format Specification, version 0 and 1
superblocks) that such files use: one root group held as a symbol table
(a version-1 B-tree of symbol-table nodes over a local heap of names) and
datasets with version-1 object headers (dataspace, datatype, fill value and
data layout messages), contiguous or compact storage, fixed-point and IEEE
floating-point element types of either byte order.  Files are written the way
the library's defaults write them (version 0 superblock, 8-byte offsets and
lengths, contiguous layout), names sorted as its group B-tree requires.
"""
from __future__ import annotations

import struct
from typing import Dict, Optional

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


# ----------------------------------------------------------------- .real
def read_real(path) -> np.ndarray:
    """readReal (python/readReal.py:41-61): shape is the stored dimensions
    reversed (slowest first); complex64 when the payload is twice the size."""
    with open(path, "rb") as f:
        raw = f.read()
    nd = struct.unpack_from("<I", raw, 0)[0]
    dims = struct.unpack_from(f"<{nd}I", raw, 4)
    pos = 4 + 4 * nd
    n = int(np.prod(dims, dtype=np.int64)) if nd else 1
    payload = len(raw) - pos
    dtype = np.complex64 if payload > 4 * n else np.float32
    a = np.frombuffer(raw, dtype=dtype, count=n, offset=pos)
    return a.reshape(tuple(reversed(dims))).copy()


def save_real(a, path, dtype=np.float32) -> None:
    """saveReal (python/readReal.py:62-76)."""
    a = np.asarray(a)
    with open(path, "wb") as f:
        f.write(struct.pack("<I", a.ndim))
        f.write(struct.pack(f"<{a.ndim}I", *reversed(a.shape)))
        f.write(np.ascontiguousarray(a, dtype=dtype).tobytes())


# ----------------------------------------------------------------- HDF5 writer
def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


def _datatype_message(dt: np.dtype) -> bytes:
    dt = np.dtype(dt)
    order = 0 if dt.byteorder in ("<", "=", "|") else 1
    if dt.kind in "ui":
        bits = order | (0x08 if dt.kind == "i" else 0)
        head = bytes([0x10 | 0, bits, 0, 0]) + struct.pack("<I", dt.itemsize)
        return head + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f" and dt.itemsize in (4, 8):
        # mantissa normalisation 2 (implied msb), sign bit at the top
        sign = 8 * dt.itemsize - 1
        head = bytes([0x10 | 1, order | 0x20, sign, 0]) + struct.pack("<I", dt.itemsize)
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        else:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        return head + props
    raise TypeError(f"element type {dt} is not supported")


def _message(mtype: int, data: bytes) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), 0) + data


def _object_header(messages) -> bytes:
    body = b"".join(messages)
    return struct.pack("<BBHII", 1, 0, len(messages), 1, len(body)) + b"\0" * 4 + body


def write_h5(path, datasets: Dict[str, np.ndarray]) -> None:
    """Writes the arrays as datasets of the root group (version 0 superblock,
    symbol-table root group, contiguous version-1 datasets)."""
    names = sorted(datasets)
    for n in names:
        if not n or "/" in n:
            raise ValueError(f"dataset name {n!r} must be a plain root-group name")
    leaf_k, internal_k = 16, 16              # symbol-table node: 2*leaf_k entries
    per_node = 2 * leaf_k
    n_nodes = max(1, -(-len(names) // per_node))
    if n_nodes > 2 * internal_k:
        raise ValueError("too many datasets for one B-tree node")
    # local heap of names: the empty name at offset 0
    heap = bytearray(b"\0" * 8)
    name_off = {}
    for n in names:
        name_off[n] = len(heap)
        heap += _pad8(n.encode() + b"\0")
    out = bytearray(96)                      # superblock, filled in at the end

    def alloc(b: bytes) -> int:
        at = len(out)
        out.extend(b)
        out.extend(b"\0" * (-len(out) % 8))
        return at

    # raw data, then dataset object headers
    headers = {}
    for n in names:
        a = np.asarray(datasets[n])
        if a.dtype.byteorder == ">":
            a = a.astype(a.dtype.newbyteorder("<"))
        a = np.ascontiguousarray(a)
        shape = a.shape if a.ndim else (1,)
        data_at = alloc(a.tobytes())
        space = struct.pack("<BBB5x", 1, len(shape), 0) + b"".join(struct.pack("<Q", d) for d in shape)
        fill = bytes([2, 2, 2, 0])           # version 2: late allocation, fill if set, no fill value
        layout = struct.pack("<BBQQ", 3, 1, data_at, a.nbytes)
        headers[n] = alloc(_object_header([_message(0x0001, space), _message(0x0003, _datatype_message(a.dtype)),
                                           _message(0x0005, fill), _message(0x0008, layout)]))
    heap_data_at = alloc(bytes(heap))
    heap_at = alloc(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap), UNDEF, heap_data_at))

    def entry(n: str) -> bytes:
        return struct.pack("<QQII16x", name_off[n], headers[n], 0, 0)

    snods = []
    for k in range(n_nodes):
        chunk = names[k * per_node:(k + 1) * per_node]
        body = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk)) + b"".join(entry(n) for n in chunk)
        body += b"\0" * (8 + per_node * 40 - len(body))
        snods.append((alloc(body), chunk[-1]))
    # version-1 B-tree leaf (group node): key(0) = "", child(i), key(i+1) = last name of child i
    tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, n_nodes, UNDEF, UNDEF) + struct.pack("<Q", 0)
    for at, last in snods:
        tree += struct.pack("<QQ", at, name_off[last])
    tree += b"\0" * (24 + (2 * internal_k + 1) * 8 + 2 * internal_k * 8 - len(tree))
    tree_at = alloc(tree)
    root_at = alloc(_object_header([_message(0x0011, struct.pack("<QQ", tree_at, heap_at))]))
    sb = SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", leaf_k, internal_k, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(out), UNDEF)
    sb += struct.pack("<QQII", 0, root_at, 1, 0) + struct.pack("<QQ", tree_at, heap_at)
    assert len(sb) == 96
    out[:96] = sb
    with open(path, "wb") as f:
        f.write(bytes(out))


# ----------------------------------------------------------------- HDF5 reader
class _File:
    def __init__(self, raw: bytes):
        self.raw = raw
        at = raw.find(SIGNATURE)
        if at != 0:
            raise ValueError("not an HDF5 file (no superblock signature at offset 0)")
        ver = raw[8]
        if ver not in (0, 1):
            raise ValueError(f"HDF5 superblock version {ver} is not supported (versions 0 and 1 are)")
        self.so, self.sl = raw[13], raw[14]
        if self.so != 8 or self.sl != 8:
            raise ValueError("only 8-byte offsets and lengths are supported")
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", raw, 16)
        pos = 24 + (4 if ver == 1 else 0)
        self.base = struct.unpack_from("<Q", raw, pos)[0]
        pos += 32
        # root group symbol table entry
        _, self.root_header, cache, _ = struct.unpack_from("<QQII", raw, pos)
        self.root_scratch = struct.unpack_from("<QQ", raw, pos + 24) if cache == 1 else None

    def u(self, fmt, at):
        return struct.unpack_from("<" + fmt, self.raw, at)

    def addr(self, a):
        return self.base + a

    def sig(self, at, s):
        if self.raw[self.addr(at):self.addr(at) + 4] != s:
            raise ValueError(f"corrupt HDF5 file: expected {s!r} at {at}")

    # object headers (version 1, with continuation messages) -> [(type, data)]
    def messages(self, at):
        at = self.addr(at)
        ver = self.raw[at]
        if ver != 1:
            raise ValueError(f"HDF5 object header version {ver} is not supported")
        nmsg, _, size = self.u("HII", at + 2)
        blocks = [(at + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            p, n = blocks.pop(0)
            end = p + n
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize, _ = self.u("HHB", p)
                data = self.raw[p + 8:p + 8 + msize]
                if mtype == 0x0010:                  # continuation
                    off, ln = struct.unpack_from("<QQ", data, 0)
                    blocks.append((self.addr(off), ln))
                out.append((mtype, data))
                p += 8 + msize
        return out

    def heap_name(self, heap_at, off):
        self.sig(heap_at, b"HEAP")
        data_at = self.u("Q", self.addr(heap_at) + 24)[0]
        p = self.addr(data_at) + off
        e = self.raw.index(b"\0", p)
        return self.raw[p:e].decode()

    def group_entries(self, tree_at, heap_at):
        """name -> object header address, walking the group's version-1 B-tree."""
        self.sig(tree_at, b"TREE")
        p = self.addr(tree_at)
        ntype, level, used = self.u("BBH", p + 4)
        if ntype != 0:
            raise ValueError("corrupt HDF5 file: group B-tree of the wrong node type")
        out = {}
        q = p + 24 + 8                               # key(0)
        for i in range(used):
            child = self.u("Q", q)[0]
            q += 16                                  # child(i), key(i+1)
            if level > 0:
                out.update(self.group_entries(child, heap_at))
                continue
            self.sig(child, b"SNOD")
            c = self.addr(child)
            nsym = self.u("H", c + 6)[0]
            for k in range(nsym):
                e = c + 8 + 40 * k
                name_off, header = self.u("QQ", e)
                out[self.heap_name(heap_at, name_off)] = header
        return out

    def root(self):
        if self.root_scratch is not None:
            tree_at, heap_at = self.root_scratch
        else:
            st = [d for t, d in self.messages(self.root_header) if t == 0x0011]
            if not st:
                raise ValueError("root group is not a symbol-table group (not supported)")
            tree_at, heap_at = struct.unpack_from("<QQ", st[0], 0)
        return self.group_entries(tree_at, heap_at)

    def dataset(self, header):
        shape, dtype, layout = None, None, None
        for t, d in self.messages(header):
            if t == 0x0001:
                ver, nd = d[0], d[1]
                p = 8 if ver == 1 else 4
                shape = struct.unpack_from(f"<{nd}Q", d, p)
            elif t == 0x0003:
                dtype = _parse_datatype(d)
            elif t == 0x0008:
                layout = d
        if shape is None or dtype is None or layout is None:
            raise ValueError("dataset without dataspace, datatype or layout message")
        n = int(np.prod(shape, dtype=np.int64)) if len(shape) else 1
        ver = layout[0]
        if ver == 3:
            cls = layout[1]
            if cls == 1:
                at, size = struct.unpack_from("<QQ", layout, 2)
                if at == UNDEF:
                    raw = b"\0" * (n * dtype.itemsize)
                else:
                    raw = self.raw[self.addr(at):self.addr(at) + size]
            elif cls == 0:
                size = struct.unpack_from("<H", layout, 2)[0]
                raw = layout[4:4 + size]
            else:
                raise ValueError("chunked datasets are not supported")
        elif ver in (1, 2):
            nd, cls = layout[1], layout[2]
            if cls != 1:
                raise ValueError("only contiguous storage of version-1/2 layouts is supported")
            at = struct.unpack_from("<Q", layout, 8)[0]
            raw = self.raw[self.addr(at):self.addr(at) + n * dtype.itemsize]
        else:
            raise ValueError(f"layout message version {ver} is not supported")
        a = np.frombuffer(raw, dtype=dtype, count=n).reshape(shape if len(shape) else ())
        return a.astype(dtype.newbyteorder("="))


def _parse_datatype(d: bytes) -> np.dtype:
    cls = d[0] & 0x0F
    bits0 = d[1]
    size = struct.unpack_from("<I", d, 4)[0]
    order = ">" if (bits0 & 1) else "<"
    if cls == 0:
        signed = bool(bits0 & 0x08)
        return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
    if cls == 1 and size in (4, 8):
        return np.dtype(f"{order}f{size}")
    raise ValueError(f"HDF5 datatype class {cls} (size {size}) is not supported")


def read_h5(path) -> Dict[str, np.ndarray]:
    """Every dataset of the root group, by name (without the leading '/')."""
    with open(path, "rb") as f:
        F = _File(f.read())
    return {name: F.dataset(h) for name, h in F.root().items()}


# ----------------------------------------------------------------- acquisition and binning
def load_acquisition(path):
    """CBCT_acquisition::load (xray/CBCT_acquisition.h:178-303): returns
    (SAD, SDD, FOV (2,), angles (P,), offsets (P, 2), projections (P, H, W))."""
    d = read_h5(path)

    def need(name):
        if name not in d:
            raise RuntimeError(f"Error reading /{name} from file.")
        return d[name]

    gv = int(need("geometry_dataformat_version").reshape(-1)[0])
    if gv != 2:
        raise RuntimeError(f"wrong geometry data version inside hdf5 file, found: {gv}, needed: 2")
    angles = need("angles").astype(np.float32).reshape(-1)
    ox = need("offsetx").astype(np.float32).reshape(-1)
    oy = need("offsety").astype(np.float32).reshape(-1)
    if ox.size != oy.size:
        raise RuntimeError("CBCT_geometry::load : x/y offset arrays has different lengths")
    pv = int(need("projection_dataformat_version").reshape(-1)[0])
    if pv != 1:
        raise RuntimeError(f"wrong projection data format version inside hdf5 file, found: {pv}, needed: 1")
    proj = need("projections").astype(np.float32)
    SAD = float(need("SAD").reshape(-1)[0])
    SDD = float(need("SDD").reshape(-1)[0])
    if "FOV" in d:
        fov = d["FOV"].astype(np.float32).reshape(-1)[:2]
    elif "spacing" in d:
        # FOV = spacing x detector size (W, H), :286-291
        sp = d["spacing"].astype(np.float32).reshape(-1)
        fov = np.array([sp[0] * proj.shape[-1], sp[1] * proj.shape[-2]], np.float32)
    else:
        raise RuntimeError("Error reading /FOV from file.")
    return SAD, SDD, fov, angles, np.stack([ox, oy], axis=1), proj


def save_acquisition(path, SAD, SDD, fov, angles, offsets, projections) -> None:
    """CBCT_acquisition::save and CBCT_geometry::save (xray/CBCT_acquisition.h:76-107, :305-322)."""
    off = np.asarray(offsets, np.float32).reshape(-1, 2)
    write_h5(path, {
        "projection_dataformat_version": np.array([1], np.uint32),
        "projections": np.ascontiguousarray(projections, np.float32),
        "geometry_dataformat_version": np.array([2], np.uint32),
        "SAD": np.array([SAD], np.float32),
        "SDD": np.array([SDD], np.float32),
        "FOV": np.asarray(fov, np.float32).reshape(2),
        "angles": np.asarray(angles, np.float32).reshape(-1),
        "offsetx": np.ascontiguousarray(off[:, 0]),
        "offsety": np.ascontiguousarray(off[:, 1]),
    })


def load_binning(path):
    """CBCT_binning::load (xray/CBCT_binning.h:106-148): list of bins, each a
    list of view indices."""
    d = read_h5(path)
    if "binning_dataformat_version" not in d:
        raise RuntimeError("Error reading /binning_dataformat_version")
    v = int(d["binning_dataformat_version"].reshape(-1)[0])
    if v != 1:
        raise RuntimeError(f"wrong format of binning file, found: {v}, needed: 1")
    if "numBins" not in d:
        raise RuntimeError("Error reading /numBins_dataformat_version")
    n = int(d["numBins"].reshape(-1)[0])
    bins = []
    for i in range(1, n + 1):
        key = f"bin_{i}"
        if key not in d:
            raise RuntimeError("Error reading bin info")
        bins.append([int(x) for x in d[key].reshape(-1)])
    return bins


def save_binning(path, bins) -> None:
    """The layout CBCT_binning::load reads (no save in the reference)."""
    data = {"binning_dataformat_version": np.array([1], np.uint32),
            "numBins": np.array([len(bins)], np.uint32)}
    for i, b in enumerate(bins, 1):
        data[f"bin_{i}"] = np.asarray(b, np.uint32)
    write_h5(path, data)

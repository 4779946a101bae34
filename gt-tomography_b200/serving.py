"""Serving loop: continuous batching of FDK and OS-MOM reconstructions.

A thin view of the cbct_server_* entry points (include/cbct.h).  The server
runs `max_inflight` request slots on one GPU; requests are admitted while a
slot is idle and their device footprint fits into the HBM budget, their
set-up, copies and kernels overlap on the device, and each result is bitwise
identical to the same request served alone.  Requests read their projections
from host memory (pinned memory gives asynchronous copies) and write the
volume to host memory; both arrays must stay alive until `wait` returns,
which this class guarantees by holding references until then.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .operators import _dtype_code, torch


def _host_ptr(t, shape, what, dtype=None):
    T = torch()
    if isinstance(t, np.ndarray):
        if not t.flags["C_CONTIGUOUS"]:
            raise ValueError(f"{what} must be contiguous")
        code = {np.dtype(np.float32): L.CBCT_F32, np.dtype(np.float16): L.CBCT_F16}.get(t.dtype)
        ptr = t.ctypes.data
    elif isinstance(t, T.Tensor):
        if t.is_cuda:
            raise TypeError(f"{what} must be in host memory")
        if not t.is_contiguous():
            raise ValueError(f"{what} must be contiguous")
        code = _dtype_code(t.dtype)
        ptr = t.data_ptr()
    else:
        raise TypeError(f"{what} must be a numpy array or a CPU torch tensor")
    if code is None:
        raise TypeError(f"{what} has an unsupported dtype {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if dtype is not None and code != dtype:
        raise TypeError(f"{what} must be float32")
    return ptr, code


class Server:
    """cbct_server: request slots, a stream-ordered memory pool and admission
    by HBM budget on one device."""

    def __init__(self, hbm_budget_bytes: float = 150e9, max_inflight: int = 4, device: int = 0):
        cfg = L.CbctServerConfig(int(hbm_budget_bytes), int(max_inflight), int(device))
        h = C.c_void_p()
        L.call("cbct_server_create", C.byref(cfg), C.byref(h))
        self._h = h
        self._keep = {}

    def close(self):
        """Serves what is queued, then releases the slots and the pool."""
        if self._h:
            L.call("cbct_server_destroy", self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _request(kind, g, angles, offsets, proj_host, vol_host, n_subsets, params, filt, fdk_flags,
                 offset_correction):
        a = np.ascontiguousarray(angles, np.float32)
        P = a.size
        o = None if offsets is None else np.ascontiguousarray(offsets, np.float32).reshape(P, 2)
        pptr, code = _host_ptr(proj_host, (P, g.height, g.width), "projections")
        vptr, _ = _host_ptr(vol_host, (g.nz, g.ny, g.nx), "volume", dtype=L.CBCT_F32)
        f = None if filt is None else np.ascontiguousarray(filt, np.float32)
        if f is not None and f.size != g.width + 1:
            raise ValueError("filter must have W+1 entries")
        req = L.CbctRequest(kind, g, a.ctypes.data, None if o is None else o.ctypes.data, P, int(n_subsets), code,
                            pptr, vptr, params, None if f is None else f.ctypes.data, int(fdk_flags),
                            int(offset_correction))
        return req, (a, o, f, proj_host, vol_host)

    @staticmethod
    def fdk_request(g, angles, offsets, proj_host, vol_host, filt=None, fdk_flags=0, offset_correction=-1):
        """A FDK request (hoCuConebeamProjectionOperator::mult_MH with FBP).
        proj_host: (P, H, W) float32/float16/bfloat16 host array in acquisition
        order; its dtype is the device storage type."""
        return Server._request(L.CBCT_REQ_FDK, g, angles, offsets, proj_host, vol_host, 1, L.CbctSolverParams(),
                               filt, fdk_flags, offset_correction)

    @staticmethod
    def osmom_request(g, angles, offsets, proj_host, vol_host, n_subsets, iterations=10, beta=1.0, gamma=0.0,
                      nonneg=True, use_graph=False, refine_every=0, offset_correction=-1):
        """An OS-MOM request (CBSubsetOperator::setup + osMOMSolverD::solve)."""
        prm = L.CbctSolverParams(int(iterations), float(beta), float(gamma), int(nonneg), int(use_graph), 0,
                                 int(refine_every), 0)
        return Server._request(L.CBCT_REQ_OSMOM, g, angles, offsets, proj_host, vol_host, n_subsets, prm, None, 0,
                               offset_correction)

    @staticmethod
    def request_bytes(request) -> int:
        req, _ = request
        n = C.c_size_t()
        L.call("cbct_server_request_bytes", C.byref(req), C.byref(n))
        return int(n.value)

    def submit(self, request) -> int:
        """Queues a request made by fdk_request / osmom_request; returns its ticket."""
        req, keep = request
        t = C.c_uint64()
        L.call("cbct_server_submit", self._h, C.byref(req), C.byref(t))
        self._keep[int(t.value)] = keep
        return int(t.value)

    def wait(self, ticket: int, timeout: float | None = None, check: bool = True) -> dict:
        """Waits for a request; returns its record (times on the server clock).
        Raises TimeoutError if it has not completed within `timeout` seconds
        and, with check, CbctError if the request itself failed."""
        info = L.CbctRequestInfo()
        st = L.lib().cbct_server_wait(self._h, C.c_uint64(ticket), -1.0 if timeout is None else float(timeout),
                                      C.byref(info))
        if st == 6:  # CBCT_ERR_TIMEOUT
            raise TimeoutError(f"request {ticket} has not completed")
        L.check(st, "cbct_server_wait")
        self._keep.pop(ticket, None)
        rec = dict(ticket=ticket, status=int(info.status), slot=int(info.slot), t_submit=info.t_submit,
                   t_admit=info.t_admit, t_done=info.t_done, bytes_reserved=int(info.bytes_reserved),
                   bytes_peak=int(info.bytes_peak), message=info.message.decode())
        if check and rec["status"] != 0:
            raise L.CbctError(rec["status"], f"request {ticket}", rec["message"])
        return rec

    def now(self) -> float:
        t = C.c_double()
        L.call("cbct_server_now", self._h, C.byref(t))
        return float(t.value)

"""Shared geometries of the parity tests (small enough for the FP64 oracle)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    W: int
    H: int
    fov_u: float
    fov_v: float
    SAD: float
    SDD: float
    angles: np.ndarray
    offsets: np.ndarray
    spp: float = 1.5

    def oracle_geom(self, O):
        return O.Geometry(self.nx, self.ny, self.nz, self.lx, self.ly, self.lz, self.W, self.H,
                          self.fov_u, self.fov_v, self.SAD, self.SDD)

    def cgeom(self, gtb):
        return gtb._lib.CbctGeometry(self.SAD, self.SDD, self.fov_u, self.fov_v, self.W, self.H, self.nx,
                                     self.ny, self.nz, self.lx, self.ly, self.lz, self.spp)


def _ang(n, span=360.0, start=0.0):
    return (start + np.arange(n) * (span / n)).astype(np.float32)


def make(name: str) -> Case:
    if name == "cube":          # centred detector, full scan
        return Case(name, 32, 32, 32, 32.0, 32.0, 32.0, 48, 40, 72.0, 60.0, 1000.0, 1500.0,
                    _ang(12), np.zeros((12, 2), np.float32))
    if name == "aniso":         # anisotropic voxels, odd sizes, rays missing the box, odd angles
        a = np.array([0, 17, 44.9, 45, 45.1, 90, 133, 181, 225, 270.5, 300, 359], np.float32)
        return Case(name, 28, 36, 20, 33.6, 36.0, 30.0, 44, 30, 110.0, 60.0, 800.0, 1300.0,
                    a, np.zeros((a.size, 2), np.float32))
    if name == "offset":        # half-fan offset detector with a vertical shift
        a = _ang(16)
        o = np.tile(np.array([[14.0, 1.5]], np.float32), (16, 1))
        return Case(name, 32, 32, 24, 40.0, 40.0, 30.0, 40, 24, 64.0, 38.4, 1000.0, 1500.0, a, o)
    if name == "odd":           # nx not a multiple of 4: gather fallback for fp32 TMA pitch
        return Case(name, 30, 26, 18, 30.0, 26.0, 18.0, 36, 28, 60.0, 46.0, 700.0, 1100.0,
                    _ang(10, 200.0, 7.0), np.zeros((10, 2), np.float32))
    if name == "short":         # short volume under a tall detector: most rows leave through top/bottom
        return Case(name, 40, 48, 12, 40.0, 48.0, 12.0, 64, 48, 96.0, 96.0, 600.0, 1000.0,
                    _ang(14, 360.0, 3.0), np.zeros((14, 2), np.float32))
    if name == "c1small":       # config 1 geometry scaled down (128^3 -> 64^3, 180 -> 45 views)
        return Case(name, 64, 64, 64, 64.0, 64.0, 64.0, 128, 96, 192.0, 144.0, 1000.0, 1500.0,
                    _ang(45), np.zeros((45, 2), np.float32))
    raise KeyError(name)


ALL = ["cube", "aniso", "offset", "odd", "short"]

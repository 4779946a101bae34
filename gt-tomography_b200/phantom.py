"""Seeded synthetic phantoms and acquisitions for the benchmarks and tests.

Ellipsoid records are 10 floats: cx cy cz ax ay az phi theta psi density
(mm, radians, 1/mm).  Parameters are drawn from numpy's PCG64 generator with
a recorded seed:
  centres uniform in +-0.35 L, semi-axes uniform in [0.05, 0.35] L, Euler
  angles uniform in [0, pi), densities uniform in [0, 0.05] 1/mm;
  optional small spheres (radius 0.5..2 mm, density up to 0.5 1/mm) placed
  inside +-0.4 L.
Voxelisation and exact line integrals run on the device (libcbct.so).
"""
from __future__ import annotations

import numpy as np


def ellipsoids(seed: int, lengths_mm, n: int = 10, n_spheres: int = 0, density_max: float = 0.05,
               sphere_density_max: float = 0.5) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    Lv = np.asarray(lengths_mm, np.float64)
    e = np.zeros((n + n_spheres, 10), np.float64)
    e[:n, 0:3] = rng.uniform(-0.35, 0.35, (n, 3)) * Lv
    e[:n, 3:6] = rng.uniform(0.05, 0.35, (n, 3)) * Lv
    e[:n, 6:9] = rng.uniform(0.0, np.pi, (n, 3))
    e[:n, 9] = rng.uniform(0.0, density_max, n)
    if n_spheres:
        r = rng.uniform(0.5, 2.0, n_spheres)
        e[n:, 0:3] = rng.uniform(-0.4, 0.4, (n_spheres, 3)) * Lv
        e[n:, 3:6] = r[:, None]
        e[n:, 9] = rng.uniform(0.0, sphere_density_max, n_spheres)
    return e.astype(np.float32)


def circular_orbit(n_views: int, span_deg: float = 360.0, start_deg: float = 0.0) -> np.ndarray:
    """Angles start + i*span/n (CBCT_forwards_projection.cpp:167-172 uses start + i*spacing)."""
    return (start_deg + np.arange(n_views, dtype=np.float64) * (span_deg / n_views)).astype(np.float32)


def poisson_log(line_integrals, I0: float, seed: int):
    """counts ~ Poisson(I0 exp(-p)), p = -ln(max(counts,1)/I0), on the device (torch RNG seeded)."""
    import torch
    gen = torch.Generator(device=line_integrals.device)
    gen.manual_seed(int(seed))
    lam = I0 * torch.exp(-line_integrals.double())
    counts = torch.poisson(lam, generator=gen)
    return (-torch.log(torch.clamp(counts, min=1.0) / I0)).float()


def uneven_scans(n: int = 64, seed0: int = 1000, vol_range=(96, 320), z_range=(64, 320), view_range=(90, 720),
                 width_range=(256, 768), step: int = 8):
    """Scan shapes of the batched workload: volume x/y uniform in vol_range, z in
    z_range, views in view_range, detector width in width_range with a 4:3
    aspect; 1 mm voxels; pixel pitch 1.2*1.5*max(nx,ny)/W mm so that the
    detector covers the volume.  Sizes are multiples of `step` (8), as CT grids
    and detectors usually are.  Scan i uses seed seed0 + i."""
    out = []
    for i in range(n):
        rng = np.random.Generator(np.random.PCG64(seed0 + i))
        q = lambda lo, hi: int(rng.integers(lo // step, hi // step + 1)) * step
        nx, ny, nz = q(*vol_range), q(*vol_range), q(*z_range)
        P = int(rng.integers(view_range[0], view_range[1] + 1))
        W = q(*width_range)
        H = (3 * W) // 4
        pitch = 1.2 * 1.5 * max(nx, ny) / W
        out.append(dict(seed=seed0 + i, n=(nx, ny, nz), P=P, W=W, H=H, pitch=pitch))
    return out


def make_osmom_scan(spec: dict, subsets: int, I0: float, device, offset_mm: float = 0.0, SAD: float = 1000.0,
                    SDD: float = 1500.0, n_ellipsoids: int = 10):
    """Device-resident OS-MOM problem for one scan shape (from uneven_scans):
    views over 360 degrees in subset order, a seeded ellipsoid phantom, its exact
    line integrals with Poisson noise (I0 > 0) and the log transform.
    Returns (plan, b, (angles, offsets, subset_sizes, offset_correction))."""
    import torch
    from . import _lib as L
    from .operators import Plan, offset_override, subset_partition
    nx, ny, nz = spec["n"]
    P, W, H, pitch = spec["P"], spec["W"], spec["H"], spec["pitch"]
    lengths = (float(nx), float(ny), float(nz))
    g = L.CbctGeometry(SAD, SDD, W * pitch, H * pitch, W, H, nx, ny, nz, *lengths, 1.5)
    ang = circular_orbit(P)
    off = np.tile(np.array([[offset_mm, 0.0]], np.float32), (P, 1))
    order, sizes = subset_partition(P, subsets)
    a, o = ang[order] - ang.min(), off[order]
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    oc = [int(offset_override(g, o[f:f + n])) if n else 0 for f, n in zip(first, sizes)]
    plan = Plan(g, a, o, sizes, oc)
    ell = torch.from_numpy(ellipsoids(spec["seed"], lengths, n=n_ellipsoids).reshape(-1)).to(device)
    exact = torch.empty(plan.proj_shape(), dtype=torch.float32, device=device)
    plan.phantom_project(ell, exact)
    b = poisson_log(exact, I0, spec["seed"] + 1) if I0 else exact
    return plan, b.contiguous(), (a, o, sizes, oc)

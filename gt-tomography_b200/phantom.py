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

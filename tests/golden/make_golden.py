"""Generates tests/golden/oracle_small.npz: seeded inputs and FP64 oracle
outputs of the hot path on a tiny geometry.

The reference ships no golden vectors and cannot run here, so these fixtures
pin the oracle against regressions (tests/test_golden.py) and give the GPU
path committed vectors to match.  Regenerate with:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

GEOM = dict(nx=24, ny=20, nz=16, lx=24.0, ly=20.0, lz=16.0, W=32, H=24, fov_u=48.0, fov_v=36.0,
            SAD=600.0, SDD=900.0)


def make():
    g = O.Geometry(**GEOM)
    rng = np.random.default_rng(20261203)
    P = 8
    angles = np.sort(rng.uniform(0, 360, P)).astype(np.float32)
    offsets = np.stack([np.full(P, 6.0), rng.uniform(-1, 1, P)], 1).astype(np.float32)
    vol = rng.uniform(0, 0.05, (g.nz, g.ny, g.nx)).astype(np.float32)
    proj = rng.uniform(0, 1, (P, g.H, g.W)).astype(np.float32)
    filt = O.default_filter(g.W)
    order, sizes = O.subset_partition(P, 3)
    oc = np.ones(3, np.int32)
    b = O.forward(g, vol.astype(np.float64), angles[order], offsets[order]).astype(np.float32)
    out = dict(
        angles=angles, offsets=offsets, vol=vol, proj=proj,
        forward=O.forward(g, vol.astype(np.float64), angles, offsets),
        backproject=O.backproject(g, proj.astype(np.float64), angles, offsets),
        backproject_fdk=O.backproject(g, proj.astype(np.float64), angles, offsets, fbp=True),
        offset_full=O.offset_weight(g, proj, offsets, 0),
        offset_sqrt=O.offset_weight(g, proj, offsets, 1),
        filter=filt,
        filter_rows=O.fdk_filter_rows(proj, filt),
        fdk=O.fdk(g, proj, angles, offsets, offset_corr=True),
        order=order, sizes=sizes, b=b,
        osmom=O.osmom(g, b.astype(np.float64), angles[order], offsets[order], sizes, oc, iters=2,
                      nonneg=True)[0],
        ossart=O.ossart(g, b.astype(np.float64), angles[order], offsets[order], sizes, oc, iters=2,
                        nonneg=True)[0],
        spacecarver=O.spacecarver(g, proj, angles, offsets, 0.3),
    )
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **out)


if __name__ == "__main__":
    make()
    print("wrote", os.path.join(HERE, "oracle_small.npz"))

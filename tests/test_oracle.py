"""CPU checks of the oracle (oracle/cbct_oracle.cpp).

The reference cannot be built or run here and ships no golden vectors, so the
oracle is checked against (1) a second, independent pure-Python/numpy
restatement of each reference formula on small cases, and (2) closed-form
known answers (exact ellipsoid line integrals, redundancy-weight identities,
FDK reconstruction of a phantom)."""
import math

import numpy as np
import pytest

from cases import make


# ------------------------------------------------------------ pure-Python restatements
def _tex3(vol, c):
    """tex3D with normalised coords already converted to texel coords c (x,y,z), border 0."""
    nz, ny, nx = vol.shape
    f = [math.floor(v) for v in c]
    a = [c[i] - f[i] for i in range(3)]
    s = 0.0
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                x, y, z = f[0] + dx, f[1] + dy, f[2] + dz
                if 0 <= x < nx and 0 <= y < ny and 0 <= z < nz:
                    w = (a[0] if dx else 1 - a[0]) * (a[1] if dy else 1 - a[1]) * (a[2] if dz else 1 - a[2])
                    s += w * vol[z, y, x]
    return s


def _ray_py(case, vol, p, u, v):
    """conebeam_forwards_projection_kernel (conebeam_projection.cu:429-527) for one ray."""
    th = float(case.angles[p]) * math.pi / 180.0
    c, s = math.cos(th), math.sin(th)
    S = (case.SAD * s, -case.SAD * c, 0.0)
    q = ((u + 0.5) / case.W - 0.5) * case.fov_u + float(case.offsets[p, 0])
    r = ((v + 0.5) / case.H - 0.5) * case.fov_v + float(case.offsets[p, 1])
    add = case.SDD - case.SAD
    E = (c * q - s * add, s * q + c * add, r)
    d = [E[i] - S[i] for i in range(3)]
    L = (case.lx, case.ly, case.lz)
    lo, hi = [], []
    for i in range(3):
        t1 = (L[i] / 2 - S[i]) / d[i] if d[i] != 0 else math.copysign(math.inf, L[i] / 2 - S[i])
        t2 = (-L[i] / 2 - S[i]) / d[i] if d[i] != 0 else math.copysign(math.inf, -L[i] / 2 - S[i])
        lo.append(min(t1, t2))
        hi.append(max(t1, t2))
    a1, a2 = max(max(lo), 0.0), min(min(hi), 1.0)
    N = int(np.float32(case.spp) * np.float32(case.nx))
    delta = math.sqrt(sum(((a2 - a1) * d[i]) ** 2 for i in range(3))) / N
    n = (case.nx, case.ny, case.nz)
    acc = 0.0
    for k in range(N):
        P = [((S[i] + a1 * d[i]) / L[i] + 0.5) + d[i] / L[i] * ((a2 - a1) / N) * k for i in range(3)]
        acc += _tex3(vol, [P[i] * n[i] - 0.5 for i in range(3)])
    return acc * delta


def _voxel_py(case, proj, i, j, k, fbp):
    """conebeam_backwards_projection_kernel (conebeam_projection.cu:938-1036) for one voxel."""
    x = ((i + 0.5) / case.nx - 0.5) * case.lx
    y = ((j + 0.5) / case.ny - 0.5) * case.ly
    z = ((k + 0.5) / case.nz - 0.5) * case.lz
    acc = 0.0
    for p in range(case.angles.size):
        th = float(case.angles[p]) * math.pi / 180.0
        c, s = math.cos(-th), math.sin(-th)
        pr = (c * x - s * y, s * x + c * y, z)
        d = (pr[0], pr[1] + case.SAD, pr[2])
        d = (d[0] / d[1], 1.0, d[2] / d[1])
        e = (case.SDD * d[0] - float(case.offsets[p, 0]), case.SDD * d[2] - float(case.offsets[p, 1]))
        uv = (e[0] / case.fov_u + 0.5, e[1] / case.fov_v + 0.5)
        cu, cv = uv[0] * case.W - 0.5, uv[1] * case.H - 0.5
        fu, fv = math.floor(cu), math.floor(cv)
        au, av = cu - fu, cv - fv
        smp = 0.0
        for dv in (0, 1):
            for du in (0, 1):
                uu, vv = fu + du, fv + dv
                if 0 <= uu < case.W and 0 <= vv < case.H:
                    smp += (au if du else 1 - au) * (av if dv else 1 - av) * proj[p, vv, uu]
        w = 1.0
        if fbp:
            r, phi = math.hypot(x, y), math.atan2(y, x)
            U = (case.SAD + r * math.sin(th - phi)) / case.SAD
            w = 1.0 / (U * U)
        acc += w * smp
    return acc


@pytest.mark.parametrize("name", ["cube", "aniso", "offset"])
def test_forward_oracle_vs_python(O, name):
    case = make(name)
    rng = np.random.default_rng(0)
    vol = rng.uniform(0, 1, (case.nz, case.ny, case.nx))
    out = O.forward(case.oracle_geom(O), vol, case.angles, case.offsets, spp=case.spp)
    for p, v, u in [(0, 0, 0), (1, case.H // 2, case.W // 2), (case.angles.size - 1, case.H - 1, 3),
                    (3, 5, case.W - 1), (2, case.H // 3, case.W // 4)]:
        ref = _ray_py(case, vol, p, u, v)
        assert abs(out[p, v, u] - ref) <= 1e-10 * max(1.0, abs(ref)), (p, v, u)


@pytest.mark.parametrize("fbp", [False, True])
def test_backproject_oracle_vs_python(O, fbp):
    case = make("offset")
    rng = np.random.default_rng(1)
    proj = rng.uniform(0, 1, (case.angles.size, case.H, case.W))
    out = O.backproject(case.oracle_geom(O), proj, case.angles, case.offsets, fbp=fbp)
    for i, j, k in [(0, 0, 0), (16, 16, 12), (31, 5, 23), (7, 30, 1)]:
        ref = _voxel_py(case, proj, i, j, k, fbp)
        assert abs(out[k, j, i] - ref) <= 1e-10 * max(1.0, abs(ref))


def test_fdk_filter_oracle_vs_numpy_fft(O):
    """pad to 2W (centred), rfft, multiply W+1 bins, irfft (/2W), crop."""
    W = 48
    rng = np.random.default_rng(2)
    rows = rng.normal(0, 1, (7, W))
    filt = O.default_filter(W)
    pad = np.zeros((7, 2 * W))
    pad[:, W // 2:W // 2 + W] = rows
    ref = np.fft.irfft(np.fft.rfft(pad, axis=1) * filt[None], n=2 * W, axis=1)[:, W // 2:W // 2 + W]
    got = O.fdk_filter_rows(rows, filt)
    assert np.max(np.abs(got - ref)) < 1e-12


def test_fdk_filter_non_power_of_two(O):
    W = 30  # 2W = 60 exercises the Bluestein path
    rng = np.random.default_rng(3)
    rows = rng.normal(0, 1, (3, W))
    filt = O.default_filter(W)
    pad = np.zeros((3, 2 * W))
    pad[:, W // 2:W // 2 + W] = rows
    ref = np.fft.irfft(np.fft.rfft(pad, axis=1) * filt[None], n=2 * W, axis=1)[:, W // 2:W // 2 + W]
    assert np.max(np.abs(O.fdk_filter_rows(rows, filt) - ref)) < 1e-11


def test_default_filter_formula(O):
    """hoCuConebeamProjectionOperator.cpp:41-61 evaluated in float32."""
    for W in (64, 256, 511):
        K = W + 1
        A2 = np.float32(0.2 * K * K)
        k = np.arange(K, dtype=np.float32)
        with np.errstate(all="ignore"):
            h = np.where(k * k < A2, k * A2 / (A2 - k * k) * np.exp(-A2 / (A2 - k * k)), np.float32(0))
        h = h.astype(np.float64) * (K / np.abs(h.astype(np.float64)).sum())
        got = O.default_filter(W)
        assert np.allclose(got, h, rtol=1e-6, atol=1e-9)
        assert abs(got.sum() - K) < 1e-6 * K


def test_cosine_weights_formula(O):
    case = make("offset")
    g = case.oracle_geom(O)
    w = O.cosine_weights(g)
    x = np.arange(case.W) / case.W - 0.5
    y = np.arange(case.H) / case.H - 0.5
    s = case.SAD * (x * case.fov_u) / case.SDD
    v = case.SAD * (y * case.fov_v) / case.SDD
    ref = (case.SAD / np.sqrt(case.SAD ** 2 + s[None] ** 2 + v[:, None] ** 2)).astype(np.float32)
    assert np.array_equal(w, ref.astype(np.float64))


def test_offset_weight_redundancy(O):
    """Wang weights: sin^2 at mirrored positions sum to 1 (a known identity)."""
    case = make("offset")
    g = case.oracle_geom(O)
    o = float(case.offsets[0, 0])
    ones = np.ones((1, case.H, case.W))
    w = O.offset_weight(g, ones, case.offsets[:1], 0)[0, 0]
    t = case.fov_u * (np.arange(case.W) / case.W - 0.5) + o
    om = case.fov_u / 2 - abs(o)
    for u in range(case.W):
        if abs(t[u]) <= om:
            ref = math.sin(math.pi * (t[u] + om) / (4 * om)) ** 2
            mirrored = math.sin(math.pi * (-t[u] + om) / (4 * om)) ** 2
            assert abs(w[u] - ref) < 1e-12 and abs(ref + mirrored - 1) < 1e-12
        elif t[u] < -om:
            assert w[u] == 0
        else:
            assert w[u] == 1
    # zero offset: no weight at all (t is NaN in the reference)
    z = O.offset_weight(g, ones, np.zeros((1, 2), np.float32), 0)
    assert np.array_equal(z, ones)


def test_parker_weights_redundancy(O):
    """Known answer: with conjugate rays weighted to sum to 1, every detector
    column's weights integrate to pi over a short scan of pi + 2 delta."""
    case = make("cube")
    case.H = 1
    g = case.oracle_geom(O)
    delta = math.atan(case.fov_u / (2 * case.SDD))
    span = math.pi + 2 * delta
    n = 4000
    ang = (np.arange(n) * (span / n) * 180.0 / math.pi).astype(np.float32)
    assert O.is_short_scan(g, ang)
    w = O.parker_weight(g, np.ones((n, 1, case.W)), ang)[:, 0, :]
    assert np.all(w >= -1e-12) and np.all(w <= 1 + 1e-12)
    integral = w.sum(axis=0) * (span / n)
    assert np.allclose(integral, math.pi, rtol=2e-2), integral
    assert not O.is_short_scan(g, np.linspace(0, 359, 60, dtype=np.float32))


def test_subset_partition_round_robin(O):
    order, sizes = O.subset_partition(360, 10)
    assert sizes.tolist() == [36] * 10
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    for s in range(10):
        sub = order[first[s]:first[s] + sizes[s]]
        assert sorted(sub.tolist()) == list(range(s, 360, 10))
    # views outside every bin are skipped; round-robin counts only binned views
    vb = np.zeros(10, np.int32)
    vb[[2, 5]] = -1
    order, sizes = O.subset_partition(10, 3, vb)
    assert sorted(order.tolist()) == [0, 1, 3, 4, 6, 7, 8, 9]
    assert sizes.tolist() == [3, 3, 2]


def test_forward_analytic_known_answer(O):
    """Exact chord integrals of the box-truncated phantom vs the discrete projector."""
    case = make("c1small")
    case.angles = case.angles[:8]
    case.offsets = case.offsets[:8]
    rng = np.random.default_rng(4)
    ell = np.zeros((4, 10))
    ell[:, 0:3] = rng.uniform(-12, 12, (4, 3))
    ell[:, 3:6] = rng.uniform(6, 18, (4, 3))
    ell[:, 6:9] = rng.uniform(0, np.pi, (4, 3))
    ell[:, 9] = rng.uniform(0.01, 0.05, 4)
    g = case.oracle_geom(O)
    vol = O.phantom_voxelize(g, ell, ss=4)
    exact = O.phantom_project(g, ell, case.angles, case.offsets)
    disc = O.forward(g, vol, case.angles, case.offsets, spp=4.0)
    e64 = O.rel_l2(disc, exact)
    assert e64 < 0.03
    assert abs(disc.sum() / exact.sum() - 1) < 2e-4          # line-integral mass is conserved
    # halving the voxel size shrinks the (edge) discretisation error
    case.nx = case.ny = case.nz = 128
    g2 = case.oracle_geom(O)
    disc2 = O.forward(g2, O.phantom_voxelize(g2, ell, ss=2), case.angles, case.offsets, spp=2.0)
    e128 = O.rel_l2(disc2, O.phantom_project(g2, ell, case.angles, case.offsets))
    assert e128 < 0.8 * e64


def test_osmom_recurrence_vs_numpy(O):
    """osMOMSolverD.h:82-196 restated in numpy over the oracle's projectors."""
    case = make("cube")
    g = case.oracle_geom(O)
    rng = np.random.default_rng(5)
    truth = np.zeros((case.nz, case.ny, case.nx))
    truth[8:24, 10:22, 6:26] = 0.02
    order, sizes = O.subset_partition(case.angles.size, 3)
    a, o = case.angles[order], case.offsets[order]
    b = O.forward(g, truth, a, o) + rng.normal(0, 1e-3, (a.size, case.H, case.W))
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    S, iters = 3, 3

    def M(s, x):
        f, n = first[s], sizes[s]
        return O.forward(g, x, a[f:f + n], o[f:f + n])

    def MH(s, y):
        f, n = first[s], sizes[s]
        return O.backproject(g, y, a[f:f + n], o[f:f + n])

    ones = np.ones_like(truth)
    pre = sum(MH(s, M(s, ones)) for s in range(S))
    D = 1.0 / np.maximum(pre, 1e-6)
    z = np.zeros_like(truth)
    x, xold = z.copy(), z.copy()
    t = told = 1.0
    for it in range(iters):
        for s in range(S):
            t = 0.5 * (1 + math.sqrt(1 + 4 * t * t))
            r = M(s, x) - b[first[s]:first[s] + sizes[s]]
            z = z - S * (MH(s, r) * D)
            x = np.maximum(z, 0)
            z = x * (1 + (told - 1) / t) - (told - 1) / t * xold
            x, xold = xold, x
            x = z.copy()
            told = t
    zo, _ = O.osmom(g, b, a, o, sizes, np.zeros(S, np.int32), iters=iters, nonneg=True)
    assert np.max(np.abs(zo - z)) <= 1e-9 * max(1.0, np.max(np.abs(z)))


def test_binned_osmom_is_per_bin(O, gtb):
    """With bins, each bin's reconstruction equals the one-bin solve of that
    bin's views under the same subset schedule (the bins share only t)."""
    case = make("cube")
    g = case.oracle_geom(O)
    ell = gtb.phantom.ellipsoids(13, (case.lx, case.ly, case.lz), n=5)
    b = O.phantom_project(g, ell.astype(np.float64), case.angles, case.offsets)
    P = case.angles.size
    vbin = ((np.arange(P) // 2) % 2).astype(np.int32)
    order, sizes = gtb.subset_partition(P, 3, vbin)
    a, o, bb, vb = case.angles[order], case.offsets[order], b[order], vbin[order]
    z2, _ = O.osmom(g, bb, a, o, sizes, np.zeros(3, np.int32), iters=2, nonneg=True, view_bin=vb, n_bins=2)
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    for sel in (0, 1):
        keep = vb == sel
        sz = [int(keep[f:f + n].sum()) for f, n in zip(first, sizes)]
        z1, _ = O.osmom(g, bb[keep], a[keep], o[keep], sz, np.zeros(3, np.int32), iters=2, nonneg=True)
        assert np.array_equal(z2[sel], z1)


def test_tv_osmom_vs_numpy(O):
    """The TV-regularised osMOMSolverD (denoise and updateG, osMOMSolverD.h:205-247,
    with cuTVPrimalDualOperator.cu:9-62) restated in numpy over the oracle's
    projectors; the periodic differences use np.roll."""
    case = make("cube")
    g = case.oracle_geom(O)
    rng = np.random.default_rng(7)
    truth = np.zeros((case.nz, case.ny, case.nx))
    truth[8:24, 10:22, 6:26] = 0.02
    order, sizes = O.subset_partition(case.angles.size, 3)
    a, o = case.angles[order], case.offsets[order]
    b = O.forward(g, truth, a, o) + rng.normal(0, 2e-3, (a.size, case.H, case.W))
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    S, iters, lam, alpha, tau0, steps = 3, 2, 0.05, 0.1, 1e-3, 2

    def M(s, x):
        f, n = first[s], sizes[s]
        return O.forward(g, x, a[f:f + n], o[f:f + n])

    def MH(s, y):
        f, n = first[s], sizes[s]
        return O.backproject(g, y, a[f:f + n], o[f:f + n])

    def denoise(x, sv, D, gam):
        tau, sigma = tau0, 1.0 / (tau0 * 16.0)
        for _ in range(steps):
            scale = sigma / (1.0 + sigma * alpha)
            d = np.stack([(np.roll(x, -1, axis=ax) - x) * scale for ax in (2, 1, 0)])
            P = d / np.maximum(1.0, np.sqrt((d * d).sum(axis=0)))
            gv = sum(np.roll(P[i], 1, axis=ax) - P[i] for i, ax in enumerate((2, 1, 0)))
            x = ((x - tau * gv) + tau / lam * (sv / D)) / ((1.0 / D) * (tau / lam) + 1.0)
            theta = 1.0 / math.sqrt(1.0 + 2.0 * gam * tau)
            tau, sigma = tau * theta, sigma / theta
        return x

    ones = np.ones_like(truth)
    pre = sum(MH(s, M(s, ones)) for s in range(S))
    D = 1.0 / np.maximum(pre, 1e-6)
    gam = 0.35 / lam / (D.size / np.abs(D).sum())
    z = np.zeros_like(truth)
    x, xold = z.copy(), z.copy()
    t = told = 1.0
    for it in range(iters):
        for s in range(S):
            t = 0.5 * (1 + math.sqrt(1 + 4 * t * t))
            r = M(s, x) - b[first[s]:first[s] + sizes[s]]
            z = z - S * (MH(s, r) * D)
            x = np.maximum(denoise(x, z, D, gam), 0)
            z = x * (1 + (told - 1) / t) - (told - 1) / t * xold
            x, xold = xold, x
            x = z.copy()
            told = t
    zo, _ = O.osmom(g, b, a, o, sizes, np.zeros(S, np.int32), iters=iters, nonneg=True, tv_weight=lam,
                    tv_alpha=alpha, tau=tau0, reg_steps=steps)
    assert np.max(np.abs(zo - z)) <= 1e-9 * max(1.0, np.max(np.abs(z)))
    plain, _ = O.osmom(g, b, a, o, sizes, np.zeros(S, np.int32), iters=iters, nonneg=True)
    assert np.max(np.abs(plain - z)) > 1e-6   # the prior does change the result

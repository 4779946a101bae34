"""The roofline fields of bench.py's JSON line (CPU): per-variant ncu counters
read from profiles/traffic.json, and the issue ceiling of the forward
projector (warp instructions per launch over 148 SMs x 4 issue slots)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_traffic_per_variant():
    bench = _bench()
    for v in ("tma-quad", "tma-pair", "tma-slab"):
        t = bench.traffic_for("forward_residual", "c2", v)
        n = bench.traffic_for("forward_residual_warp_instr", "c2", v)
        assert isinstance(t, int) and t > 152_043_520          # at least the algorithmic bytes
        assert isinstance(n, int) and n > 0
    assert bench.traffic_for("forward_residual", "c2", "gather") is None
    assert bench.traffic_for("forward_residual", "no-such-workload", "tma-quad") is None


def test_issue_roofline():
    bench = _bench()
    samples = 512 * 384 * 36 * 384
    # one warp instruction per sample at 1965 MHz: 148 * 4 * 1.965e9 samples/s
    r = bench.issue_roofline(samples, samples, 1.0, 1965.0)
    assert abs(r["ceiling_gsamples_per_s"] - 148 * 4 * 1.965) < 0.1
    assert abs(r["frac"] - samples / 1e9 / r["ceiling_gsamples_per_s"]) < 1e-3
    assert bench.issue_roofline(None, samples, 1.0, 1965.0) is None
    assert bench.issue_roofline(samples, samples, 1.0, None) is None

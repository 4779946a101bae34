"""Benchmark of the cone-beam OS-MOM hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2|c1|c3|c4|c5]

Workload (default, c2): OS-MOM reconstruction (osMOMSolverD semantics,
positivity, no regulariser) of a 256^3 seeded ellipsoid phantom from 360
views over 360 degrees on a 512x384 detector at 0.8 mm with an 80 mm half-fan
offset, Poisson noise at I0 = 1e5, log transform; 10 subsets, 20 iterations,
FP32.  Voxel size 1 mm and SAD/SDD = 1000/1500 mm are assumptions (the
workload does not state them).  A step is one full reconstruction
(preconditioner + 20 x 10 subset steps).

value  = GUPS: (forward ray samples + back-projection voxel-view updates) per
         second, all ranks, device-timed with CUDA events, inputs resident.
e2e    = the same metric through the public API with host buffers: each step
         copies the measured projections host->device (pinned) and the
         reconstruction device->host inside the timed region.
N > 1  = independent replicas (one reconstruction per GPU, no collective),
         weak scaling; time is the max over ranks.
--impl reference times the reference algorithm's CPU restatement (the oracle,
FP32, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "traffic.json")


def _package():
    name = "gt_tomography_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "gt-tomography_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------ workload
class Workload:
    def __init__(self, name: str):
        self.name = name
        if name == "c2":
            self.n = (256, 256, 256)
            self.voxel = 1.0
            self.P = 360
            self.W, self.H, self.pitch = 512, 384, 0.8
            self.offset = 80.0
            self.S, self.iters = 10, 20
            self.I0 = 1e5
            self.n_ell = 10
        elif name == "c1":
            self.n = (128, 128, 128)
            self.voxel = 1.0
            self.P = 180
            self.W, self.H, self.pitch = 256, 192, 1.5
            self.offset = 0.0
            self.S, self.iters = 1, 0
            self.I0 = 0
            self.n_ell = 10
        else:
            raise ValueError(name)
        self.SAD, self.SDD = 1000.0, 1500.0
        self.L = tuple(v * self.voxel for v in self.n)
        self.spp = 1.5
        self.Nsamp = int(np.float32(self.spp) * np.float32(self.n[0]))
        self.seed = 1234

    def config(self):
        if self.name == "c2":
            wl = (f"osmom {self.n[0]}^3 from {self.P} views {self.W}x{self.H}@{self.pitch}mm, "
                  f"offset {self.offset:g}mm, {self.S} subsets x {self.iters} iterations, fp32")
        else:
            wl = (f"forward + FDK {self.n[0]}^3 from {self.P} views {self.W}x{self.H}@{self.pitch}mm, "
                  "Hann ramp, fp32")
        return {
            "workload": wl,
            "volume": list(self.n), "voxel_mm": self.voxel, "views": self.P, "detector": [self.W, self.H],
            "pixel_mm": self.pitch, "offset_mm": self.offset, "SAD_mm": self.SAD, "SDD_mm": self.SDD,
            "subsets": self.S, "iterations": self.iters, "I0": self.I0, "samples_per_ray": self.Nsamp,
            "ellipsoids": self.n_ell, "seed": self.seed, "storage": "fp32",
            "assumed": ["voxel_mm", "SAD_mm", "SDD_mm"],
            "step": "one full reconstruction" if self.name == "c2" else "one forward pass + one FDK",
            "l2": "flushed between steps (256 MiB write); projections exceed L2",
            "parallelism": "replicas",
        }

    def geometry(self, gtb):
        return gtb._lib.CbctGeometry(self.SAD, self.SDD, self.W * self.pitch, self.H * self.pitch, self.W, self.H,
                                     *self.n, *self.L, self.spp)

    def updates_per_step(self):
        """(forward samples, back-projection voxel-view updates) per step."""
        rays = self.W * self.H * self.P
        nvox = self.n[0] * self.n[1] * self.n[2]
        if self.name == "c2":
            passes = self.iters + 1      # + preconditioner A^T A 1
            return rays * self.Nsamp * passes, nvox * self.P * passes
        return rays * self.Nsamp, nvox * self.P

    def launches_per_step(self):
        # Every subset of this orbit holds x-dominant views, so each forward
        # launch is preceded by the x/y transpose of the volume.
        if self.name == "c2":
            # fill + S (transpose + forward) + 1 back-projection (preconditioner), then
            # per subset step: transpose, forward-residual, norm finalise,
            # back-projection with the update.
            return 1 + 2 * self.S + 1 + self.iters * self.S * 4
        return 2 + 1 + 1            # transpose + forward, FDK filter, FDK back-projection


FORWARD_KERNELS = {"auto": 0, "slab": 1, "gather": 2, "fan": 3, "pair": 4, "quad": 5}
FORWARD_KERNEL_NAMES = {"tma-quad": "fwd_quad_kernel", "tma-pair": "fwd_pair_kernel", "tma-slab": "fwd_slab_kernel",
                        "tma-fan": "fwd_fan_kernel", "gather": "fwd_gather_kernel"}


def make_inputs(wl: Workload, gtb, dev, forward_kernel: str = "auto"):
    """Seeded phantom, exact line integrals on the device, Poisson noise, log.
    forward_kernel: the plan's forward projector (CBCT_OPT_FORWARD_KERNEL)."""
    import torch
    ang = gtb.phantom.circular_orbit(wl.P)
    off = np.tile(np.array([[wl.offset, 0.0]], np.float32), (wl.P, 1))
    ell = gtb.phantom.ellipsoids(wl.seed, wl.L, n=wl.n_ell)
    order, sizes = gtb.subset_partition(wl.P, wl.S)
    a, o = ang[order] - ang.min(), off[order]
    g = wl.geometry(gtb)
    fw = float(wl.W * wl.pitch)
    oc = [int(abs(float(o[f:f + n, 0].mean())) > 0.1 * fw) if n else 0
          for f, n in zip(np.concatenate([[0], np.cumsum(sizes)[:-1]]), sizes)]
    plan = gtb.Plan(g, a, o, sizes, oc)
    if forward_kernel != "auto":
        plan.set_option(gtb._lib.CBCT_OPT_FORWARD_KERNEL, FORWARD_KERNELS[forward_kernel])
    ell_d = torch.from_numpy(ell.reshape(-1)).to(dev)
    exact = torch.empty(plan.proj_shape(), dtype=torch.float32, device=dev)
    plan.phantom_project(ell_d, exact)
    b = gtb.phantom.poisson_log(exact, wl.I0, wl.seed + 1) if wl.I0 else exact
    torch.cuda.synchronize()
    return plan, b.contiguous(), ell_d, (a, o, sizes, oc)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"cbct_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ helpers
def peaks():
    try:
        d = json.load(open(PEAKS_PATH))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_for(kernel: str, workload: str, variant: str | None = None):
    """A per-launch ncu counter of `kernel` (DRAM bytes, or warp instructions for
    the `_warp_instr` entries) from one capture (profiles/traffic.json), per
    forward variant where the file keeps several."""
    try:
        d = json.load(open(TRAFFIC_PATH))
        t = d.get(workload, {}).get(kernel)
        return t.get(variant) if isinstance(t, dict) else t
    except Exception:
        return None


def issue_roofline(warp_instr, samples, seconds, sm_mhz, n_sm=148, issue_per_clk=4):
    """The forward projector's own ceiling: warp instructions per launch (ncu)
    over the SMs' issue slots (4 per SM per clock) at the sampled SM clock."""
    if not warp_instr or not sm_mhz:
        return None
    peak = n_sm * issue_per_clk * sm_mhz * 1e6            # warp instructions per second
    ceiling = samples / (warp_instr / peak)               # samples per second at 100 % issue
    achieved = samples / seconds
    return {"warp_instr_per_launch": warp_instr, "ceiling_gsamples_per_s": round(ceiling / 1e9, 1),
            "achieved_gsamples_per_s": round(achieved / 1e9, 1), "frac": round(achieved / ceiling, 3),
            "source": "ncu smsp__inst_executed.sum of one launch (profiles/), 148 SMs x 4 issue slots"}


def flush_l2(buf):
    buf.fill_(1.0)


def dist_setup(backend: str = "nccl", timeout_s: float = 600.0):
    """Rank, world size and local rank from the torchrun environment; joins the
    process group when there is more than one rank (replicas: the group only
    carries the barrier and the max-over-ranks reduction of the step time)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not torch.distributed.is_initialized():
        import datetime
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def max_over_ranks(v: float, world: int, device: str = "cuda") -> float:
    import torch
    if world == 1:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Units processed by all ranks (replicas do equal work) per second of the
    slowest rank, in billions."""
    return units_per_rank * world / (ms_max * 1e-3) / 1e9


def barrier(world, sync_cuda: bool = True):
    import torch
    if world > 1:
        torch.distributed.barrier()
    if sync_cuda:
        torch.cuda.synchronize()


# ------------------------------------------------------------------ CPU legs
def cpu_sample(wl: Workload, budget_s: float = 6.0):
    """The reference algorithm's CPU restatement (oracle, FP32, all host threads)
    on a bounded sample: forward + back-projection of k views of the workload."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_num_threads(threads)
    g = O.Geometry(*wl.n, *wl.L, wl.W, wl.H, wl.W * wl.pitch, wl.H * wl.pitch, wl.SAD, wl.SDD)
    rng = np.random.default_rng(0)
    vol = rng.uniform(0, 0.02, wl.n[::-1]).astype(np.float32)
    ang = np.arange(wl.P, dtype=np.float32) * (360.0 / wl.P)
    off = np.tile(np.array([[wl.offset, 0.0]], np.float32), (wl.P, 1))

    def run(k):
        t0 = time.perf_counter()
        p = O.forward(g, vol, ang[:k], off[:k], spp=wl.spp, dtype=np.float32)
        O.backproject(g, p, ang[:k], off[:k], dtype=np.float32)
        return time.perf_counter() - t0

    t1 = run(1)
    k = int(max(1, min(wl.P, budget_s / max(t1, 1e-3))))
    return O, g, vol, ang, off, k, threads, run


def cpu_gups(wl, k, t):
    rays = wl.W * wl.H * k
    nvox = wl.n[0] * wl.n[1] * wl.n[2]
    return (rays * wl.Nsamp + nvox * k) / t / 1e9


def reference_arm(args, wl: Workload):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O, g, vol, ang, off, k, threads, run = cpu_sample(wl, budget_s=4.0)
    for _ in range(args.warmup):
        run(k)
    times = [run(k) for _ in range(args.steps)]
    t = sum(times) / len(times)
    v = cpu_gups(wl, k, t)
    sample = f"forward + back-projection of {k} of {wl.P} views per step (oracle port, fp32)"
    line = {
        "metric": "GUPS fwd+back projection (OS-MOM reconstruction)", "value": round(v, 4), "unit": "GUPS",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": wl.config(),
        "cpu_baseline": {"value": round(v, 4), "unit": "GUPS", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 4), "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def ours(args, wl: Workload):
    import torch
    rank, world, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    gtb = _package()
    plan, b, ell_d, (a, o, sizes, oc) = make_inputs(wl, gtb, dev, args.forward_kernel)
    nvox = wl.n[0] * wl.n[1] * wl.n[2]
    z = torch.empty(plan.vol_shape, dtype=torch.float32, device=dev)
    resid = torch.zeros(max(wl.iters * wl.S, 1), dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    filt = gtb.hann_ramp_filter(wl.W)

    def step():
        if wl.name == "c2":
            plan.osmom(b, z, None, wl.iters, nonneg=True, use_graph=True, resid=resid)
        else:
            tmp = proj_tmp
            plan.forward(vol_c1, tmp)
            plan.fdk(b, z, filt, 0)

    if wl.name == "c1":
        vol_c1 = torch.empty(plan.vol_shape, dtype=torch.float32, device=dev)
        gtb.phantom_voxelize(wl.geometry(gtb), ell_d, vol_c1, 4)
        proj_tmp = torch.empty_like(b)

    # ---- device-timed region (inputs resident)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    times = []
    barrier(world)
    for _ in range(args.steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(sum(times) / len(times), world)
    fs, bv = wl.updates_per_step()
    gups = whole_job_rate(fs + bv, world, ms)

    # ---- end-to-end through the public API with host buffers
    b_host = b.cpu().pin_memory()
    z_host = torch.empty(plan.vol_shape, dtype=torch.float32).pin_memory()
    b_dev = torch.empty_like(b)
    e2e_times = []

    def e2e_step():
        b_dev.copy_(b_host, non_blocking=True)
        if wl.name == "c2":
            plan.osmom(b_dev, z, None, wl.iters, nonneg=True, use_graph=True, resid=resid)
        else:
            plan.forward(vol_c1, proj_tmp)
            plan.fdk(b_dev, z, filt, 0)
        z_host.copy_(z, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    for _ in range(args.steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_times.append(e0.elapsed_time(e1))
    barrier(world)
    # Device-side status of everything above: raises CBCT_ERR_TIMEOUT or
    # CBCT_ERR_DEVICE_CHECK if any kernel gave up a bounded wait or overflowed
    # a shared-memory box (the solve reports it on return as well).
    plan.check()
    ms_e2e = max_over_ranks(sum(e2e_times) / len(e2e_times), world)
    gups_e2e = whole_job_rate(fs + bv, world, ms_e2e)

    # ---- dominant kernel: forward residual of one subset, timed alone
    s0 = 0
    n0 = int(sizes[s0])
    r = torch.empty(plan.proj_shape(s0), dtype=torch.float32, device=dev)
    bs = b[:n0]
    n2 = torch.zeros(1, dtype=torch.float64, device=dev)
    for _ in range(3):
        plan.forward_residual(z, bs, r, s0, 1.0, bool(oc[s0]), n2)
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        plan.forward_residual(z, bs, r, s0, 1.0, bool(oc[s0]), None)
    e1.record(stream)
    e1.synchronize()
    t_fwd = e0.elapsed_time(e1) / reps * 1e-3
    rays0 = wl.W * wl.H * n0
    alg_bytes = 4 * nvox + 4 * rays0 * 3        # volume + b read + r write (+ per-pixel offset weight computed)
    hbm, peak_kind = peaks()
    variant = plan.forward_variant()
    achieved = alg_bytes / t_fwd / 1e9
    samples_s = rays0 * wl.Nsamp / t_fwd

    # ---- the back-projector of the same subset, timed alone (store epilogue)
    vtmp = torch.empty(plan.vol_shape, dtype=torch.float32, device=dev)
    for _ in range(3):
        plan.backproject(r, vtmp, s0, 0, False, False)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        plan.backproject(r, vtmp, s0, 0, False, False)
    e1.record(stream)
    e1.synchronize()
    t_bp = e0.elapsed_time(e1) / reps * 1e-3
    bp_bytes = 4 * rays0 + 4 * nvox                # r read + volume write
    plan.check()

    # ---- on-chip ceilings of the projectors' inner operation (this run, this GPU)
    import ctypes as C
    L = gtb._lib
    tri, bil = C.c_double(0.0), C.c_double(0.0)
    L.call("cbct_microbench_interp", 3, 256, C.byref(tri), None)
    L.call("cbct_microbench_interp", 2, 256, C.byref(bil), None)
    bp_rate = nvox * n0 / t_bp

    # ---- the reference's own kernel structure on the same subset, device-only
    ref_kernels = None
    if rank == 0:
        ms2 = (C.c_float * 2)()
        g_ = wl.geometry(gtb)
        aa0 = np.ascontiguousarray(a[:n0], np.float32)
        oo0 = np.ascontiguousarray(o[:n0], np.float32)
        ptmp = torch.empty(plan.proj_shape(s0), dtype=torch.float32, device=dev)
        L.call("cbct_plain_kernel_times", C.byref(g_), aa0.ctypes.data, oo0.ctypes.data, n0, z.data_ptr(),
               bs.data_ptr(), ptmp.data_ptr(), vtmp.data_ptr(), 3, ms2)
        ref_kernels = {
            "what": "the reference's conebeam_forwards_projection_kernel and conebeam_backwards_projection_kernel "
                    "(tex3D / tex2DLayered, one thread per ray / voxel) on the same subset, textures built "
                    "outside the timed launches",
            "forward_ms": round(ms2[0], 4), "forward_gsamples_per_s": round(rays0 * wl.Nsamp / ms2[0] * 1e-6, 1),
            "backproject_ms": round(ms2[1], 4), "backproject_gups": round(nvox * n0 / ms2[1] * 1e-6, 1),
            "ours_forward_speedup": round(ms2[0] / (t_fwd * 1e3), 3),
            "ours_backproject_speedup": round(ms2[1] / (t_bp * 1e3), 3)}

    line = {
        "metric": "GUPS fwd+back projection (OS-MOM reconstruction)",
        "value": round(gups, 3), "unit": "GUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": wl.config(),
        "recon_per_s": round(world * 1e3 / ms, 4) if wl.name == "c2" else None,
        "e2e": {"value": round(gups_e2e, 3), "unit": "GUPS", "ms_per_step": round(ms_e2e, 3),
                "h2d_bytes_per_step": int(b.numel() * 4), "d2h_bytes_per_step": int(nvox * 4)},
        "roofline": {"bound": "hbm", "kernel": f"{FORWARD_KERNEL_NAMES.get(variant, variant)} (forward residual, "
                                                 "one subset)",
                     "achieved": round(achieved, 2), "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / hbm, 5), "traffic": traffic_for("forward_residual", wl.name, variant),
                     "launch_ms": round(t_fwd * 1e3, 4), "alg_bytes_per_launch": alg_bytes,
                     "gsamples_per_s": round(samples_s / 1e9, 2),
                     "issue": issue_roofline(traffic_for("forward_residual_warp_instr", wl.name, variant),
                                             rays0 * wl.Nsamp, t_fwd, clk.get("sm_mhz") if clk else None),
                     "limiter": "on chip: shared-memory interpolation and FP32 issue (compulsory HBM bytes are "
                                "a small fraction by design)",
                     "onchip": {"achieved_gsamples_per_s": round(samples_s / 1e9, 1),
                                "peak_gsamples_per_s": round(tri.value / 1e9, 1),
                                "frac": round(samples_s / tri.value, 3),
                                "peak": "cbct_microbench_interp kind 3: FP32 trilinear interpolations per second "
                                        "from a shared-memory box, this run"}},
        "backproject": {"kernel": "bp_tma_kernel (store epilogue, one subset)", "launch_ms": round(t_bp * 1e3, 4),
                        "gups": round(bp_rate / 1e9, 1),
                        "hbm": {"achieved": round(bp_bytes / t_bp / 1e9, 2), "peak": hbm,
                                "frac": round(bp_bytes / t_bp / 1e9 / hbm, 5), "alg_bytes_per_launch": bp_bytes},
                        "onchip": {"peak_gups": round(bil.value / 1e9, 1), "frac": round(bp_rate / bil.value, 3),
                                   "peak": "cbct_microbench_interp kind 2: FP32 bilinear interpolations per "
                                           "second from a shared-memory box, this run"}},
        "reference_kernels": ref_kernels,
        "gpu_launches": wl.launches_per_step() * args.steps,
        "forward_variant": variant,
        "device_flags": "clear",
        "clocks": clk,
    }
    if rank == 0 and world == 1 and wl.name == "c2" and not args.no_plain:
        # The plain FP32 one-scan-at-a-time path (reference structure, texture
        # filtering) on the same inputs: one warm-up and three timed
        # reconstructions, the median reported.  Its per-call allocations,
        # array copies and host-synchronised norms make it host-bound, so its
        # time varies between hosts far more than the device-resident path's.
        import ctypes as C
        L = gtb._lib
        g = wl.geometry(gtb)
        aa = np.ascontiguousarray(a, np.float32)
        oo = np.ascontiguousarray(o, np.float32)
        sz = np.ascontiguousarray(sizes, np.int32)
        ocv = np.ascontiguousarray(oc, np.int32)
        zp = torch.empty_like(z)

        def plain_step():
            L.call("cbct_plain_osmom_solve", C.byref(g), aa.ctypes.data, oo.ctypes.data, aa.size, sz.ctypes.data,
                   len(sz), ocv.ctypes.data, b.data_ptr(), zp.data_ptr(), wl.iters, 1, None)

        plain_step()
        torch.cuda.synchronize()
        plain_ms = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plain_step()
            e1.record(stream)
            e1.synchronize()
            plain_ms.append(e0.elapsed_time(e1))
        ms_plain = sorted(plain_ms)[1]
        plan.osmom(b, z, None, wl.iters, nonneg=True, use_graph=True, resid=resid)
        torch.cuda.synchronize()
        diff = float((z.double() - zp.double()).norm() / zp.double().norm())
        line["plain_path"] = {"ms_per_step": round(ms_plain, 1), "ms_each": [round(t, 1) for t in plain_ms],
                              "value": round(whole_job_rate(fs + bv, 1, ms_plain), 3),
                              "unit": "GUPS", "speedup_of_value": round(ms_plain / ms, 3),
                              "rel_l2_ours_vs_plain": diff,
                              "what": "reference structure re-hosted on B200: texture filtering, per-call "
                                      "cudaArray copies and uploads, element-wise passes, host-synced norms"}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            O, g, vol, ang, off, k, threads, run = cpu_sample(wl, budget_s=8.0)
            t = run(k)
            line["cpu_baseline"] = {"value": round(cpu_gups(wl, k, t), 4), "unit": "GUPS", "cores": threads,
                                    "kind": "port",
                                    "sample": f"forward + back-projection of {k} of {wl.P} views (oracle, fp32)"}
            # accuracy of the FP32 device path against the FP64 oracle at full size (2 views)
            pl2 = gtb.Plan(wl.geometry(gtb), ang[:2], off[:2])
            vt = torch.from_numpy(vol).to(dev)
            pg = torch.empty(pl2.proj_shape(), dtype=torch.float32, device=dev)
            pl2.forward(vt, pg)
            ref = O.forward(g, vol.astype(np.float64), ang[:2], off[:2], spp=wl.spp)
            bg = torch.empty(pl2.vol_shape, dtype=torch.float32, device=dev)
            pl2.backproject(torch.from_numpy(ref.astype(np.float32)).to(dev), bg, -1, 0, False)
            refb = O.backproject(g, ref, ang[:2], off[:2])
            line["rel_l2_vs_fp64"] = {"forward_2views": O.rel_l2(pg.cpu().numpy(), ref),
                                      "backproject_2views": O.rel_l2(bg.cpu().numpy(), refb)}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "GUPS", "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {e}"}
    if rank == 0 and world == 1 and wl.name == "c2" and not args.no_legs:
        line["batching_serving"] = batching_serving_legs(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def batching_serving_legs(args):
    """The batching and serving comparisons at reduced size, so that the
    default run carries them: the serving loop on the first 12 requests of the
    C5 stream (same seeds, kinds, storage and 20/s arrivals) with the plain
    FP32 FIFO beside it, the batch executors on the first 8 scans of the C4
    set against the same scans solved one at a time (and the plain path on
    two of them), and the batch executors on 64 smaller scans (64-128^3, the
    "small" set), where the fused work lists merge the scans' partly idle
    waves.  The full runs are --config c5 and --config c4."""
    import copy
    out = {"sizes": "reduced: 12 served requests (C5 stream, seed 5), 8 batched scans (C4 seeds 1000..1007); "
                    "64 batched scans of the small set (seeds 3000..3063)"}
    try:
        a = copy.copy(args)
        a.requests, a.no_plain = 12, False
        s = served_line(a)
        out["served"] = {k: s.get(k) for k in ("value", "unit", "latency_p50_s", "latency_p99_s",
                                               "peak_requests_in_flight", "plain_path", "speedup_vs_plain",
                                               "storage_bf16_vs_f32_rel_l2")}
    except Exception as e:  # reported, never required
        out["served"] = {"error": str(e)}
    try:
        a = copy.copy(args)
        a.scans, a.steps, a.warmup, a.plain_sample, a.autotune = 8, 1, 1, 2, False
        b = batched_line(a)
        out["batched"] = {k: b.get(k) for k in ("value", "unit", "one_at_a_time", "stream_pool", "fused",
                                                "speedup_batched_vs_one_at_a_time", "plain_path")}
        out["batched"]["executor"] = b["config"]["executor"]
    except Exception as e:
        out["batched"] = {"error": str(e)}
    try:
        a = copy.copy(args)
        a.scans, a.steps, a.warmup, a.plain_sample, a.autotune, a.scan_sizes = 64, 1, 1, 0, False, "small"
        b = batched_line(a)
        out["batched_small"] = {k: b.get(k) for k in ("value", "unit", "one_at_a_time", "stream_pool", "fused",
                                                      "speedup_batched_vs_one_at_a_time")}
        out["batched_small"]["executor"] = b["config"]["executor"]
    except Exception as e:
        out["batched_small"] = {"error": str(e)}
    out["note"] = ("kernels here are bound on chip, not by HBM: 16-bit storage halves memory per request but "
                   "adds a conversion per tap; scans that fill the GPU gain nothing from running together, "
                   "smaller scans gain from the fused work lists; the ratios against the plain path come from "
                   "its per-call host work and texture path")
    return out


def kernel_only(args, wl: Workload):
    """Runs one kernel of the workload `--steps` times after `--warmup` launches
    (for profiler captures): forward = forward residual of subset 0,
    backproject = back-projection of subset 0, fdk = the FDK row filter of
    every view, tv = one TV primal-dual step (primal + fused dual/update)."""
    import torch
    dev = torch.device("cuda", 0)
    gtb = _package()
    L = gtb._lib
    plan, b, ell_d, (a, o, sizes, oc) = make_inputs(wl, gtb, dev, args.forward_kernel)
    n0 = int(sizes[0])
    vol = torch.full(plan.vol_shape, 0.01, dtype=torch.float32, device=dev)
    r = torch.empty(plan.proj_shape(0), dtype=torch.float32, device=dev)
    bs = b[:n0].contiguous()
    stream = torch.cuda.current_stream()

    if args.only == "fdk":
        # FDK filter of every view (cosine + ramp + offset weight), 283 MB in and out
        rf = torch.empty_like(b)
        filt = gtb.hann_ramp_filter(wl.W)
    if args.only == "tv":
        # one TV primal-dual step on the volume (gradient field 201 MB)
        P3 = torch.empty((3,) + plan.vol_shape, dtype=torch.float32, device=dev)
        sv = torch.full(plan.vol_shape, 0.01, dtype=torch.float32, device=dev)
        D = torch.full(plan.vol_shape, 0.02, dtype=torch.float32, device=dev)
        nz_, ny_, nx_ = plan.vol_shape

    def one():
        if args.only == "forward":
            plan.forward_residual(vol, bs, r, 0, 1.0, bool(oc[0]), None)
        elif args.only == "backproject":
            plan.backproject(bs, vol, 0, 0, False, True)
        elif args.only == "fdk":
            plan.fdk_filter(b, rf, -1, filt, L.CBCT_FDK_RAMP | L.CBCT_FDK_COSINE | L.CBCT_FDK_OFFSET)
        else:
            gtb.operators.tv_step(vol, P3, sv, D, 0.5, 1e-3, 0.02)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        one()
    e1.record(stream)
    e1.synchronize()
    print(json.dumps({"kernel": args.only, "ms_per_launch": e0.elapsed_time(e1) / max(args.steps, 1),
                      "variant": plan.forward_variant(), "views": n0}), flush=True)


def batched(args):
    print(json.dumps(batched_line(args)), flush=True)


# Scan sets of the batched configuration: uneven_scans ranges and first seed.
SCAN_SETS = {
    "c4": dict(seed0=1000),
    "small": dict(seed0=3000, vol_range=(64, 128), z_range=(64, 128), view_range=(60, 180), width_range=(128, 256)),
    "medium": dict(seed0=3000, vol_range=(96, 160), z_range=(96, 160), view_range=(90, 360),
                   width_range=(256, 384)),
    "tiny": dict(seed0=3000, vol_range=(32, 64), z_range=(32, 64), view_range=(40, 120), width_range=(64, 128)),
}


def batched_line(args):
    """Batched reconstruction of many uneven scans (the batched
    configuration): 64 seeded scans, volumes 96..320 (z 64..320), 90..720
    views, detectors 256x192..768x576, I0 = 1e5, OS-MOM with 8 subsets x 10
    iterations, fp32.  A step solves every scan once.  Reports recon/s of the
    batch executors (stream pool, fused work lists) and of the same solves run
    one scan at a time.  --scan-sizes picks a set of smaller scans instead,
    --executor one executor alone, --iterations the OS-MOM iterations."""
    import torch
    dev = torch.device("cuda", 0)
    gtb = _package()
    it = args.iterations
    specs = gtb.phantom.uneven_scans(args.scans, **SCAN_SETS[args.scan_sizes])
    scans = [gtb.phantom.make_osmom_scan(sp, 8, 1e5, dev) for sp in specs]
    variants = {}
    if args.autotune:
        # per-scan choice of projector variants (timed on each plan's largest subset)
        for pl, _, _ in scans:
            t = pl.autotune()
            key = (t["forward_variant"], "bp-tma" if (t["backproject_tma"] or 1e9) <= (t["backproject_global"] or 1e9)
                   else "bp-global")
            variants["+".join(key)] = variants.get("+".join(key), 0) + 1
    zs = [torch.empty(pl.vol_shape, dtype=torch.float32, device=dev) for pl, _, _ in scans]
    jobs = [dict(plan=pl, b=b, z=z, iterations=it, nonneg=True) for (pl, b, _), z in zip(scans, zs)]
    stream = torch.cuda.current_stream()
    updates = 0
    for sp in specs:
        nvox = sp["n"][0] * sp["n"][1] * sp["n"][2]
        N = int(np.float32(1.5) * np.float32(sp["n"][0]))
        updates += (it + 1) * (sp["W"] * sp["H"] * sp["P"] * N + nvox * sp["P"])

    def one_at_a_time():
        for j in jobs:
            j["plan"].osmom(j["b"], j["z"], None, it, nonneg=True, use_graph=True)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    run_pool, run_fused, run_seq = (args.executor in ("both", "pool"), args.executor in ("both", "fused"),
                                    args.executor == "both")

    def pool():
        gtb.batch_osmom(jobs, n_streams=args.streams)

    def fused():
        gtb.batch_osmom(jobs, fused=True)

    for _ in range(max(args.warmup, 1)):
        for run, fn in ((run_seq, one_at_a_time), (run_pool, pool), (run_fused, fused)):
            if run:
                fn()
    clocks = ClockSampler(0)
    clocks.start()
    mean = lambda fn, run: sum(timed(fn) for _ in range(args.steps)) / args.steps if run else None
    ms_p, ms_f, ms_s = mean(pool, run_pool), mean(fused, run_fused), mean(one_at_a_time, run_seq)
    clk = clocks.stop()
    # The headline is the faster executor; both are reported.
    ms_b, executor = min((t, name) for t, name in ((ms_f, "fused work-list"), (ms_p, "stream pool")) if t is not None)
    plain = None
    if args.plain_sample > 0:
        # The plain FP32 one-scan-at-a-time path (reference structure) on an
        # evenly spaced sample of the scans, each next to the same scan solved
        # alone through a plan; the plain time of all scans is estimated as
        # ours-one-at-a-time x (plain / ours on the sample).
        import ctypes as C
        L = gtb._lib
        idx = list(range(0, len(jobs), max(1, len(jobs) // args.plain_sample)))[:args.plain_sample]

        def plain_solve(i):
            pl, b, (a, o, sizes, oc) = scans[i]
            aa = np.ascontiguousarray(a, np.float32)
            oo = np.ascontiguousarray(o, np.float32)
            sz = np.ascontiguousarray(sizes, np.int32)
            ocv = np.ascontiguousarray(oc, np.int32)
            zp = torch.empty_like(zs[i])
            L.call("cbct_plain_osmom_solve", C.byref(pl.g), aa.ctypes.data, oo.ctypes.data, aa.size, sz.ctypes.data,
                   len(sz), ocv.ctypes.data, b.data_ptr(), zp.data_ptr(), it, 1, None)

        plain_solve(idx[0])   # warm-up
        plain_ms = [timed(lambda i=i: plain_solve(i)) for i in idx]
        ours_ms = [timed(lambda i=i: jobs[i]["plan"].osmom(jobs[i]["b"], jobs[i]["z"], None, it, nonneg=True,
                                                            use_graph=True)) for i in idx]
        ours_all = ms_s if ms_s is not None else sum(ours_ms) * len(jobs) / len(idx)
        est = ours_all * sum(plain_ms) / sum(ours_ms)
        plain = {"scans": idx, "ms_each": [round(t, 1) for t in plain_ms], "ours_ms_each": [round(t, 1) for t in ours_ms],
                 "ms_per_step_est": round(est, 1), "recon_per_s_est": round(len(jobs) * 1e3 / est, 3),
                 "speedup_batched_vs_plain": round(est / ms_b, 3),
                 "what": "reference structure re-hosted on B200 (texture filtering, per-call copies, host-synced "
                         "norms), timed on the sampled scans; all-scan time estimated by the sampled ratio"}
    n = len(jobs)
    leg = lambda ms, **kw: None if ms is None else dict(ms_per_step=round(ms, 1), recon_per_s=round(n * 1e3 / ms, 3),
                                                         gups=round(updates / (ms * 1e-3) / 1e9, 2), **kw)
    sset = SCAN_SETS[args.scan_sizes]
    line = {"metric": "batched recon/s (OS-MOM, uneven scans)", "value": round(n * 1e3 / ms_b, 3),
            "unit": "recon/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_b, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{n} uneven scans ({args.scan_sizes} set), OS-MOM 8 subsets x {it} iterations, "
                                   "fp32",
                       "scan_set": {k: v for k, v in sset.items()} if args.scan_sizes != "c4" else "c4 (seeds 1000+i)",
                       "executor": executor, "streams": args.streams, "sizes": "multiples of 8",
                       "autotune": bool(args.autotune), "variants": variants or None},
            "gups": round(updates / (ms_b * 1e-3) / 1e9, 2),
            "one_at_a_time": leg(ms_s),
            "stream_pool": leg(ms_p, what="one captured graph per scan, replayed on a pool of streams"),
            "fused": leg(ms_f, speedup_vs_stream_pool=round(ms_p / ms_f, 3) if ms_p and ms_f else None,
                         what="scans in two lockstep groups side by side: one persistent work-list launch per "
                              "projector kind and box width per subset step (scans that fill the GPU 16 waves keep "
                              "one-scan launches), one graph, replayed while the call repeats"),
            "speedup_batched_vs_one_at_a_time": round(ms_s / ms_b, 3) if ms_s else None, "plain_path": plain,
            "clocks": clk}
    return line


def mixed_precision(args):
    """Mixed-precision OS-MOM (the mixed-precision configuration): a 512^3
    phantom of 10 seeded ellipsoids plus 2000 small spheres (radius 0.5..2 mm,
    density up to 0.5/mm), 0.5 mm voxels (assumed), 720 views of 1024x768 at
    0.4 mm, Poisson noise at I0 = 5e4, 10 subsets x 20 iterations, positivity.
    Solved with fp32, bf16 and fp16 storage (16-bit: the measured projections
    and the forward projector's volume input; FP32 interpolation and
    accumulation, FP64 norms; the forward reads the FP32 image every 5th
    iteration).  Timed with CUDA events; the 16-bit results are compared with
    the fp32 result.  The per-iteration error against FP64 is measured on the
    same scene at a quarter of the resolution (128^3 at 2 mm, 180 views of
    256x192 at 1.6 mm), where the FP64 oracle finishes on the host: z after
    iteration k of the device solve (a k-iteration solve, the same
    computation prefix) against the oracle's z after iteration k."""
    import torch
    gtb = _package()
    L = gtb._lib
    dev = torch.device("cuda", 0)
    seed, iters, S = 4321, args.c3_iters, 10
    half = 128.0  # mm, half the volume
    ell = gtb.phantom.ellipsoids(seed, (2 * half,) * 3, n=10, n_spheres=2000)
    ell_d = torch.from_numpy(ell.reshape(-1)).to(dev)

    def problem(n, P, W, H, pitch, I0):
        g = L.CbctGeometry(1000.0, 1500.0, W * pitch, H * pitch, W, H, n, n, n, 2 * half, 2 * half, 2 * half, 1.5)
        ang = gtb.phantom.circular_orbit(P)
        order, sizes = gtb.subset_partition(P, S)
        a = ang[order].copy()
        o = np.zeros((P, 2), np.float32)
        plan = gtb.Plan(g, a, o, sizes, np.zeros(S, np.int32))
        exact = torch.empty(plan.proj_shape(), dtype=torch.float32, device=dev)
        plan.phantom_project(ell_d, exact)
        b = gtb.phantom.poisson_log(exact, I0, seed + 1).contiguous()
        return g, a, o, sizes, plan, b

    storages = [("fp32", torch.float32, L.CBCT_F32), ("bf16", torch.bfloat16, L.CBCT_BF16),
                ("fp16", torch.float16, L.CBCT_F16)]

    def solve(plan, b, dt, code, k, z):
        bt = b if dt == torch.float32 else b.to(dt).contiguous()
        plan.osmom(bt, z, None, k, nonneg=True, use_graph=True, storage=code, refine_every=5)

    # full size
    g, a, o, sizes, plan, b = problem(512, 720, 1024, 768, 0.4, 5e4)
    clocks = ClockSampler(0)
    clocks.start()
    results, times = {}, {}
    for name, dt, code in storages:
        z = torch.empty(plan.vol_shape, dtype=torch.float32, device=dev)
        solve(plan, b, dt, code, 1, z)          # warm-up: kernels, graph capture
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solve(plan, b, dt, code, iters, z)
        e1.record()
        e1.synchronize()
        times[name] = e0.elapsed_time(e1)
        results[name] = z.cpu()
    clk = clocks.stop()
    ref = results["fp32"].double()
    rel_vs_fp32 = {k: float((v.double() - ref).norm() / ref.norm()) for k, v in results.items() if k != "fp32"}
    n_upd = (iters + 1) * (1024 * 768 * 720 * int(np.float32(1.5) * np.float32(512)) + 512 ** 3 * 720)
    plan.close()
    del results, b
    torch.cuda.empty_cache()
    # quarter resolution against the FP64 oracle, per iteration
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    O.set_num_threads(os.cpu_count() or 1)
    g2, a2, o2, sizes2, plan2, b2 = problem(128, 180, 256, 192, 1.6, 5e4)
    og = O.Geometry(128, 128, 128, 2 * half, 2 * half, 2 * half, 256, 192, 256 * 1.6, 192 * 1.6, 1000.0, 1500.0)
    snaps = np.zeros((iters, 128, 128, 128), np.float64)
    t0 = time.perf_counter()
    O.osmom(og, b2.double().cpu().numpy(), a2, o2, sizes2, np.zeros(S, np.int32), iters=iters, nonneg=True,
            snapshots=snaps)
    oracle_s = time.perf_counter() - t0
    per_iter = {}
    for name, dt, code in storages:
        errs = []
        z = torch.empty(plan2.vol_shape, dtype=torch.float32, device=dev)
        for k in range(1, iters + 1):
            solve(plan2, b2, dt, code, k, z)
            ref_k = snaps[k - 1]
            errs.append(float(np.linalg.norm(z.cpu().numpy().astype(np.float64) - ref_k) / np.linalg.norm(ref_k)))
        per_iter[name] = [float(f"{e:.3e}") for e in errs]
    # the plain FP32 path (the reference's structure: texture weights, per-call copies) for context
    import ctypes as C
    errs = []
    bt2 = b2.contiguous()
    zp = torch.empty(plan2.vol_shape, dtype=torch.float32, device=dev)
    ap2, op2 = np.ascontiguousarray(a2, np.float32), np.ascontiguousarray(o2, np.float32)
    sz2, oc2 = np.ascontiguousarray(sizes2, np.int32), np.zeros(S, np.int32)
    for k in range(1, iters + 1):
        L.call("cbct_plain_osmom_solve", C.byref(g2), ap2.ctypes.data, op2.ctypes.data, ap2.size, sz2.ctypes.data, S,
               oc2.ctypes.data, bt2.data_ptr(), zp.data_ptr(), k, 1, None)
        ref_k = snaps[k - 1]
        errs.append(float(np.linalg.norm(zp.cpu().numpy().astype(np.float64) - ref_k) / np.linalg.norm(ref_k)))
    per_iter["plain_fp32_path"] = [float(f"{e:.3e}") for e in errs]
    ms = times["bf16"]
    line = {"metric": "mixed-precision OS-MOM recon/s (512^3, 720 views)", "value": round(1e3 / ms, 4),
            "unit": "recon/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": round(ms, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 storage, f32 compute",
            "data": "synthetic",
            "config": {"workload": "osmom 512^3 (0.5 mm, assumed) from 720 views 1024x768@0.4mm, I0=5e4, "
                                   f"10 ellipsoids + 2000 spheres, {S} subsets x {iters} iterations, positivity",
                       "storage": "projections and forward volume input 16-bit; FP32 forward every 5th iteration",
                       "assumed": ["voxel_mm", "SAD_mm", "SDD_mm"]},
            "ms_per_reconstruction": {k: round(v, 1) for k, v in times.items()},
            "gups": {k: round(n_upd / (v * 1e-3) / 1e9, 1) for k, v in times.items()},
            "rel_l2_vs_fp32_storage": {k: float(f"{v:.3e}") for k, v in rel_vs_fp32.items()},
            "per_iteration_rel_l2_vs_fp64_quarter_scale": per_iter,
            "fp64_oracle_seconds": round(oracle_s, 1), "clocks": clk}
    print(json.dumps(line), flush=True)


def _scan_host(gtb, sp, dev, I0=1e5):
    """One seeded scan of the batched shapes: geometry, acquisition-order
    angles/offsets and noisy log projections (pinned float32 host tensor)."""
    import torch
    L = gtb._lib
    nx, ny, nz = sp["n"]
    P, W, H, pitch = sp["P"], sp["W"], sp["H"], sp["pitch"]
    g = L.CbctGeometry(1000.0, 1500.0, W * pitch, H * pitch, W, H, nx, ny, nz, float(nx), float(ny), float(nz), 1.5)
    ang = gtb.phantom.circular_orbit(P)
    off = np.zeros((P, 2), np.float32)
    plan = gtb.Plan(g, ang, off)
    ell = torch.from_numpy(gtb.phantom.ellipsoids(sp["seed"], (nx, ny, nz)).reshape(-1)).to(dev)
    exact = torch.empty(plan.proj_shape(), dtype=torch.float32, device=dev)
    plan.phantom_project(ell, exact)
    b = gtb.phantom.poisson_log(exact, I0, sp["seed"] + 1)
    host = torch.empty(b.shape, dtype=torch.float32).pin_memory()
    host.copy_(b)
    plan.close()
    return g, ang, off, host


def served(args):
    print(json.dumps(served_line(args)), flush=True)


def served_line(args):
    """Serving loop (the served configuration): Poisson arrivals
    at --rate requests/s of FDK (70 %, Hann-windowed ramp) and OS-MOM (30 %,
    8 subsets x 10 iterations, positivity) reconstructions with the batched
    configuration's scan shapes (seeds 2000+i), projections stored as
    bfloat16 or float32 per request (seeded coin; arithmetic FP32), admitted
    against a --budget-gb HBM budget on --slots request slots.  Inputs are made on the device beforehand and held in pinned host
    memory; every request copies its projections in and its volume out.
    Latency = completion - submission on the host clock (a request is
    submitted at its arrival time).  The plain FP32 path then serves the same
    requests one at a time (host arrays in and out); its latencies follow from
    its measured service times and the same arrival times, first in first out."""
    import ctypes as C
    import torch
    gtb = _package()
    L = gtb._lib
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(args.seed))
    n = args.requests
    specs = gtb.phantom.uneven_scans(n, seed0=2000)
    kinds = ["fdk" if u < 0.7 else "osmom" for u in rng.random(n)]
    use_bf16 = rng.random(n) < 0.5
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, n))
    arrivals -= arrivals[0]

    def make_request(i, proj, vol):
        g, ang, off = inputs[i][:3]
        if kinds[i] == "fdk":
            return gtb.Server.fdk_request(g, ang, off, proj, vol, filt=gtb.hann_ramp_filter(g.width))
        return gtb.Server.osmom_request(g, ang, off, proj, vol, 8, iterations=10, nonneg=True, use_graph=True)

    inputs, reqs, vols = [], [], []
    for i, sp in enumerate(specs):
        g, ang, off, p32 = _scan_host(gtb, sp, dev)
        proj = p32.to(torch.bfloat16).pin_memory() if use_bf16[i] else p32
        inputs.append((g, ang, off, proj))
        vols.append(torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32).pin_memory())
        reqs.append(make_request(i, proj, vols[i]))
    h2d = sum(x[3].numel() * x[3].element_size() for x in inputs)
    d2h = sum(v.numel() * 4 for v in vols)
    torch.cuda.synchronize()
    srv = gtb.Server(args.budget_gb * 1e9, args.slots)
    # Warm-up (untimed): one request of each kind and storage loads every kernel.
    for i in [kinds.index(k) for k in ("fdk", "osmom") if k in kinds]:
        for dt in (torch.float32, torch.bfloat16):
            p = inputs[i][3].to(dt).pin_memory()
            srv.wait(srv.submit(make_request(i, p, torch.empty_like(vols[i]).pin_memory())))
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    tickets = []
    for i in range(n):
        delay = arrivals[i] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        tickets.append(srv.submit(reqs[i]))
    recs = [srv.wait(t) for t in tickets]
    clk = clocks.stop()
    lat = np.array([r["t_done"] - r["t_submit"] for r in recs])
    span = max(r["t_done"] for r in recs) - min(r["t_submit"] for r in recs)
    peak_inflight = max(sum(1 for r in recs if r["t_admit"] <= q["t_admit"] < r["t_done"]) for q in recs)
    # bfloat16 storage against float32 storage of the same requests
    storage_effect = {}
    for k in ("fdk", "osmom"):
        i = next((j for j in range(n) if kinds[j] == k and use_bf16[j]), None)
        if i is None:
            continue
        p32 = _scan_host(gtb, specs[i], dev)[3]
        v32 = torch.empty_like(vols[i]).pin_memory()
        srv.wait(srv.submit(make_request(i, p32, v32)))
        storage_effect[k] = float((vols[i] - v32).double().norm() / v32.double().norm())
    srv.close()
    # The plain FP32 path, one request at a time, on the same requests.
    service, plain_err = [], {}
    n_plain = n if not args.no_plain else 0
    for i in range(n_plain):
        g, ang, off = inputs[i][:3]
        p32 = _scan_host(gtb, specs[i], dev)[3]
        out = torch.empty_like(vols[i]).pin_memory()
        a = np.ascontiguousarray(ang - ang.min(), np.float32)
        o = np.ascontiguousarray(off, np.float32)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if kinds[i] == "fdk":
            f = gtb.hann_ramp_filter(g.width).astype(np.float32)
            oc = int(gtb.operators.offset_override(g, off))
            L.call("cbct_plain_fdk", C.byref(g), a.ctypes.data, o.ctypes.data, a.size, p32.data_ptr(),
                   out.data_ptr(), f.ctypes.data, oc, 20)
        else:
            order, sizes = gtb.subset_partition(a.size, 8)
            ap, op = np.ascontiguousarray(a[order]), np.ascontiguousarray(o[order])
            first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
            oc = np.array([int(gtb.operators.offset_override(g, op[f:f + s])) if s else 0
                           for f, s in zip(first, sizes)], np.int32)
            b = p32[torch.from_numpy(order.astype(np.int64))].to(dev)
            z = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device=dev)
            L.call("cbct_plain_osmom_solve", C.byref(g), ap.ctypes.data, op.ctypes.data, a.size,
                   sizes.astype(np.int32).ctypes.data, 8, oc.ctypes.data, b.data_ptr(), z.data_ptr(), 10, 1, None)
            out.copy_(z)
        torch.cuda.synchronize()
        service.append(time.perf_counter() - t1)
        if kinds[i] not in plain_err and not use_bf16[i]:
            plain_err[kinds[i]] = float((vols[i] - out).double().norm() / out.double().norm())
    line = {"metric": "served recon/s (Poisson arrivals, 70% FDK / 30% OS-MOM)", "value": round(n / span, 3),
            "unit": "recon/s", "n_gpus": 1, "steps": 1, "warmup": 4, "ms_per_step": round(span * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/bf16 storage, f32 compute",
            "data": "synthetic",
            "config": {"workload": f"{n} requests at {args.rate}/s, sizes of the batched configuration (seeds 2000+i)",
                       "fdk": int(sum(k == "fdk" for k in kinds)), "osmom": int(sum(k == "osmom" for k in kinds)),
                       "bf16_requests": int(use_bf16.sum()), "slots": args.slots, "budget_gb": args.budget_gb,
                       "osmom": "8 subsets x 10 iterations, positivity, CUDA graph; bf16 = projections stored bf16",
                       "fdk_filter": "Hann-windowed ramp", "latency": "host clock, completion - arrival"},
            "latency_p50_s": round(float(np.percentile(lat, 50)), 3),
            "latency_p99_s": round(float(np.percentile(lat, 99)), 3),
            "peak_requests_in_flight": int(peak_inflight),
            "e2e": {"value": round(n / span, 3), "unit": "recon/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "storage_bf16_vs_f32_rel_l2": {k: round(v, 6) for k, v in storage_effect.items()},
            "clocks": clk}
    if service:
        done, plain_lat = 0.0, []
        for arr, s in zip(arrivals, service):
            done = max(arr, done) + s
            plain_lat.append(done - arr)
        line["plain_path"] = {"recon_per_s": round(n / (done - arrivals[0]), 3),
                              "latency_p50_s": round(float(np.percentile(plain_lat, 50)), 3),
                              "latency_p99_s": round(float(np.percentile(plain_lat, 99)), 3),
                              "service_s_total": round(float(sum(service)), 2),
                              "served_vs_plain_rel_l2": {k: round(v, 6) for k, v in plain_err.items()}}
        line["speedup_vs_plain"] = round((n / span) / line["plain_path"]["recon_per_s"], 3)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c2", "c1", "c3", "c4", "c5"])
    ap.add_argument("--scans", type=int, default=64, help="c4: number of scans")
    ap.add_argument("--streams", type=int, default=8, help="c4: streams of the batch executor")
    ap.add_argument("--scan-sizes", choices=list(SCAN_SETS), default="c4",
                    help="c4: scan set (c4: the configuration's sizes; small/medium/tiny: smaller scans)")
    ap.add_argument("--executor", choices=["both", "fused", "pool"], default="both",
                    help="c4: batch executor(s) to time (one of them: no one-at-a-time leg)")
    ap.add_argument("--iterations", type=int, default=10, help="c4: OS-MOM iterations")
    ap.add_argument("--requests", type=int, default=32, help="c5: requests in the arrival stream")
    ap.add_argument("--c3-iters", type=int, default=20, help="c3: OS-MOM iterations")
    ap.add_argument("--autotune", action="store_true", help="c4: autotune each scan's projector variants")
    ap.add_argument("--plain-sample", type=int, default=8,
                    help="c4: scans also solved by the plain path (0: none)")
    ap.add_argument("--rate", type=float, default=20.0, help="c5: Poisson arrival rate, requests/s")
    ap.add_argument("--slots", type=int, default=4, help="c5: request slots of the server")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="c5: HBM budget of the server")
    ap.add_argument("--seed", type=int, default=5, help="c5: seed of kinds, storage and arrivals")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path comparison leg")
    ap.add_argument("--no-legs", action="store_true",
                    help="c2: skip the reduced serving and batching legs of the default line")
    ap.add_argument("--forward-kernel", choices=list(FORWARD_KERNELS), default="auto",
                    help="c1/c2: forward projector variant of the plan (auto: the plan's choice)")
    ap.add_argument("--only", choices=["forward", "backproject", "fdk", "tv"], default=None,
                    help="time one kernel of the workload (profiling)")
    args = ap.parse_args()
    if args.config == "c4":
        batched(args)
        return
    if args.config == "c5":
        served(args)
        return
    if args.config == "c3":
        mixed_precision(args)
        return
    wl = Workload(args.config)
    if args.only:
        kernel_only(args, wl)
        return
    if args.impl == "reference":
        reference_arm(args, wl)
    else:
        ours(args, wl)


if __name__ == "__main__":
    main()

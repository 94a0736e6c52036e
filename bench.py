#!/usr/bin/env python
"""Benchmark of the nonlocal LBM acoustics step (node updates per second).

Workload (default): the 3-D D3Q27 single scene -- 63^3 = 250,047 points in
the unit cube (regular grid jittered by U(-h/4, h/4), seed 1), k = 32,
8-layer PML, Gaussian pulse (1e-3, width 0.05), dt = 0.5 h / c, 8 probes --
stepped on one GPU. Also measured: the batched form (256 D2Q9 scenes of
2k-100k nodes, one launch per kernel for all scenes, CUDA graph) against the
plain single-scene D2Q9 step of 20,164 nodes.

One "step" = one time step of the scene(s). `value` = node updates per
second of the whole job (all ranks), inputs resident in HBM; the scene
state (~1.4 KB/node, ~350 MB) exceeds the 126 MB L2, so no flush is needed.
`e2e` = the same metric through the public API with host buffers: the
initial state is uploaded from host memory and every step's probe samples
are read back, as NAGA's density observer does each step.

--impl reference times the reference's algorithm on the host CPU: the CPU
oracle (a restatement of NAGA's step; NAGA has no CPU path of its own and
its GPU runtime cannot be built) in NAGA's own FP32 arithmetic.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PROBES3 = [[x, y, z] for z in (0.35, 0.65) for y in (0.35, 0.65) for x in (0.35, 0.65)]
PROBES2 = [[0.3, 0.5], [0.7, 0.5], [0.5, 0.3], [0.5, 0.7]]
CONFIG3 = dict(dim=3, n_side=63, layers=8, seed=1, k=32, shape=0, width=0.05, probes=PROBES3)
CONFIG2 = dict(dim=2, n_side=142, layers=10, seed=0, k=16, shape=1, width=0.05, probes=PROBES2)


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ------------------------------------------------------------ scenes
def make_scene(naga, cfg, seed=None, width=None, center=None):
    g = naga.generate_grid(cfg["dim"], cfg["n_side"], cfg["layers"],
                           cfg["seed"] if seed is None else seed)
    s = naga.Scene(g, k=cfg["k"], shape=cfg["shape"], probes=np.array(cfg["probes"], np.float32),
                   probe_capacity=8192)
    c = center if center is not None else [0.5] * cfg["dim"]
    drho = naga.gaussian_pulse(g["points"], c, 1e-3, cfg["width"] if width is None else width)
    s.set_density(drho)
    return s, g, drho


def batched_scenes(naga, n_scenes=256, lo=2e3, hi=1e5):
    """256 D2Q9 scenes, point counts log-uniform in [2k, 100k], seeds 100..355,
    pulse width U(0.03, 0.08), pulse centre U(0.3, 0.7)^2 per scene."""
    out = []
    for t in range(n_scenes):
        rng = np.random.default_rng(100 + t)
        n = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        n_side = max(24, int(round(np.sqrt(n))))
        cfg = dict(CONFIG2, n_side=n_side, seed=100 + t)
        s, g, _ = make_scene(naga, cfg, width=float(rng.uniform(0.03, 0.08)),
                             center=list(rng.uniform(0.3, 0.7, 2)))
        out.append(s)
    return out


# ------------------------------------------------------- algorithmic bytes
def kernel_bytes(dim, N, nb, nl, nbd, k, kb):
    """Compulsory HBM bytes per launch of each step kernel (FP32 values, u32
    indices; rows of Q populations; neighbour rows counted once)."""
    Q = 9 if dim == 2 else 27
    row = 4 * Q
    st = 4 * k * (dim + 1)  # weights + index per neighbour
    nbl = nb + nl
    return {
        # G, Q1_prev in; Q1, S1 out (+ S1P on sources, not counted); M in/out;
        # the PML field rows of the layer out
        "macro_pml": N * (4 * row + 32) + nl * row,
        # stencil + S1 read/write + PV per node, the layer's field rows once
        "pml_gather": nbl * (st + 2 * row + 32) + nl * row,
        "edge_collide": nbd * (2 * row + 8 * kb),
        "filter": N * 2 * row + nbl * 8 * k,
        "rk_stage1": nbl * (st + 3 * row),
        "rk_stage2": nbl * (st + 5 * row),
        "rk_stage3": nbl * (st + 5 * row),
        "rk_stage4": nbl * (st + 4 * row),
        "edge_interp": nbd * (8 * kb + row),
    }


# ------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# ------------------------------------------------------------- timing
def time_steps(torch, step_fn, stream_ptr, warmup, steps):
    """Warm-up, then `steps` single steps bracketed by events on the stream
    the step runs on; returns (total ms, per-step ms list)."""
    st = torch.cuda.ExternalStream(stream_ptr)
    for _ in range(warmup):
        step_fn()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(st)
    for t in range(steps):
        step_fn()
        evs[t + 1].record(st)
    torch.cuda.synchronize()
    per = [evs[t].elapsed_time(evs[t + 1]) for t in range(steps)]
    return evs[0].elapsed_time(evs[-1]), per


def profile_kernels(naga, step_fn, steps=5):
    with naga.profile() as p:
        for _ in range(steps):
            step_fn()
    return p.result


def cpu_baseline(cfg, max_seconds=20.0):
    """The oracle in NAGA's FP32 arithmetic on all host threads: set-up is
    not timed; steps are timed until max_seconds (at least one)."""
    from oracle import oracle
    import naga_b200 as naga

    arch = os.environ.get("NAGA_ORACLE_ARCH", "-march=native")
    path = os.path.join(ROOT, "oracle", "_native", "libnaga_oracle.so")
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        oracle.build(arch_flags=arch, out=path)
        L = oracle.lib(path)
    except Exception:
        L, arch = oracle.lib(), ""
    oracle._lib = L
    g = naga.generate_grid(cfg["dim"], cfg["n_side"], cfg["layers"], cfg["seed"])
    S = oracle.Scene(cfg["dim"], g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"],
                     g["normals"], g["sigma"], g["h"], k=cfg["k"], shape=cfg["shape"], precision=1,
                     probes=np.array(cfg["probes"], np.float32))
    S.set_density(naga.gaussian_pulse(g["points"], [0.5] * cfg["dim"], 1e-3, cfg["width"]))
    n, t0 = 0, time.perf_counter()
    while True:
        S.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el > max_seconds or n >= 50:
            break
    N = g["points"].shape[0]
    return {"value": N * n / el / 1e6, "unit": "MNUPS", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n} time steps of the {N:,}-node scene (set-up excluded), FP32 as NAGA, "
                      f"OpenMP, {arch or 'generic x86-64'}"}


# ------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    cfg = CONFIG3
    if rank != 0:
        return 0
    cb = cpu_baseline(cfg, max_seconds=max(5.0, 4.0 * args.steps / 100.0))
    v = cb["value"]
    line = {"metric": "MNUPS (node updates/s) of the nonlocal LBM acoustics step", "value": v,
            "unit": "MNUPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "D3Q27 single scene, 250,047 jittered nodes, k=32, 8-layer PML"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "MNUPS", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_naga(args, rank, world, local_rank):
    import torch

    import naga_b200 as naga

    global CONFIG3
    if args.n_side != CONFIG3["n_side"]:
        CONFIG3 = dict(CONFIG3, n_side=args.n_side)
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    cfg = CONFIG3
    scene, g, drho = make_scene(naga, cfg)
    N = scene.N
    K, W = args.steps, args.warmup

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput (value) and per-step latency
    barrier()
    with ClockSampler(local_rank) as clk:
        total_ms, per = time_steps(torch, lambda: scene.step(1), scene.stream, W, K)
    barrier()
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * N * K / (total_ms * 1e-3) / 1e6

    # ---- end to end through the public API with host buffers: the initial
    # density goes up from page-locked host memory, and every step's probe
    # samples come back (the observer read of each step, queued behind the
    # step so the device never waits for the host)
    host_drho = torch.empty(N, dtype=torch.float32, pin_memory=True).numpy()
    host_drho[:] = drho
    np_ = len(cfg["probes"])
    host_probes = torch.empty((K, np_), dtype=torch.float32, pin_memory=True)
    barrier()
    t0 = time.perf_counter()
    scene.set_density(host_drho)
    for t in range(K):
        scene.step(1)
        scene.probes_async(t, 1, host_probes.data_ptr() + 4 * np_ * t)
    scene.sync()
    e2e_s = time.perf_counter() - t0
    e2e_trace_ok = bool(np.array_equal(host_probes.numpy(), scene.probes(0, K)))
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * N * K / e2e_s / 1e6

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- per-kernel timing (CUDA events around each launch, separate run)
    prof = profile_kernels(naga, lambda: scene.step(1), steps=5)
    kb = kernel_bytes(3, N, g["n_bulk"], g["n_layer"], g["n_boundary"], cfg["k"], cfg["k"])
    step_ms = sum(ms for (_, ms) in prof.values()) / 5
    top = max(kb, key=lambda n: prof.get(n, (0, 0.0))[1])
    launches, tot = prof[top]
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = kb[top] / (tot / launches * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(top)
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": "measured" if peaks else "fallback",
            "algorithmic_bytes_per_launch": kb[top], "avg_launch_ms": tot / launches,
            "kernel_share": {n: round(prof[n][1] / 5 / step_ms, 4) for n in prof if prof[n][0]}}
    gpu_launches = sum(l for (l, _) in prof.values()) // 5 * K

    # ---- batched form vs plain single scene (D2Q9)
    batched = None
    if not args.no_batched:
        plain2, g2, _ = make_scene(naga, CONFIG2)
        p_ms, _ = time_steps(torch, lambda: plain2.step(1), plain2.stream, W, K)
        plain_mnups = plain2.N * K / (p_ms * 1e-3) / 1e6
        scenes = batched_scenes(naga, args.batched_scenes)
        b = naga.Batch(2)
        for s in scenes:
            b.add(s)
        nodes = sum(s.N for s in scenes)
        b_ms, b_per = time_steps(torch, lambda: b.step(1), b.stream, W, K)
        bm = nodes * K / (b_ms * 1e-3) / 1e6
        batched = {"scenes": len(scenes), "nodes": nodes, "mnups": bm,
                   "plain_2d_mnups": plain_mnups, "ratio_vs_plain": bm / plain_mnups,
                   "p50_step_ms": float(np.percentile(b_per, 50)),
                   "p99_step_ms": float(np.percentile(b_per, 99))}
        b.close()
        for s in scenes:
            s.close()
        plain2.close()

    cb = None
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(cfg, max_seconds=15.0)

    line = {
        "metric": "MNUPS (node updates/s) of the nonlocal LBM acoustics step",
        "value": value, "unit": "MNUPS", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "D3Q27 single scene, 250,047 jittered nodes (63^3, seed 1), k=32, "
                               "MQ RBF, 8-layer PML, FP32 populations, FP64 weight solves",
                   "nodes": N, "l2": "working set ~350 MB > 126 MB L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "p50_step_ms": float(np.percentile(per, 50)), "p99_step_ms": float(np.percentile(per, 99)),
        "roofline": roof, "cpu_baseline": cb,
        "e2e": {"value": e2e, "unit": "MNUPS", "h2d_bytes_per_step": int(N * 4 / K),
                "d2h_bytes_per_step": 4 * len(cfg["probes"]), "probe_trace_read_back": e2e_trace_ok},
        "gpu_launches": int(gpu_launches), "clocks": clk.summary(), "batched": batched,
        "launch_shapes": naga.tuning_report().strip().splitlines(),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="naga", choices=["naga", "reference"])
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched-scenes", type=int, default=256)
    ap.add_argument("--n-side", type=int, default=63,
                    help="grid nodes per side of the 3-D scene (63 = the benchmark workload; "
                         "smaller values give profiling cases)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_naga(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())

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


def batched_specs(n_scenes=256, lo=2e3, hi=1e5):
    """The batched 2-D workload: n_scenes D2Q9 scenes, point counts
    log-uniform in [2k, 100k] (jittered grids, seeds 100..), pulse width
    U(0.03, 0.08) and centre U(0.3, 0.7)^2 per scene. Returns per scene
    (grid side, seed, width, centre)."""
    out = []
    for t in range(n_scenes):
        rng = np.random.default_rng(100 + t)
        n = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        n_side = max(24, int(round(np.sqrt(n))))
        out.append((n_side, 100 + t, float(rng.uniform(0.03, 0.08)), list(rng.uniform(0.3, 0.7, 2))))
    return out


def build_batched(naga, specs):
    out = []
    for n_side, seed, width, center in specs:
        s, _, _ = make_scene(naga, dict(CONFIG2, n_side=n_side, seed=seed), width=width, center=center)
        out.append(s)
    return out


# ------------------------------------------------------- algorithmic bytes
def pml_counts(naga, scene):
    """(nodes the PML gather visits, layer-support records they hold): a
    bulk or layer node is visited when a stencil support lies in the
    absorbing layer, and its tile holds those supports' records."""
    import ctypes as C

    d = scene.desc
    nbl = d.n_bulk + d.n_layer
    idx = np.zeros((scene.N, d.k), np.uint32)
    naga._check(naga.lib().naga_scene_read_tables(scene.h, idx.ctypes.data_as(C.c_void_p), *([None] * 6)))
    sup = idx[:nbl]
    cnt = ((sup >= d.n_bulk) & (sup < nbl)).sum(1)
    return int((cnt > 0).sum()), int(cnt.sum())


def kernel_bytes(dim, N, nb, nl, nbd, k, kb, pml=None):
    """Compulsory HBM bytes per launch of each step kernel (FP32 values, u32
    indices; rows of Q populations; neighbour rows counted once). The RK
    stages and the PML gather touch only the populations with a streaming
    rate: all 27 in D3Q27, the 8 moving ones of D2Q9 (its rest population's
    rate is zero)."""
    Q = 9 if dim == 2 else 27
    row = 4 * Q
    grow = 4 * 8 if dim == 2 else row  # the gathered part of a row
    st = 4 * k * (dim + 1)  # weights + index per neighbour
    nbl = nb + nl
    return {
        # G, Q1_prev in; Q1, S1 out (+ S1P on sources, not counted); M in/out;
        # the PML field rows of the layer out
        "macro_pml": N * (4 * row + 32) + nl * grow,
        # per visited node its layer supports' records (16 B), S1 read and
        # write, PV; the layer's field rows once (pml = (visited nodes,
        # records), from pml_counts; without it every fluid node and its
        # whole stencil, an upper bound)
        "pml_gather": ((pml[1] * 16 + pml[0] * (2 * grow + 32)) if pml else nbl * (st + 2 * grow + 32)) + nl * grow,
        "edge_collide": nbd * (2 * row + 8 * kb),
        "filter": N * 2 * row + nbl * 8 * k,
        # Horner RK4: stencil, the stage rows gathered (counted once), the
        # node's own start row in, the stage row out
        "rk_stage1": nbl * (st + 2 * grow),
        "rk_stage2": nbl * (st + 3 * grow),
        "rk_stage3": nbl * (st + 3 * grow),
        "rk_stage4": nbl * (st + 3 * grow),
        "edge_interp": nbd * (8 * kb + row),
    }


def gather_bytes(nb, nl, nbd, k, kb, pml):
    """Bytes the neighbour-row loads of each D3Q27 gather kernel move into the
    SMs per launch: one 112-B row per (node, stencil support) reference --
    from L2 in the L2-form kernels, from shared memory in the halo RK stages
    (whose L2 traffic is each pass's distinct rows once). Beside the DRAM
    fraction it shows the load the gather path carries: a kernel low on the
    HBM roofline may still move several times the HBM bandwidth in rows."""
    row = 4 * 28
    nbl = nb + nl
    rk = nbl * k * row
    return {"pml_gather": pml[1] * row, "edge_collide": nbd * kb * row, "filter": nbl * k * row,
            "rk_stage1": rk, "rk_stage2": rk, "rk_stage3": rk, "rk_stage4": rk, "edge_interp": nbd * kb * row}


RK_STAGES = ("rk_stage1", "rk_stage2", "rk_stage3", "rk_stage4")


def dominant_kernel(kb, prof):
    """The step kernel with the largest share of the step time, over the
    kernels with algorithmic bytes (kb) and launches (prof: name -> (launches,
    total ms)). The four RK stages are one kernel -- one template launched
    four times a step -- named "rk_stage1..4"; every other step kernel is
    its own. Returns (name, bytes per launch, mean launch ms, launch names)."""
    fam = {}
    for n in kb:
        if prof.get(n, (0, 0.0))[0]:
            fam.setdefault("rk_stage1..4" if n in RK_STAGES else n, []).append(n)
    top = max(fam, key=lambda f: sum(prof[n][1] for n in fam[f]))
    members = fam[top]
    launches = sum(prof[n][0] for n in members)
    per_launch = sum(kb[n] * prof[n][0] for n in members) / launches
    return top, per_launch, sum(prof[n][1] for n in members) / launches, members


def batch_roofline(naga, scenes, prof, peak):
    """Roofline of the batch's longest step kernel: its algorithmic bytes
    summed over the member scenes per launch, over its mean launch time."""
    tot = {}
    for sc in scenes:
        d = sc.desc
        for name, b in kernel_bytes(sc.dim, sc.N, d.n_bulk, d.n_layer, d.n_boundary, d.k, d.k_boundary,
                                    pml_counts(naga, sc)).items():
            tot[name] = tot.get(name, 0) + b
    top, per_launch, avg_ms, _ = dominant_kernel(tot, prof)
    achieved = per_launch / (avg_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": avg_ms,
            "kernel_fracs": {n: round(tot[n] / (prof[n][1] / prof[n][0] * 1e-3) / 1e9 / peak, 3)
                             for n in tot if prof.get(n, (0, 0.0))[0]}}


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


def headline_config(n_nodes, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": "D3Q27 single scene, 250,047 jittered nodes (63^3, seed 1), k=32, "
                        "MQ RBF, 8-layer PML, FP32 populations, FP64 weight solves",
            "nodes": n_nodes, "l2": "working set ~350 MB > 126 MB L2, no flush",
            "parallelism": f"replicas x{world}"}


def physical_cores() -> int:
    """Physical cores of this host (distinct (core, socket) pairs of lscpu),
    else the logical CPU count."""
    try:
        out = subprocess.run(["lscpu", "-p=CORE,SOCKET"], capture_output=True, text=True,
                             timeout=10).stdout
        pairs = {ln for ln in out.splitlines() if ln and not ln.startswith("#")}
        if pairs:
            return len(pairs)
    except (OSError, subprocess.SubprocessError):
        pass
    return os.cpu_count() or 1


def cpu_scene(cfg):
    """The oracle in NAGA's FP32 arithmetic on the workload's scene. The grid
    and the pulse come from the oracle's own generator (bit-identical to the
    library's, tests/test_oracle.py), so this leg never loads libnaga_b200."""
    from oracle import oracle

    arch = os.environ.get("NAGA_ORACLE_ARCH", "-march=native")
    path = os.path.join(ROOT, "oracle", "_native", "libnaga_oracle.so")
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        oracle.build(arch_flags=arch, out=path)
        L = oracle.lib(path)
    except Exception:
        L, arch = oracle.lib(), ""
    oracle._lib = L
    g = oracle.generate_grid(cfg["dim"], cfg["n_side"], cfg["layers"], cfg["seed"])
    S = oracle.Scene(cfg["dim"], g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"],
                     g["normals"], g["sigma"], g["h"], k=cfg["k"], shape=cfg["shape"], precision=1,
                     probes=np.array(cfg["probes"], np.float32))
    S.set_density(oracle.gaussian_pulse(g["points"], [0.5] * cfg["dim"], 1e-3, cfg["width"]))
    return oracle, S, g["points"].shape[0], arch


def cpu_baseline(cfg, steps=None, warmup=1, max_seconds=15.0, one_thread_steps=2):
    """The CPU leg: the oracle in NAGA's FP32 arithmetic, set-up untimed.
    With `steps`, exactly that many steps are timed after `warmup` untimed
    ones on all host threads; otherwise steps are timed until max_seconds.
    Then `one_thread_steps` steps on one thread (0 skips them)."""
    oracle, S, N, arch = cpu_scene(cfg)
    threads = oracle.set_threads(os.cpu_count() or 1)
    for _ in range(warmup):
        S.step(1)
    n, t0 = 0, time.perf_counter()
    while True:
        S.step(1)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or (steps is None and (el > max_seconds or n >= 50)):
            break
    out = {"value": N * n / el / 1e6, "unit": "MNUPS", "cores": threads, "kind": "port",
           "physical_cores": physical_cores(), "ms_per_step": el / n * 1e3, "nodes": N,
           "sample": f"{n} time steps of the {N:,}-node scene after {warmup} untimed (set-up "
                     f"excluded), FP32 as NAGA, OpenMP on {threads} threads, {arch or 'generic x86-64'}"}
    if one_thread_steps:
        oracle.set_threads(1)
        t0 = time.perf_counter()
        S.step(one_thread_steps)
        el1 = time.perf_counter() - t0
        oracle.set_threads(threads)
        out["one_thread"] = {"value": N * one_thread_steps / el1 / 1e6, "unit": "MNUPS",
                             "ms_per_step": el1 / one_thread_steps * 1e3,
                             "sample": f"{one_thread_steps} further steps of the same scene on 1 thread"}
    return out


def probe_error_block(scene, g, drho):
    """Probe error of the benchmarked scene: the scene restarts from its
    initial pulse, takes the fixture's steps (1000) and its probe trace is
    compared with the FP64 oracle's trace of the same scene
    (tests/golden/trace_d3q27_63.npz; the input digest must match):
    max_t |p_gpu - p_oracle| / max_t |p_oracle| over all probes."""
    path = os.path.join(ROOT, "tests", "golden", "trace_d3q27_63.npz")
    if not os.path.exists(path):
        return {"value": None, "reason": "fixture missing"}
    from tests.golden.make_config2_trace import scene_hash

    fx = np.load(path)
    if scene_hash(g, drho) != str(fx["sha256"]):
        return {"value": None, "reason": "scene differs from the fixture's"}
    ref = fx["probes"]
    scene.set_density(drho)
    scene.step(len(ref))
    got = scene.probes(0, len(ref)).astype(np.float64)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    return {"value": err, "steps": int(len(ref)), "bar": 1e-5, "ok": err <= 1e-5,
            "against": "FP64 CPU oracle trace of the same scene (tests/golden/trace_d3q27_63.npz)"}


def measured_hbm_peak():
    """(GB/s, source): MEASURED_PEAKS.json's copy bandwidth, else the pool's
    earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------ extra blocks
def batched_block(naga, torch, args, rank, world, dist, W, K):
    """256 D2Q9 scenes stepped as one batch (one launch per kernel, CUDA
    graph), sharded over the ranks by size, against the plain 20,164-node
    D2Q9 scene stepped alone (one replica per rank)."""
    from naga_b200 import replicas

    plain2, _, _ = make_scene(naga, CONFIG2)
    p_ms, _ = time_steps(torch, lambda: plain2.step(1), plain2.stream, W, K)
    p_ms = replicas.max_over_ranks(p_ms, dist, "cuda")
    plain_mnups = world * plain2.N * K / (p_ms * 1e-3) / 1e6
    plain2.close()
    specs = batched_specs(args.batched_scenes)
    mine = replicas.shard([sp[0] ** 2 for sp in specs], rank, world)
    scenes = build_batched(naga, [specs[i] for i in mine])
    b = naga.Batch(2)
    for s in scenes:
        b.add(s)
    b.prepare()
    b_ms, b_per = time_steps(torch, lambda: b.step(1), b.stream, W, K)
    b_ms = replicas.max_over_ranks(b_ms, dist, "cuda")
    nodes = int(replicas.sum_over_ranks(sum(s.N for s in scenes), dist, "cuda"))
    p99 = replicas.max_over_ranks(float(np.percentile(b_per, 99)), dist, "cuda")
    bm = nodes * K / (b_ms * 1e-3) / 1e6
    # per-kernel device time of this rank's batch step (event-bracketed
    # launches, after the timed region) and the roofline of its top kernel
    prof = profile_kernels(naga, lambda: b.step(1))
    roof = batch_roofline(naga, scenes, prof, measured_hbm_peak()[0])
    b.close()
    for s in scenes:
        s.close()
    return {"scenes": len(specs), "nodes": nodes, "mnups": bm, "plain_2d_mnups": plain_mnups,
            "ratio_vs_plain": bm / plain_mnups, "p50_step_ms": float(np.percentile(b_per, 50)),
            "p99_step_ms": p99, "sharding": f"{world} rank(s), size-balanced",
            "kernel_ms_rank0": {n: round(t / 5, 4) for n, (l, t) in prof.items() if l},
            "roofline_rank0": roof}


def serving_block(naga, torch, args, rank, world, dist, step_priority=0, target_step_ms=0.0, seconds=None):
    """The continuous-batching loop on the 3-D serving workload, for a
    bounded window: requests arrive as a Poisson process (20/s, seeded) with
    point counts log-uniform in [1e4, 1e6] (jittered unit cubes seeded per
    request), 2000 steps each, FP64 weight solves, admitted under a 150 GB
    device budget and, with target_step_ms > 0, a per-step latency target of
    the batch; each rank serves the requests the deterministic router gives
    it. Requests still running at the end of the window count by the steps
    they took. step_priority 1 runs the batch's steps ahead of the set-up
    kernels of admissions."""
    from naga_b200 import replicas

    rng = np.random.default_rng(2024)
    T = args.serving_seconds if seconds is None else seconds
    arrivals, t = [], 0.0
    while True:
        t += float(rng.exponential(1 / 20.0))
        if t >= T:
            break
        n = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        arrivals.append((t, max(16, int(round(n ** (1 / 3)))), len(arrivals)))
    router = replicas.Router(world)
    owner = [router.place(n_side ** 3, 2000) for (_, n_side, _) in arrivals]
    mine = [a for a, o in zip(arrivals, owner) if o == rank]
    server = naga.Server(3, memory_budget=150 * 10 ** 9, steps_per_tick=20, step_priority=step_priority,
                         target_step_ms=target_step_ms)
    probes = np.array(PROBES3, np.float32)
    # the clients: a producer thread builds each request's point cloud and
    # pulse in arrival order (the generator releases the GIL), the loop
    # submits what has arrived and ticks
    import queue

    ready: queue.Queue = queue.Queue()
    stop = threading.Event()

    def produce():
        for at, n_side, seed in mine:
            if stop.is_set():
                return
            g = naga.generate_grid(3, n_side, max(2, n_side // 8), 1000 + seed)
            ready.put((at, g, naga.gaussian_pulse(g["points"], [0.5] * 3, 1e-3, 0.05)))

    producer = threading.Thread(target=produce, daemon=True)
    submitted, pending = 0, None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    producer.start()
    while True:
        el = time.perf_counter() - t0
        if el >= T:
            break
        while True:
            if pending is None:
                try:
                    pending = ready.get_nowait()
                except queue.Empty:
                    break
            if pending[0] > el:
                break
            _, g, drho = pending
            server.submit(g, drho, 2000, k=32, shape=0, probes=probes, probe_capacity=2048)
            submitted += 1
            pending = None
        server.tick()
    stop.set()
    torch.cuda.synchronize()
    st = server.stats()
    server.close()
    node_updates = replicas.sum_over_ranks(st["node_updates"], dist, "cuda")
    busy = replicas.max_over_ranks(st["busy_ms"], dist, "cuda")
    done = int(replicas.sum_over_ranks(st["done"], dist, "cuda"))
    return {"window_s": T, "target_step_ms": target_step_ms, "step_priority": step_priority,
            "arrivals": len(arrivals), "submitted_rank0": submitted,
            "node_updates": int(node_updates), "mnups_busy": node_updates / max(busy, 1e-9) / 1e3,
            "mnups_wall": node_updates / T / 1e6,
            "p50_step_ms": replicas.max_over_ranks(st["p50_step_ms"], dist, "cuda"),
            "p99_step_ms": replicas.max_over_ranks(st["p99_step_ms"], dist, "cuda"),
            "step_latency": "per-step CUDA events on the batch stream",
            "done": done, "p50_request_ms": replicas.max_over_ranks(st["p50_request_ms"], dist, "cuda"),
            "p99_request_ms": replicas.max_over_ranks(st["p99_request_ms"], dist, "cuda"),
            "p50_queue_ms_rank0": st["p50_queue_ms"], "admitted_rank0": st["admitted"],
            "ticks_rank0": st["ticks"], "active_at_end": st["active"],
            "queued_at_end": st["queued"], "failed": st["failed"], "peak_bytes_rank0": st["peak_bytes"],
            "host_ms_rank0": {k: round(st[k + "_ms"], 1) for k in ("prepare", "admit", "wait", "retire")}}


def setup_block(naga, torch, args):
    """Set-up microbench: exact kNN (k = 32) over 64 clouds with point
    counts log-uniform in [5k, 200k] (uniform in the unit cube, seed 2) in
    one batched call; then the inverses of `setup_systems` 36 x 36 augmented
    r^3 RBF moment matrices (random k = 32 stencils of those clouds, centred
    and scaled), FP64 LU against FP32 LU with FP64-residual refinement, with
    the error of each against a CPU FP64 inverse (LAPACK through numpy) on
    a sample of 512 systems."""
    rng = np.random.default_rng(2)
    sizes = np.exp(rng.uniform(np.log(5e3), np.log(2e5), 64)).astype(np.int64)
    pts = torch.from_numpy(rng.random((int(sizes.sum()), 3)).astype(np.float32)).cuda()
    off = np.concatenate([[0], np.cumsum(sizes)])
    naga.knn_clouds(pts, off, 32)  # warm-up at full size (grows the allocation pool)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    idx, _ = naga.knn_clouds(pts, off, 32)
    e1.record()
    torch.cuda.synchronize()
    knn_ms = e0.elapsed_time(e1)
    # moment matrices of random stencils: centre, scale to unit box, r^3 + [1, x]
    n = args.setup_systems
    gen = torch.Generator(device="cuda").manual_seed(3)
    centre = torch.randint(0, pts.shape[0], (n,), device="cuda", generator=gen)
    X = pts.double()[idx[centre].long()] - pts.double()[centre][:, None]
    X /= X.abs().amax(dim=(1, 2), keepdim=True)
    A = torch.zeros((n, 36, 36), dtype=torch.float64, device="cuda")
    A[:, :32, :32] = torch.cdist(X, X) ** 3
    A[:, :32, 32] = 1.0
    A[:, 32, :32] = 1.0
    A[:, :32, 33:] = X
    A[:, 33:, :32] = X.transpose(1, 2)
    del X
    torch.cuda.synchronize()
    out = {"knn_clouds": 64, "knn_points": int(sizes.sum()), "knn_ms": knn_ms,
           "knn_mqueries_per_s": int(sizes.sum()) / knn_ms / 1e3, "inverse_systems": n}
    sample = np.random.default_rng(4).choice(n, 512, replace=False)
    # column-major storage: the inverse of the stored (transposed) matrix is
    # the transpose of the inverse, so compare in the same storage order
    ref = np.linalg.inv(A[torch.from_numpy(sample).cuda()].cpu().numpy().transpose(0, 2, 1)).transpose(0, 2, 1)
    for name, fn in (("f64", lambda: naga.batched_inverse_f64(A)),
                     ("f32r", lambda: naga.batched_inverse_f32r(A, max_iter=30, rel_tol=1e-14))):
        fn()
        torch.cuda.synchronize()
        e0.record()
        inv, info = fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        got = inv[torch.from_numpy(sample).cuda()].cpu().numpy()
        err = np.abs(got - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))
        out[f"inverse_{name}_ms"] = ms
        out[f"inverse_{name}_gflops"] = 2 * 36 ** 3 * n / (ms * 1e-3) / 1e9
        out[f"inverse_{name}_max_rel_err"] = float(err.max())
        out[f"inverse_{name}_flagged"] = int((info != 0).sum().item())
        del inv, info
    out["refinement_fallbacks"] = naga.refinement_fallbacks()
    return out


# ------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    cfg = CONFIG3
    if rank != 0:
        return 0
    cb = cpu_baseline(cfg, steps=args.steps, warmup=args.warmup)
    v = cb["value"]
    line = {"metric": "MNUPS (node updates/s) of the nonlocal LBM acoustics step", "value": v,
            "unit": "MNUPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(cb["nodes"], args.gpus),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "MNUPS", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_naga(args, rank, world, local_rank):
    import torch

    import naga_b200 as naga
    from naga_b200 import replicas

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
    total_ms = replicas.max_over_ranks(total_ms, dist, "cuda")
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
    e2e_s = replicas.max_over_ranks(e2e_s, dist, "cuda")
    e2e = world * N * K / e2e_s / 1e6

    # ---- the probe error the throughput is quoted at (1000 steps against
    # the FP64 oracle; after the timed regions)
    probe_error = probe_error_block(scene, g, drho) if args.n_side == 63 and not args.no_probe_error else None

    # ---- batched form (every rank steps its size-balanced share of the
    # scenes; time = slowest rank) vs the plain single 2-D scene
    batched = None
    if not args.no_batched:
        batched = batched_block(naga, torch, args, rank, world, dist, W, K)
    # ---- serving loop and set-up microbench (bounded samples)
    serving = serving_latency = None
    if not args.no_serving:
        serving = serving_block(naga, torch, args, rank, world, dist)
        serving_latency = serving_block(naga, torch, args, rank, world, dist, step_priority=1,
                                        target_step_ms=args.target_step_ms,
                                        seconds=args.serving_target_seconds)
    setup = None
    if not args.no_setup and rank == 0:
        setup = setup_block(naga, torch, args)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- per-kernel timing (CUDA events around each launch, separate run)
    prof = profile_kernels(naga, lambda: scene.step(1), steps=5)
    pmlc = pml_counts(naga, scene)
    kb = kernel_bytes(3, N, g["n_bulk"], g["n_layer"], g["n_boundary"], cfg["k"], cfg["k"], pmlc)
    gb = gather_bytes(g["n_bulk"], g["n_layer"], g["n_boundary"], cfg["k"], cfg["k"], pmlc)
    step_ms = sum(ms for (_, ms) in prof.values()) / 5
    # the dominant kernel: the largest share of the step (the four RK
    # stages count as the one kernel they are)
    top, per_launch, avg_ms, members = dominant_kernel(kb, prof)
    peak, peak_source = measured_hbm_peak()
    achieved = per_launch / (avg_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and args.n_side == 63:
        tj = json.load(open(tpath))
        if all(n in tj for n in members):
            traffic = sum(tj[n] for n in members) / len(members)
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": peak_source,
            "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": avg_ms,
            "launches_per_step": len(members),
            "kernel_share": {n: round(prof[n][1] / 5 / step_ms, 4) for n in prof if prof[n][0]},
            # every step kernel's algorithmic bytes / its launch time / peak
            "kernel_fracs": {n: round(kb[n] / (prof[n][1] / prof[n][0] * 1e-3) / 1e9 / peak, 3)
                             for n in kb if prof.get(n, (0, 0.0))[0]},
            "step_frac": sum(kb.values()) / (step_ms * 1e-3) / 1e9 / peak,
            # neighbour-row bytes each gather kernel's loads move into the
            # SMs (L2 or shared memory) per launch, and their rate
            "gather": {"unit": "GB/s", "row_bytes_per_launch": gb,
                       "achieved": {n: round(gb[n] / (prof[n][1] / prof[n][0] * 1e-3) / 1e9)
                                    for n in gb if prof.get(n, (0, 0.0))[0]}}}
    gpu_launches = sum(l for (l, _) in prof.values()) // 5 * K

    cb = None
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(cfg, max_seconds=15.0)

    line = {
        "metric": "MNUPS (node updates/s) of the nonlocal LBM acoustics step",
        "value": value, "unit": "MNUPS", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(N, world),
        "p50_step_ms": float(np.percentile(per, 50)), "p99_step_ms": float(np.percentile(per, 99)),
        "probe_error": probe_error, "roofline": roof, "cpu_baseline": cb,
        "e2e": {"value": e2e, "unit": "MNUPS", "h2d_bytes_per_step": int(N * 4 / K),
                "d2h_bytes_per_step": 4 * len(cfg["probes"]), "probe_trace_read_back": e2e_trace_ok},
        "gpu_launches": int(gpu_launches), "clocks": clk.summary(), "batched": batched,
        "serving": serving, "serving_latency_target": serving_latency, "setup": setup,
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
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-seconds", type=float, default=10.0)
    ap.add_argument("--serving-target-seconds", type=float, default=20.0)
    ap.add_argument("--target-step-ms", type=float, default=4.0,
                    help="per-step latency target of the second serving run")
    ap.add_argument("--no-setup", action="store_true")
    ap.add_argument("--no-probe-error", action="store_true",
                    help="skip the 1000-step probe-error check (profiling runs)")
    ap.add_argument("--setup-systems", type=int, default=1_000_000)
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

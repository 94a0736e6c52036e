"""The CUDA time step (FP32, centred populations) against the FP64 oracle of
the same step: set-up tables, single steps, probe traces, batches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROBES2 = np.array([[0.3, 0.5], [0.7, 0.5], [0.5, 0.3], [0.5, 0.7]], np.float32)
PROBES3 = np.array([[x, y, z] for z in (0.35, 0.65) for y in (0.35, 0.65) for x in (0.35, 0.65)],
                   np.float32)


def pair(naga, oracle, dim, n_side, layers, seed=0, shape=None, pml_indexing=0, width=0.05,
         n_ghost=0, sigma_peak=0.1):
    g = naga.generate_grid(dim, n_side, layers, seed, sigma_peak=sigma_peak)
    if n_ghost:
        rng = np.random.default_rng(seed)
        extra = rng.random((n_ghost, dim)).astype(np.float32) * 0.9 + 0.05
        g["points"] = np.concatenate([g["points"], extra]).astype(np.float32)
    k = 16 if dim == 2 else 32
    shape = (1 if dim == 2 else 0) if shape is None else shape
    probes = PROBES2 if dim == 2 else PROBES3
    gpu = naga.Scene(g, k=k, shape=shape, pml_indexing=pml_indexing, probes=probes, n_ghost=n_ghost)
    orc = oracle.Scene(dim, g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"], g["normals"],
                       g["sigma"], g["h"], k=k, shape=shape, pml_indexing=pml_indexing,
                       probes=probes, n_ghost=n_ghost)
    drho = naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, width)
    gpu.set_density(drho)
    orc.set_density(drho)
    return gpu, orc, g


def rel_err(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("dim", [2, 3])
def test_setup_tables_match_oracle(naga, oracle, dim):
    gpu, orc, g = pair(naga, oracle, dim, 30 if dim == 2 else 14, 3)
    t, o = gpu.tables(), orc.tables()
    nd = gpu.N
    assert np.array_equal(t["idx"][:nd], o["idx"][:nd])
    assert rel_err(t["W"], o["W"]) < 1e-6
    assert rel_err(t["fw"], o["fw"]) < 1e-6
    assert np.array_equal(t["bidx"], o["bidx"])
    assert rel_err(t["bw"], o["bw"]) < 1e-6
    assert np.array_equal(t["pidx"], o["pidx"])
    assert rel_err(t["pw"], o["pw"]) < 1e-6


@pytest.mark.parametrize("dim,pml_indexing", [(2, 0), (2, 1), (3, 0)])
def test_single_steps_match_oracle(naga, oracle, dim, pml_indexing):
    gpu, orc, _ = pair(naga, oracle, dim, 30 if dim == 2 else 14, 3, pml_indexing=pml_indexing,
                       width=0.1)
    for n in range(3):
        gpu.step(1)
        orc.step(1)
        gg, _ = gpu.state()
        go, _ = orc.state()
        assert rel_err(gg, go) < 1e-5, n


@pytest.mark.parametrize("dim,n_side,layers,steps", [(2, 40, 4, 200), (3, 16, 3, 60)])
def test_probe_trace_matches_oracle(naga, oracle, dim, n_side, layers, steps):
    gpu, orc, _ = pair(naga, oracle, dim, n_side, layers, width=0.08)
    gpu.step(steps)
    po = orc.step(steps)
    pg = gpu.probes(0, steps)
    assert rel_err(pg, po) <= 1e-5


def test_ghost_nodes_match_oracle(naga, oracle):
    gpu, orc, _ = pair(naga, oracle, 2, 30, 3, n_ghost=7, width=0.1)
    gpu.step(5)
    orc.step(5)
    assert rel_err(gpu.state()[0], orc.state()[0]) < 1e-5


@pytest.mark.slow
def test_config1_probe_trace_500_steps(naga, oracle):
    """2-D D2Q9, 20,164 jittered nodes (h = 1/141, seed 0), k = 16, r^3 RBF,
    10-layer PML, Gaussian pulse (1e-3, width 0.05), dt = 0.5 h / c, 500
    steps, 4 probes: probe error <= 1e-5 against the FP64 oracle."""
    gpu, orc, _ = pair(naga, oracle, 2, 142, 10, seed=0, width=0.05)
    gpu.step(500)
    po = orc.step(500)
    assert rel_err(gpu.probes(0, 500), po) <= 1e-5


@pytest.mark.slow
def test_config2_probe_trace_1000_steps(naga, golden_dir):
    """The benchmarked 3-D scene at full size: D3Q27, 250,047 jittered nodes
    (63^3, h = 1/62, seed 1), k = 32, multiquadric RBF, FP64 weight solves,
    8-layer PML, Gaussian pulse (1e-3, width 0.05), dt = 0.5 h / c, 8 probes,
    1000 steps. Probe error <= 1e-5 against the FP64 oracle's trace of the
    same scene (tests/golden/trace_d3q27_63.npz, made by
    tests/golden/make_config2_trace.py; the input digest proves the scene is
    the same)."""
    import os

    from tests.golden.make_config2_trace import PROBES3 as P3, scene_hash

    fx = np.load(os.path.join(golden_dir, "trace_d3q27_63.npz"))
    g = naga.generate_grid(3, 63, 8, 1)
    drho = naga.gaussian_pulse(g["points"], [0.5, 0.5, 0.5], 1e-3, 0.05)
    assert scene_hash(g, drho) == str(fx["sha256"])
    po = fx["probes"]
    gpu = naga.Scene(g, k=32, shape=0, probes=P3, probe_capacity=len(po))
    gpu.set_density(drho)
    gpu.step(len(po))
    assert rel_err(gpu.probes(0, len(po)), po) <= 1e-5


@pytest.mark.parametrize("priority", [0, 1])
def test_batch_equals_individual_scenes(naga, oracle, priority):
    gs = [naga.generate_grid(2, n, 3, s) for n, s in ((25, 1), (33, 2), (41, 3))]
    solo, members = [], []
    for g in gs:
        for lst in (solo, members):
            s = naga.Scene(g, k=16, probes=PROBES2)
            s.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.08))
            lst.append(s)
    b = naga.Batch(2, priority=priority)
    for s in members:
        b.add(s)
    b.step(25)
    for s in solo:
        s.step(25)
    for a, m in zip(solo, members):
        assert np.array_equal(a.probes(0, 25), m.probes(0, 25))
        assert np.array_equal(a.state()[0], m.state()[0])
    b.close()


_BATCH3_RUN = """
import sys, numpy as np
sys.path.insert(0, {root!r})
import naga_b200 as naga
pr = np.array({probes3!r}, np.float32)
gs = [naga.generate_grid(3, n, 3, s) for n, s in ((14, 1), (17, 2), (15, 3))]
solo, members = [], []
for g in gs:
    for lst in (solo, members):
        s = naga.Scene(g, k=32, shape=0, probes=pr)
        s.set_density(naga.gaussian_pulse(g["points"], [0.5] * 3, 1e-3, 0.08))
        lst.append(s)
b = naga.Batch(3)
for s in members:
    b.add(s)
b.step(12)
for s in solo:
    s.step(12)
ok = all(np.array_equal(a.probes(0, 12), m.probes(0, 12)) and np.array_equal(a.state()[0], m.state()[0])
         for a, m in zip(solo, members))
b.close()
print("equal" if ok else "differ")
print(naga.tuning_report())
"""


def test_batch_of_3d_scenes_with_halo_stages(tmp_path):
    """A batch of three D3Q27 scenes at k = 32 takes the same steps as each
    scene alone, bit for bit, with the shared-memory halo RK stages forced:
    their passes switch between the scenes' blobs and rows."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env["NAGA_GATHER_TPN"] = "halo"
    env.pop("NAGA_GATHER_BPS", None)
    code = _BATCH3_RUN.format(root=root, probes3=PROBES3.tolist())
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("equal"), r.stdout
    assert "tpn halo" in r.stdout


def test_batch_membership_changes(naga, oracle):
    """Scenes leave and join a stepping batch (its item tables are rebuilt
    in place on the device); every scene's trace still equals the same
    scene stepped alone for the same number of steps."""
    gs = [naga.generate_grid(2, n, 3, s) for n, s in ((25, 1), (33, 2), (41, 3), (29, 4))]

    def make(g):
        s = naga.Scene(g, k=16, probes=PROBES2)
        s.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.07))
        return s

    members = [make(g) for g in gs]
    b = naga.Batch(2)
    for s in members[:3]:
        b.add(s)
    b.step(10)
    b.remove(members[1])
    b.step(10)
    b.add(members[3])
    b.step(10)
    members[1].step(5)  # stepped alone after leaving
    steps = [30, 15, 30, 10]
    for g, m, n in zip(gs, members, steps):
        solo = make(g)
        solo.step(n)
        assert np.array_equal(solo.probes(0, n), m.probes(0, n))
        assert np.array_equal(solo.state()[0], m.state()[0])
    b.close()


def test_step_is_deterministic(naga, oracle):
    a, _, g = pair(naga, oracle, 3, 14, 3)
    b = naga.Scene(g, k=32, shape=0, probes=PROBES3)
    b.set_density(naga.gaussian_pulse(g["points"], [0.5] * 3, 1e-3, 0.05))
    a.step(10)
    b.step(10)
    assert np.array_equal(a.state()[0], b.state()[0])
    assert np.array_equal(a.probes(), b.probes())


_SHAPE_RUN = """
import sys, numpy as np
sys.path.insert(0, {root!r})
import naga_b200 as naga
out = []
for dim, n, k, scramble in ((3, 20, 32, False), (2, 48, 16, False), (3, 20, 32, True)):
    g = naga.generate_grid(dim, n, 3, 4)
    if scramble:
        # bulk and boundary nodes in random order: a pass's supports are
        # scattered and most passes list more rows than the halo stages keep
        rng = np.random.default_rng(5)
        perm = rng.permutation(g["n_bulk"])
        g["points"][: g["n_bulk"]] = g["points"][perm]
        b0 = g["n_bulk"] + g["n_layer"]
        pb = rng.permutation(g["n_boundary"])
        g["points"][b0 : b0 + g["n_boundary"]] = g["points"][b0 + pb]
        g["normals"] = np.ascontiguousarray(g["normals"][pb])
    pr = np.array({probes3!r} if dim == 3 else {probes2!r}, np.float32)
    s = naga.Scene(g, k=k, shape=0 if dim == 3 else 1, probes=pr)
    s.set_density(naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, 0.05))
    s.step(15)
    out += [s.state()[0].ravel(), s.probes().ravel()]
np.save({out!r}, np.concatenate(out))
print(naga.tuning_report())
"""


def test_launch_shape_does_not_change_results(tmp_path):
    """The tuner's choices -- resident blocks per SM of the gather kernels, of
    the filter, threads per node of the RK stages, and the shared-memory halo
    RK stages -- change only the launch: runs with the tuned shape and with
    shapes forced through NAGA_GATHER_BPS / NAGA_GATHER_TPN (D3Q27 at 7 and 4
    threads per node and with the halo stages, D2Q9 at 1) agree bit for bit,
    on Morton-ordered scenes and on one with its bulk nodes scrambled (whose
    passes overflow the halo list and gather from global memory), and the
    tuner logs what it measured."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs, logs = [], []
    for env_bps, env_tpn in ((None, None), ("2", None), (None, "7"), ("3", "4"), (None, "1"), (None, "halo")):
        out = str(tmp_path / f"run_{env_bps}_{env_tpn}.npy")
        env = dict(os.environ)
        env.pop("NAGA_GATHER_BPS", None)
        env.pop("NAGA_GATHER_TPN", None)
        if env_bps:
            env["NAGA_GATHER_BPS"] = env_bps
        if env_tpn:
            env["NAGA_GATHER_TPN"] = env_tpn
        code = _SHAPE_RUN.format(root=root, probes3=PROBES3.tolist(), probes2=PROBES2.tolist(), out=out)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append(np.load(out))
        logs.append(r.stdout)
    for o in outs[1:]:
        assert np.array_equal(outs[0], o)
    assert "dim 3 k 32 kb 32" in logs[0] and "| tpn 8 0:" in logs[0] and "| tpn 7" in logs[0]
    assert "dim 2 k 16 kb 16" in logs[0] and "| tpn 1" in logs[0] and "| filter 0:" in logs[0]
    assert "tpn 8 bps 2 filter bps" in logs[1] and "(NAGA_GATHER_BPS" in logs[1]
    assert "dim 3 k 32 kb 32 items 2^" in logs[2] and "tpn 7 bps 0 filter bps 0 (NAGA_GATHER" in logs[2]
    assert "tpn 4 bps 3 filter bps" in logs[3]
    assert "dim 2 k 16 kb 16 items 2^" in logs[4] and "tpn 1 bps 0 filter bps 0 (NAGA_GATHER" in logs[4]
    assert "| tpn halo 2:" in logs[0]
    assert "dim 3 k 32 kb 32 items 2^" in logs[5] and "tpn halo bps 0 filter bps 0 (NAGA_GATHER" in logs[5]


def test_async_probe_reads_match_synchronous(naga, oracle):
    """Probe samples queued every step behind the step (page-locked host
    buffer, one sync at the end) equal the synchronous read, including a
    read that wraps around the ring."""
    import torch

    g = naga.generate_grid(2, 30, 3, 7)
    s = naga.Scene(g, k=16, probes=PROBES2, probe_capacity=16)
    s.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.08))
    out = torch.zeros((40, 4), dtype=torch.float32, pin_memory=True)
    for t in range(40):
        s.step(1)
        s.probes_async(t, 1, out.data_ptr() + 16 * t)
    s.sync()
    ref = naga.Scene(g, k=16, probes=PROBES2, probe_capacity=64)
    ref.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.08))
    ref.step(40)
    assert np.array_equal(out.numpy(), ref.probes(0, 40))
    wrap = torch.zeros((10, 4), dtype=torch.float32, pin_memory=True)
    s.probes_async(30, 10, wrap.data_ptr())  # ring slots 14, 15, 0, ..., 7
    s.sync()
    assert np.array_equal(wrap.numpy(), ref.probes(30, 10))


@pytest.mark.parametrize("dim", [2, 3])
def test_snapshot_resumes_bit_for_bit(naga, oracle, dim):
    """Save after 17 steps, keep stepping; a new scene of the same
    description loaded from the snapshot takes the same next 13 steps bit for
    bit (state, probe trace, step count), across an odd step count so the
    PML ping-pong parity is exercised; a snapshot of another shape is
    rejected."""
    n_side, layers = (30, 3) if dim == 2 else (14, 3)
    g = naga.generate_grid(dim, n_side, layers, 2)
    k = 16 if dim == 2 else 32
    probes = PROBES2 if dim == 2 else PROBES3
    a = naga.Scene(g, k=k, shape=1 if dim == 2 else 0, probes=probes, probe_capacity=64)
    a.set_density(naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, 0.08))
    a.step(17)
    snap = a.save()
    a.step(13)
    b = naga.Scene(g, k=k, shape=1 if dim == 2 else 0, probes=probes, probe_capacity=64)
    b.load(snap)
    assert b.step_count == 17
    b.step(13)
    assert b.step_count == a.step_count == 30
    assert np.array_equal(a.state()[0], b.state()[0])
    assert np.array_equal(a.probes(0, 30), b.probes(0, 30))
    other = naga.Scene(naga.generate_grid(dim, n_side + 1, layers, 2), k=k, shape=1 if dim == 2 else 0,
                       probes=probes, probe_capacity=64)
    with pytest.raises(RuntimeError, match="another shape"):
        other.load(snap)


@pytest.mark.parametrize("dim,n_side,layers,steps", [(2, 40, 4, 60), (3, 16, 3, 40)])
def test_density_source_matches_oracle(naga, oracle, dim, n_side, layers, steps):
    """A sinusoidal point source at the node nearest the centre (every fifth
    step the sentinel: no term) through the C ABI against the FP64 oracle:
    probe traces within 1e-5, state within 1e-5; removing the sources gives
    the plain step again."""
    gpu, orc, g = pair(naga, oracle, dim, n_side, layers)
    centre = int(np.argmin(((g["points"] - 0.5) ** 2).sum(1)))
    t = np.arange(steps)
    vals = (2e-4 * np.sin(2 * np.pi * t / 17.0)).astype(np.float32)[:, None]
    vals[::5] = np.finfo(np.float32).max
    gpu.set_density_source([centre], vals)
    orc.set_sources([centre], vals)
    pg = gpu.probes(0, 0)
    gpu.step(steps)
    po = orc.step(steps)
    assert rel_err(gpu.probes(0, steps), po) <= 1e-5
    go, _ = orc.state()
    assert rel_err(gpu.state()[0], go) <= 1e-5
    # without sources the same scene steps as a plain one
    plain, orc2, _ = pair(naga, oracle, dim, n_side, layers)
    gpu.set_density(naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, 0.05))
    gpu.set_density_source([], np.zeros((0, 0), np.float32))
    gpu.step(5)
    plain.step(5)
    assert np.array_equal(gpu.state()[0], plain.state()[0])


def test_batch_of_mixed_stencil_sizes(naga, oracle):
    """Members with different k take the generic (not fully unrolled)
    kernels; each still equals the same scene stepped alone."""
    gs = [naga.generate_grid(2, n, 3, s) for n, s in ((28, 5), (35, 6))]
    ks = (12, 16)

    def make(g, k):
        s = naga.Scene(g, k=k, k_boundary=k, probes=PROBES2)
        s.set_density(naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.07))
        return s

    members = [make(g, k) for g, k in zip(gs, ks)]
    b = naga.Batch(2)
    for s in members:
        b.add(s)
    b.step(20)
    for g, k, m in zip(gs, ks, members):
        solo = make(g, k)
        solo.step(20)
        assert np.array_equal(solo.probes(0, 20), m.probes(0, 20))
        assert np.array_equal(solo.state()[0], m.state()[0])
    b.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_scene_without_layer_or_probes_matches_oracle(naga, oracle, dim):
    """No PML layer (the PML kernels have no work) and no probes."""
    g = naga.generate_grid(dim, 30 if dim == 2 else 14, 0, 9)
    assert g["n_layer"] == 0
    k = 16 if dim == 2 else 32
    shape = 1 if dim == 2 else 0
    gpu = naga.Scene(g, k=k, shape=shape)
    orc = oracle.Scene(dim, g["points"], g["n_bulk"], 0, g["n_boundary"], g["normals"], g["sigma"], g["h"],
                       k=k, shape=shape)
    drho = naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, 0.1)
    gpu.set_density(drho)
    orc.set_density(drho)
    gpu.step(4)
    orc.step(4)
    assert rel_err(gpu.state()[0], orc.state()[0]) < 1e-5


def test_bounded_wait_gives_up_and_context_stays_usable(naga, oracle):
    """The step kernels' tile wait, on a barrier that nothing completes,
    gives up at its own poll limit within seconds (no hang), the host reads
    NAGA_ETIMEOUT once (the flag is cleared), and the same context then
    steps a scene to the oracle's trace."""
    import time

    naga.selftest_wait_timeout(16)  # context warm-up
    t0 = time.perf_counter()
    assert naga.selftest_wait_timeout(0) == naga.NAGA_ETIMEOUT
    took = time.perf_counter() - t0
    print(f"step-kernel tile wait gave up after {took:.2f} s")
    assert took < 10.0
    assert "did not complete in time" in naga.lib().naga_last_error().decode()
    gpu, orc, _ = pair(naga, oracle, 2, 30, 3, width=0.1)
    gpu.step(5)
    po = orc.step(5)
    assert rel_err(gpu.probes(0, 5), po) <= 1e-5


def test_set_params_equals_scene_created_with_them(naga, oracle):
    """set_problem_parameters on a live scene (naga_scene_set_params, then
    the initial condition) gives bit for bit the scene created with those
    parameters."""
    g = naga.generate_grid(2, 30, 3, 11)
    drho = naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, 0.08)
    nu, rho0, dt = 3e-5, 1.2, 0.4 * g["h"]
    ref = naga.Scene(g, k=16, probes=PROBES2, viscosity=nu, rho0=rho0, time_step=dt)
    ref.set_density(drho)
    ref.step(12)
    s = naga.Scene(g, k=16, probes=PROBES2)
    s.set_density(drho)
    s.step(3)
    s.set_params(nu, rho0, dt, 1.0)
    s.set_initial_condition(drho)
    s.step(12)
    assert np.array_equal(s.probes(0, 12), ref.probes(0, 12))
    assert np.array_equal(s.state()[0], ref.state()[0])


def test_init_domain_rebuilds_the_handle(naga, oracle):
    """init_domain on a live handle equals a scene created on the new domain
    (nodes, stencils, probes, step count)."""
    g1 = naga.generate_grid(2, 26, 3, 12)
    g2 = naga.generate_grid(2, 33, 4, 13)
    s = naga.Scene(g1, k=16, probes=PROBES2[:2])
    s.set_density(naga.gaussian_pulse(g1["points"], [0.5, 0.5], 1e-3, 0.08))
    s.step(4)
    drho = naga.gaussian_pulse(g2["points"], [0.45, 0.5], 1e-3, 0.07)
    s.init_domain(g2, k=16, probes=PROBES2)
    assert s.step_count == 0 and s.N == len(g2["points"])
    s.set_density(drho)
    s.step(10)
    ref = naga.Scene(g2, k=16, probes=PROBES2)
    ref.set_density(drho)
    ref.step(10)
    assert np.array_equal(s.probes(0, 10), ref.probes(0, 10))
    assert np.array_equal(s.state()[0], ref.state()[0])


@pytest.mark.parametrize("dim", [2, 3])
def test_add_probe_after_creation(naga, oracle, dim):
    """A probe attached after some steps samples like the same probe given
    at creation from then on (zeros before); the other probes keep their
    history."""
    g = naga.generate_grid(dim, 30 if dim == 2 else 14, 3, 14)
    P = PROBES2 if dim == 2 else PROBES3
    k = 16 if dim == 2 else 32
    shape = 1 if dim == 2 else 0
    drho = naga.gaussian_pulse(g["points"], [0.5] * dim, 1e-3, 0.08)
    ref = naga.Scene(g, k=k, shape=shape, probes=P[:3])
    ref.set_density(drho)
    ref.step(10)
    s = naga.Scene(g, k=k, shape=shape, probes=P[:2])
    s.set_density(drho)
    s.step(4)
    assert s.add_probe(P[2]) == 2
    s.step(6)
    got, want = s.probes(0, 10), ref.probes(0, 10)
    assert np.array_equal(got[:, :2], want[:, :2])
    assert np.array_equal(got[4:, 2], want[4:, 2])
    assert (got[:4, 2] == 0).all()


def test_box_grid_scene_matches_oracle(naga, oracle):
    """A scene on NAGA's uniform_grid_provider box (non-square, offset,
    absorbing layer) steps to the FP64 oracle's probe trace."""
    g = naga.box_grid([-0.5, 0.0], [0.7, 0.9], 0.03, 0.12, 0.1)
    probes = np.array([[-0.2, 0.45], [0.3, 0.5]], np.float32)
    gpu = naga.Scene(g, k=16, shape=1, probes=probes)
    orc = oracle.Scene(2, g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"], g["normals"], g["sigma"],
                       g["h"], k=16, shape=1, probes=probes)
    drho = naga.gaussian_pulse(g["points"], [0.1, 0.45], 1e-3, 0.08)
    gpu.set_density(drho)
    orc.set_density(drho)
    gpu.step(60)
    po = orc.step(60)
    assert rel_err(gpu.probes(0, 60), po) <= 1e-5


def test_macros_as_naga_solution(naga, oracle):
    """naga_scene_read_macros: the density and velocity of the last step,
    dimensional as NAGA stores them (rho rho0, u c / c_s), equal the macros
    of the state that step started from."""
    g = naga.generate_grid(2, 30, 3, 15)
    rho0, c = 1.2, 1.3
    s = naga.Scene(g, k=16, probes=PROBES2, rho0=rho0, speed_of_sound=c)
    s.set_density(naga.gaussian_pulse(g["points"], [0.45, 0.5], 1e-3, 0.08))
    s.step(7)
    gs, _ = s.state()
    s.step(1)
    rho, u = s.macros()
    w, cv = naga.lattice(2)
    drho = gs.astype(np.float64).sum(1)
    ulat = (gs.astype(np.float64) @ cv.astype(np.float64)) / (1.0 + drho)[:, None]
    nbl = g["n_bulk"] + g["n_layer"]
    assert np.allclose(rho, (1.0 + drho) * rho0, rtol=0, atol=1e-6)
    # boundary velocities are 0 after the bounce-back, as in NAGA's solution
    assert (u[nbl:] == 0).all()
    want = ulat[:nbl] * c * np.sqrt(3.0)
    assert np.abs(u[:nbl] - want).max() <= 1e-6 * max(1.0, np.abs(want).max())
    assert np.abs(u[:nbl]).max() > 0

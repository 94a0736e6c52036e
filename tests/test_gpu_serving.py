"""The continuous-batching request loop: results alone equal results in the
mix; admission respects the memory budget and slot limit; a bad request
fails alone."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROBES2 = np.array([[0.3, 0.5], [0.7, 0.5]], np.float32)


def _req(naga, n_side, seed, width):
    g = naga.generate_grid(2, n_side, 3, seed)
    drho = naga.gaussian_pulse(g["points"], [0.5, 0.5], 1e-3, width)
    return g, drho


def _tick(srv):
    """One tick; while no scene is active (set-up still running on the
    server's own thread) it returns at once, so wait a moment then."""
    active, queued = srv.tick()
    if active == 0 and queued > 0:
        time.sleep(0.002)
    return active, queued


def _run_until_done(srv, ids, seconds=120.0):
    deadline = time.time() + seconds
    while time.time() < deadline:
        _tick(srv)
        if all(srv.state(i)[0] in (srv.DONE, srv.FAILED) for i in ids):
            return
    raise AssertionError("requests did not finish")


def test_results_alone_equal_results_in_the_mix(naga):
    reqs = [_req(naga, n, s, w) for n, s, w in ((30, 1, 0.06), (45, 2, 0.08), (26, 3, 0.05), (38, 4, 0.07))]
    steps = [60, 35, 80, 50]
    alone = []
    for (g, d), n in zip(reqs, steps):
        srv = naga.Server(2, memory_budget=1 << 30, steps_per_tick=10)
        rid = srv.submit(g, d, n, k=16, probes=PROBES2)
        _run_until_done(srv, [rid])
        alone.append(srv.result(rid))
        srv.close()
    # mixed: staggered arrivals, two slots, so requests join a running batch
    # (steps ahead of set-up on the device: same results)
    srv = naga.Server(2, memory_budget=1 << 30, steps_per_tick=10, max_active=2, step_priority=1)
    ids = [srv.submit(reqs[0][0], reqs[0][1], steps[0], k=16, probes=PROBES2)]
    deadline = time.time() + 60
    while time.time() < deadline and srv.stats()["ticks"] < 2:
        _tick(srv)
    ids += [srv.submit(g, d, n, k=16, probes=PROBES2) for (g, d), n in zip(reqs[1:], steps[1:])]
    _run_until_done(srv, ids)
    st = srv.stats()
    assert st["done"] == 4 and st["failed"] == 0 and st["p99_step_ms"] > 0
    for rid, a in zip(ids, alone):
        assert np.array_equal(srv.result(rid), a)
    srv.close()
    # and the same trace as a plain scene stepped on its own
    s = naga.Scene(reqs[2][0], k=16, probes=PROBES2)
    s.set_density(reqs[2][1])
    s.step(steps[2])
    assert np.array_equal(s.probes(0, steps[2]), alone[2])


PROBES3 = np.array([[0.35, 0.5, 0.5], [0.65, 0.5, 0.5]], np.float32)


def test_3d_results_alone_equal_results_in_the_mix(naga):
    """D3Q27 requests at k = 32 (the benchmark's lattice and stencil size:
    halo lists built on the set-up thread, steps in a growing 3-D batch)
    give the same probe traces alone, in the mix and as a plain scene."""
    reqs = []
    for n, seed, width in ((14, 1, 0.08), (17, 2, 0.1), (15, 3, 0.09)):
        g = naga.generate_grid(3, n, 3, seed)
        reqs.append((g, naga.gaussian_pulse(g["points"], [0.5] * 3, 1e-3, width)))
    steps = [24, 16, 30]
    kw = dict(k=32, shape=0, probes=PROBES3)
    alone = []
    for (g, d), n in zip(reqs, steps):
        srv = naga.Server(3, memory_budget=1 << 31, steps_per_tick=8)
        rid = srv.submit(g, d, n, **kw)
        _run_until_done(srv, [rid])
        alone.append(srv.result(rid))
        srv.close()
    srv = naga.Server(3, memory_budget=1 << 31, steps_per_tick=8, max_active=3)
    ids = [srv.submit(reqs[0][0], reqs[0][1], steps[0], **kw)]
    deadline = time.time() + 60
    while time.time() < deadline and srv.stats()["ticks"] < 2:
        _tick(srv)
    ids += [srv.submit(g, d, n, **kw) for (g, d), n in zip(reqs[1:], steps[1:])]
    _run_until_done(srv, ids)
    st = srv.stats()
    assert st["done"] == 3 and st["failed"] == 0
    for rid, a in zip(ids, alone):
        assert np.array_equal(srv.result(rid), a)
    srv.close()
    s = naga.Scene(reqs[1][0], **kw)
    s.set_density(reqs[1][1])
    s.step(steps[1])
    assert np.array_equal(s.probes(0, steps[1]), alone[1])


def test_admission_by_memory_budget(naga):
    g, d = _req(naga, 40, 5, 0.06)
    desc, _ = naga.scene_desc(g, k=16, probes=PROBES2, probe_capacity=40)
    import ctypes
    est = naga.lib().naga_scene_estimate_bytes(ctypes.byref(desc))
    assert est > 0
    # room for one scene at a time: the second waits until the first retires
    srv = naga.Server(2, memory_budget=int(est * 1.5), steps_per_tick=10)
    a = srv.submit(g, d, 30, k=16, probes=PROBES2)
    b = srv.submit(g, d, 30, k=16, probes=PROBES2)
    # set-up runs on the server's own thread: tick until the first joins
    deadline = time.time() + 60
    while time.time() < deadline and srv.state(a)[0] != srv.ACTIVE:
        _tick(srv)
    assert srv.state(a)[0] == srv.ACTIVE and srv.state(b)[0] == srv.QUEUED
    assert srv.stats()["bytes_in_use"] <= int(est * 1.5)
    _run_until_done(srv, [a, b])
    assert np.array_equal(srv.result(a), srv.result(b))
    # a request larger than the whole budget fails instead of blocking
    big, dbig = _req(naga, 120, 6, 0.06)
    c = srv.submit(big, dbig, 10, k=16, probes=PROBES2)
    e = srv.submit(g, d, 10, k=16, probes=PROBES2)
    _run_until_done(srv, [c, e])
    assert srv.state(c)[0] == srv.FAILED and srv.state(e)[0] == srv.DONE
    srv.close()


def test_invalid_request_fails_alone(naga):
    g, d = _req(naga, 30, 7, 0.06)
    srv = naga.Server(2, memory_budget=1 << 30, steps_per_tick=5)
    ok = srv.submit(g, d, 20, k=16, probes=PROBES2)
    bad = srv.submit(g, d, 20, k=16, probes=PROBES2, shape=7)  # unknown RBF shape
    _run_until_done(srv, [ok, bad])
    assert srv.state(bad)[0] == srv.FAILED
    assert srv.state(ok)[0] == srv.DONE
    assert srv.result(ok).shape == (20, 2)
    srv.close()


def test_latency_target_bounds_the_batch(naga):
    """With a per-step latency target below any two scenes' step time, the
    set-up thread admits one request at a time (after the first measured
    step): the requests still all finish, with results identical to a server
    without the target, and completion latencies are reported."""
    reqs = [_req(naga, n, s, w) for n, s, w in ((34, 11, 0.06), (30, 12, 0.07), (40, 13, 0.05))]
    free = naga.Server(2, memory_budget=1 << 30, steps_per_tick=10)
    ids = [free.submit(g, d, 30, k=16, probes=PROBES2) for g, d in reqs]
    _run_until_done(free, ids)
    ref = [free.result(i) for i in ids]
    free.close()
    srv = naga.Server(2, memory_budget=1 << 30, steps_per_tick=10, target_step_ms=1e-4)
    ids = [srv.submit(g, d, 30, k=16, probes=PROBES2) for g, d in reqs]
    most = 0
    deadline = time.time() + 120
    while time.time() < deadline:
        active, _ = _tick(srv)
        if srv.stats()["ticks"] > 0:
            most = max(most, active)
        if all(srv.state(i)[0] in (srv.DONE, srv.FAILED) for i in ids):
            break
    st = srv.stats()
    assert st["done"] == 3 and st["failed"] == 0
    assert most == 1
    assert st["p50_request_ms"] > 0 and st["p99_request_ms"] >= st["p50_request_ms"]
    assert st["p50_step_ms"] > 0 and st["admitted"] == 3
    for i, r in zip(ids, ref):
        assert np.array_equal(srv.result(i), r)
    srv.close()

"""The header-only C++ facade (include/naga/naga.hpp): a NAGA-style driver
program compiled with g++, linked against libnaga_b200.so and run."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _run_program(naga, name, *args):
    gxx = shutil.which("g++-13") or shutil.which("g++")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, name)
        r = subprocess.run([gxx, "-std=c++17", "-O2", f"-I{ROOT}/include", "-I/usr/local/cuda/include",
                            os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o", exe,
                            f"-L{os.path.dirname(naga.LIB_PATH)}", "-lnaga_b200",
                            f"-Wl,-rpath,{os.path.dirname(naga.LIB_PATH)}", "-L/usr/local/cuda/lib64",
                            "-lcudart"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stderr
    return out.stdout


def test_facade_program_matches_python_binding(naga):
    stdout = _run_program(naga, "facade_pulse", "15")
    rows = np.array([[float(v) for v in l.split()] for l in stdout.strip().splitlines()])
    g = naga.generate_grid(2, 40, 4, 0)
    s = naga.Scene(g, k=16, shape=1, probes=np.array([[0.3, 0.5], [0.7, 0.5]], np.float32))
    P = g["points"].astype(np.float64)
    drho = (1e-3 * np.exp(-((P - 0.5) ** 2).sum(1) / (2 * 0.08 ** 2))).astype(np.float32)
    s.set_density(drho)
    s.step(15)
    p = s.probes(0, 15)
    assert np.allclose(rows[:, 1:], p, rtol=0, atol=1e-7 * max(1.0, np.abs(p).max()) + 2e-7)
    assert np.allclose(rows[:, 0], np.arange(15) * 0.5 * g["h"], rtol=1e-5)


def test_facade_density_source_matches_python_binding(naga):
    """register_density_source through the facade (one row uploaded per
    step) equals the same values given to the Python binding at once."""
    lines = _run_program(naga, "facade_source", "25").strip().splitlines()
    centre = int(lines[0])
    rows = np.array([[float(v) for v in l.split()] for l in lines[1:]])
    g = naga.generate_grid(2, 40, 4, 0)
    s = naga.Scene(g, k=16, shape=1, probes=np.array([[0.3, 0.5], [0.5, 0.45]], np.float32))
    s.set_density(np.zeros(len(g["points"]), np.float32))
    s.set_density_source([centre], rows[:, 1].astype(np.float32)[:, None])
    s.step(25)
    p = s.probes(0, 25)
    assert np.abs(p).max() > 0
    assert np.allclose(rows[:, 2:], p, rtol=0, atol=1e-7 * max(1.0, np.abs(p).max()) + 2e-7)


def test_facade_live_observers_and_parameters(naga):
    """attach_observer and set_problem_parameters on a running facade engine
    (naga_scene_add_probe / naga_scene_set_params underneath) agree bit for
    bit with engines that had them from the start."""
    assert _run_program(naga, "facade_live").strip() == "ok"


def test_facade_save_and_load_state(naga):
    """simulation_engine / density_observer save_state and load_state with a
    cereal-style archive: the restored engine continues bit for bit."""
    assert _run_program(naga, "facade_state").strip() == "ok"


def test_facade_primitive_classes(naga, oracle):
    """nd_cubic_segmentation, batched_nearest_neighbors(k, query_map,
    segmentation), radial_point_method<float> and divergence_operator<T, 3>
    (T = double and float) driven as NAGA's examples drive them
    (tests/cpp/facade_primitives.cpp), against the oracle: the partition and
    the neighbours bit for bit, weights and fields within FP32 / FP64
    rounding."""
    with tempfile.TemporaryDirectory() as out:
        assert _run_program(naga, "facade_primitives", out).strip() == "ok"
        rd = lambda name, dt: np.fromfile(os.path.join(out, name), dt)
        seg_sizes, seg_idx = rd("seg_sizes.u32", np.uint32), rd("seg_indices.u32", np.uint32)
        seg_meta = rd("seg_meta.f32", np.float32)
        knn_idx, knn_d2 = rd("knn_idx.u32", np.uint32), rd("knn_d2.f32", np.float32)
        w, vals = rd("rpim_weights.f32", np.float32), rd("rpim_values.f32", np.float32)
        div64, div_idx = rd("div_f64.f64", np.float64), rd("div_idx.u32", np.uint32)
        div32 = rd("div_f32_offset.f32", np.float32)

    def grid(m, spacing, dt):
        i = np.arange(m ** 3)
        return np.stack([(i % m).astype(dt) * spacing, ((i // m) % m).astype(dt) * spacing,
                         (i // (m * m)).astype(dt) * spacing], -1).astype(dt)

    pi = np.float32(3.14159265358979)
    m, mi = 24, 17
    sp = np.float32(2) * pi / np.float32(m - 1)
    isp = np.float32(2) * pi / np.float32(mi - 1)
    src, qry = grid(m, sp, np.float32), grid(mi, isp, np.float32)
    seg = oracle.cubic_segmentation(src, 32)
    assert np.array_equal(seg_sizes, seg["sizes"]) and np.array_equal(seg_idx, seg["indices"])
    assert seg_meta[0] == np.float32(seg["width"]) and np.array_equal(seg_meta[1:], seg["shape"])
    oi, od = oracle.knn(src, qry, 32)
    assert np.array_equal(knn_idx.reshape(oi.shape), oi) and np.array_equal(knn_d2.reshape(od.shape), od)
    ow = oracle.rbf_weights(src, oi, qry.astype(np.float64), 1, float(sp), 0)
    assert np.abs(w.reshape(ow.shape) - ow).max() <= 1e-6 * np.abs(ow).max()
    S = src.astype(np.float64)
    f = np.sin(S[:, 0]) * np.cos(S[:, 1]) * S[:, 2]
    ref = np.einsum("qs,qs->q", ow, f[oi])
    assert np.abs(vals - ref).max() <= 1e-5 * np.abs(f).max()

    md = 20
    dg = grid(md, 2 * np.pi / (md - 1), np.float64)
    F = np.stack([np.sin(dg[:, 0]), 0 * dg[:, 0], np.cos(dg[:, 2])], -1)
    di, dW, _ = oracle.divergence_stencil(dg.astype(np.float32), 32, 0)
    assert np.array_equal(div_idx.reshape(di.shape), di)
    ref64 = np.einsum("nsd,nsd->n", dW, F[di])
    scale = np.abs(ref64).max()
    assert np.abs(div64 - ref64).max() <= 1e-9 * scale
    F32 = F.astype(np.float32).astype(np.float64)
    ref32 = np.einsum("nsd,nsd->n", dW, F32[di] - 0.25)
    assert np.abs(div32 - ref32).max() <= 2e-5 * scale

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

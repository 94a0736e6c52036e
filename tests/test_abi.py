"""The C ABI library loads and exports what include/naga_b200.h declares;
host-side logic (synthetic scenes) works without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "naga_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(naga_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(naga):
    names = _declared()
    assert len(names) > 30
    lib = ctypes.CDLL(naga.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_channel(naga):
    assert naga.lib().naga_version() >= 100
    with pytest.raises(naga.NagaError) as e:
        naga.generate_grid(4, 10, 1, 0)
    assert e.value.code == naga.NAGA_EINVAL
    assert "grid" in str(e.value)


@pytest.mark.parametrize("dim,n_side,layers,counts", [
    (2, 142, 10, (14626, 4974, 564)),
    (3, 63, 8, (97491, 129490, 23066)),
])
def test_grid_scene_counts(naga, dim, n_side, layers, counts):
    g = naga.generate_grid(dim, n_side, layers, seed=0 if dim == 2 else 1)
    assert (g["n_bulk"], g["n_layer"], g["n_boundary"]) == counts
    assert g["points"].shape == (sum(counts), dim)
    assert abs(g["h"] - 1.0 / (n_side - 1)) < 1e-15


def test_grid_scene_properties(naga):
    g = naga.generate_grid(2, 50, 5, seed=7, sigma_peak=0.2)
    a = naga.generate_grid(2, 50, 5, seed=7, sigma_peak=0.2)
    b = naga.generate_grid(2, 50, 5, seed=8, sigma_peak=0.2)
    assert np.array_equal(g["points"], a["points"])
    assert not np.array_equal(g["points"], b["points"])
    nb, nl, nbd, h = g["n_bulk"], g["n_layer"], g["n_boundary"], g["h"]
    P = g["points"].astype(np.float64)
    bnd = P[nb + nl:]
    # boundary nodes on the walls, normals unit and pointing inward
    assert np.all(np.min(np.minimum(bnd, 1 - bnd), 1) < 1e-6)
    n = g["normals"]
    assert np.allclose(np.linalg.norm(n, axis=1), 1, atol=1e-6)
    assert np.all(((bnd + 0.5 * h * n) > 0) & ((bnd + 0.5 * h * n) < 1))
    # layer: within L of the boundary, sigma in [0, peak]
    L = 5 * h
    dist = np.sqrt(((P[nb:nb + nl, None, :] - bnd[None]) ** 2).sum(-1)).min(1)
    assert np.all(dist <= L * (1 + 1e-6))
    dbulk = np.sqrt(((P[:nb, None, :] - bnd[None]) ** 2).sum(-1)).min(1)
    assert np.all(dbulk > L * (1 - 1e-6))
    s = g["sigma"]
    assert np.all((s >= 0) & (s <= 0.2 + 1e-7))
    assert np.allclose(s, 0.2 * ((L - dist) / L) ** 2, atol=1e-6)
    # interior jitter bounded by h / 4
    assert np.all(np.abs(P[:nb] * 49 - np.round(P[:nb] * 49)) <= 0.25 + 1e-5)


def test_gaussian_pulse(naga):
    pts = np.array([[0.5, 0.5], [0.55, 0.5], [0.0, 0.0]], np.float32)
    d = naga.gaussian_pulse(pts, [0.5, 0.5], 1e-3, 0.05)
    ref = 1e-3 * np.exp(-((pts.astype(np.float64) - 0.5) ** 2).sum(1) / (2 * 0.05 ** 2))
    assert np.allclose(d, ref.astype(np.float32), rtol=1e-6, atol=0)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_scene_without_device_fails_loudly(naga):
    g = naga.generate_grid(2, 20, 3, 0)
    with pytest.raises(naga.NagaError) as e:
        naga.Scene(g, k=16)
    assert e.value.code == naga.NAGA_ENODEVICE


def test_scene_argument_validation_precedes_device(naga):
    g = naga.generate_grid(2, 20, 3, 0)
    with pytest.raises(naga.NagaError) as e:
        naga.Scene(g, k=2)
    assert e.value.code == naga.NAGA_EINVAL
    with pytest.raises(naga.NagaError) as e:
        naga.Scene(g, k=16, pml_indexing=5)
    assert e.value.code == naga.NAGA_EINVAL


@pytest.mark.parametrize("name", sorted(f for f in os.listdir(os.path.join(ROOT, "tests", "cpp"))
                                         if f.endswith(".cpp")))
def test_cpp_facade_compiles(name):
    import shutil
    import subprocess

    gxx = shutil.which("g++-13") or shutil.which("g++")
    src = os.path.join(ROOT, "tests", "cpp", name)
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", f"-I{ROOT}/include",
                        "-I/usr/local/cuda/include", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("dim", [2, 3])
def test_library_lattice_matches_oracle(naga, oracle, dim):
    """naga_lattice: the population order and weights the library uses (and
    read_state / write_state expose) are the oracle's, i.e. NAGA's."""
    w, c = naga.lattice(dim)
    oc, ow, _, _ = oracle.lattice(dim)
    assert np.array_equal(c, oc.astype(np.int32))
    assert np.allclose(w, ow, rtol=0, atol=1e-7)


def test_scene_estimate_counts_the_halo_lists(naga):
    """The admission estimate grows linearly with k (stencil records), except
    at k = 32 in 3-D, where the scene also holds the halo lists of its RK
    stages: 17,488 B per 32-node bulk/layer pass."""
    import ctypes as C

    g = naga.generate_grid(3, 20, 3, 1)
    est = {}
    for k in (31, 32, 33):
        d, keep = naga.scene_desc(g, k=k)
        est[k] = naga.lib().naga_scene_estimate_bytes(C.byref(d))
    passes = (g["n_bulk"] + g["n_layer"] + 31) // 32
    linear = (est[31] + est[33]) // 2
    assert est[32] - linear == 17488 * passes
    g2 = naga.generate_grid(2, 30, 3, 1)
    e2 = {}
    for k in (31, 32, 33):
        d, keep = naga.scene_desc(g2, k=k)
        e2[k] = naga.lib().naga_scene_estimate_bytes(C.byref(d))
    assert e2[32] * 2 == e2[31] + e2[33]

"""ctypes binding of the CPU oracle (oracle/libnaga_oracle.so).

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may import this module; the product never
does. `build()` compiles the library from the sources beside this file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnaga_oracle.so")
_lib = None


def build(arch_flags: str = "", out: str | None = None) -> str:
    """Compile the oracle with make; returns the path of the library."""
    out = out or LIB_PATH
    cmd = ["make", "-s", "-C", HERE, f"OUT={out}"]
    if arch_flags:
        cmd.append(f"ARCHFLAGS={arch_flags}")
    subprocess.run(cmd, check=True)
    return out


class SceneDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("k", C.c_int), ("k_boundary", C.c_int), ("k_probe", C.c_int),
        ("shape", C.c_int), ("pml_indexing", C.c_int), ("precision", C.c_int),
        ("n_bulk", C.c_int64), ("n_layer", C.c_int64), ("n_boundary", C.c_int64),
        ("n_ghost", C.c_int64), ("nodal_spacing", C.c_double), ("viscosity", C.c_double),
        ("rho0", C.c_double), ("time_step", C.c_double), ("speed_of_sound", C.c_double),
        ("points", C.c_void_p), ("normals", C.c_void_p), ("sigma", C.c_void_p),
        ("n_probes", C.c_int), ("probes", C.c_void_p),
    ]


def lib(path: str | None = None):
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        build(out=p)
    L = C.CDLL(p)
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    L.orc_knn.argtypes = [vp, i64, vp, i64, i32, i32, i32, vp, vp]
    L.orc_knn_ring_reference.argtypes = [vp, i64, vp, i64, i32, i32, i32, vp, vp]
    L.orc_batched_inverse_f64.argtypes = [vp, i32, i64, vp, vp]
    L.orc_rbf_weights.argtypes = [vp, i64, i32, vp, i32, vp, i64, i32, dbl, i32, vp]
    L.orc_divergence_stencil.argtypes = [vp, i64, i32, i32, i32, vp, vp, vp]
    L.orc_scene_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(vp)]
    L.orc_scene_destroy.argtypes = [vp]
    L.orc_scene_destroy.restype = None
    L.orc_scene_set_density.argtypes = [vp, vp]
    L.orc_scene_step.argtypes = [vp, i32, vp]
    L.orc_scene_step_phase.argtypes = [vp, i32]
    L.orc_scene_read_state.argtypes = [vp, vp, vp]
    L.orc_scene_write_state.argtypes = [vp, vp]
    L.orc_scene_tables.argtypes = [vp] * 8
    L.orc_scene_pml_state.argtypes = [vp, vp, vp]
    L.orc_scene_set_sources.argtypes = [vp, vp, i64, vp, i64]
    L.orc_lattice.argtypes = [i32, vp, vp, vp, vp, vp]
    L.orc_collision.argtypes = [i32, vp, dbl, vp, dbl, dbl, vp]
    L.orc_grid_generate.argtypes = [i32, i64, i32, dbl, dbl, C.c_uint64, vp, vp, vp, vp, vp]
    L.orc_gaussian_pulse.argtypes = [vp, i64, i32, vp, dbl, dbl, vp]
    L.orc_set_threads.argtypes = [i32]
    L.orc_cubic_segmentation.argtypes = [vp, i64, i32, i32] + [vp] * 8
    if path is None:
        _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def set_threads(n: int) -> int:
    """OpenMP threads for the oracle's later calls from this thread (n <= 0
    keeps the current number); returns the number in effect."""
    return lib().orc_set_threads(n)


def generate_grid(dim, n_side, n_layers, seed, jitter=0.25, sigma_peak=0.1):
    """The jittered benchmark grid (orc_grid_generate), as a dict with the
    keys of the scene constructors: points, normals, sigma, class counts, h."""
    counts = np.zeros(3, np.int64)
    h = C.c_double()
    assert lib().orc_grid_generate(dim, n_side, n_layers, jitter, sigma_peak, seed, _p(counts), None,
                                   None, None, C.byref(h)) == 0
    nb, nl, nw = (int(c) for c in counts)
    pts = np.zeros((nb + nl + nw, dim), np.float32)
    nrm = np.zeros((nw, dim), np.float32)
    sig = np.zeros(nl, np.float32)
    assert lib().orc_grid_generate(dim, n_side, n_layers, jitter, sigma_peak, seed, None, _p(pts),
                                   _p(nrm), _p(sig), None) == 0
    return dict(dim=dim, points=pts, n_bulk=nb, n_layer=nl, n_boundary=nw, normals=nrm, sigma=sig,
                h=h.value)


def gaussian_pulse(points, center, amplitude, width):
    pts = np.ascontiguousarray(points, np.float32)
    c = np.ascontiguousarray(center, np.float64)
    out = np.zeros(pts.shape[0], np.float32)
    assert lib().orc_gaussian_pulse(_p(pts), pts.shape[0], pts.shape[1], _p(c), amplitude, width,
                                    _p(out)) == 0
    return out


def knn(src, qry, k, grid=True):
    src = np.ascontiguousarray(src, np.float32)
    qry = np.ascontiguousarray(qry, np.float32)
    dim = src.shape[1]
    idx = np.zeros((qry.shape[0], k), np.uint32)
    d2 = np.zeros((qry.shape[0], k), np.float32)
    rc = lib().orc_knn(_p(src), src.shape[0], _p(qry), qry.shape[0], dim, k, int(grid), _p(idx), _p(d2))
    assert rc == 0, rc
    return idx, d2


def cubic_segmentation(src, approx):
    """NAGA's nd_cubic_segmentation restated: dict of lower, upper, width,
    shape, sizes, offsets, indices (ascending within a partition)."""
    src = np.ascontiguousarray(src, np.float32)
    n, dim = src.shape
    lo, hi, shape = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(3, np.int64)
    w, cells = C.c_float(), C.c_int64()
    assert lib().orc_cubic_segmentation(_p(src), n, dim, approx, _p(lo), _p(hi), C.byref(w), _p(shape),
                                        C.byref(cells), None, None, None) == 0
    sizes = np.zeros(cells.value, np.uint32)
    offsets = np.zeros(cells.value, np.uint32)
    indices = np.zeros(n, np.uint32)
    assert lib().orc_cubic_segmentation(_p(src), n, dim, approx, None, None, None, None, None, _p(sizes),
                                        _p(offsets), _p(indices)) == 0
    return dict(lower=lo[:dim], upper=hi[:dim], width=w.value, shape=shape[:dim], sizes=sizes,
                offsets=offsets, indices=indices)


def knn_ring_reference(src, qry, k, approx=None):
    """NAGA's ring search restated (cells of ~approx points, default k)."""
    src = np.ascontiguousarray(src, np.float32)
    qry = np.ascontiguousarray(qry, np.float32)
    idx = np.zeros((qry.shape[0], k), np.uint32)
    d2 = np.zeros((qry.shape[0], k), np.float32)
    rc = lib().orc_knn_ring_reference(_p(src), src.shape[0], _p(qry), qry.shape[0], src.shape[1], k,
                                      int(approx or k), _p(idx), _p(d2))
    assert rc == 0, rc
    return idx, d2


def batched_inverse(A):
    """A: [batch][n][n] with matrix (i, j) at A[b][j][i] (column-major)."""
    A = np.ascontiguousarray(A, np.float64)
    b, n, _ = A.shape
    out = np.zeros_like(A)
    info = np.zeros(b, np.int32)
    assert lib().orc_batched_inverse_f64(_p(A), n, b, _p(out), _p(info)) == 0
    return out, info


def rbf_weights(src, support, qry, group, spacing, shape):
    src = np.ascontiguousarray(src, np.float32)
    support = np.ascontiguousarray(support, np.uint32)
    qry = np.ascontiguousarray(qry, np.float64)
    ng, k = support.shape
    w = np.zeros((ng * group, k), np.float64)
    rc = lib().orc_rbf_weights(_p(src), src.shape[0], src.shape[1], _p(support), k, _p(qry), ng,
                               group, spacing, shape, _p(w))
    assert rc == 0, rc
    return w


def divergence_stencil(pts, k, shape):
    pts = np.ascontiguousarray(pts, np.float32)
    n, dim = pts.shape
    idx = np.zeros((n, k), np.uint32)
    W = np.zeros((n, k, dim), np.float64)
    delta = np.zeros(n, np.float64)
    rc = lib().orc_divergence_stencil(_p(pts), n, dim, k, shape, _p(idx), _p(W), _p(delta))
    assert rc == 0, rc
    return idx, W, delta


def lattice(dim):
    Q = C.c_int()
    q = 9 if dim == 2 else 27
    c = np.zeros((q, dim)); w = np.zeros(q); bb = np.zeros(q, np.int32); K = np.zeros((q, q))
    assert lib().orc_lattice(dim, C.byref(Q), _p(c), _p(w), _p(bb), _p(K)) == 0
    return c, w, bb, K


def collision(dim, f, rho, u, nu, dt):
    f = np.ascontiguousarray(f, np.float64)
    u = np.ascontiguousarray(u, np.float64)
    df = np.zeros_like(f)
    assert lib().orc_collision(dim, _p(f), rho, _p(u), nu, dt, _p(df)) == 0
    return df


class Scene:
    """FP64 (precision=0) or reference-FP32 (precision=1) oracle scene."""

    def __init__(self, dim, points, n_bulk, n_layer, n_boundary, normals, sigma, h, *,
                 k, k_boundary=None, k_probe=None, shape=1, pml_indexing=0, precision=0,
                 viscosity=1e-5, rho0=1.0, time_step=None, speed_of_sound=1.0, probes=None,
                 n_ghost=0):
        self.dim = dim
        self.Q = 9 if dim == 2 else 27
        self._keep = [np.ascontiguousarray(points, np.float32),
                      np.ascontiguousarray(normals, np.float32).reshape(-1),
                      np.ascontiguousarray(sigma, np.float32),
                      np.ascontiguousarray(probes if probes is not None else np.zeros((0, dim)),
                                           np.float32)]
        self.N = self._keep[0].shape[0]
        self.np_ = self._keep[3].shape[0]
        d = SceneDesc()
        d.dim, d.k = dim, k
        d.k_boundary = k_boundary or k
        d.k_probe = k_probe or k
        d.shape, d.pml_indexing, d.precision = shape, pml_indexing, precision
        d.n_bulk, d.n_layer, d.n_boundary, d.n_ghost = n_bulk, n_layer, n_boundary, n_ghost
        d.nodal_spacing = h
        d.viscosity, d.rho0 = viscosity, rho0
        d.time_step = time_step if time_step is not None else 0.5 * h / speed_of_sound
        d.speed_of_sound = speed_of_sound
        d.points, d.normals, d.sigma, d.probes = (_p(a) for a in self._keep)
        d.n_probes = self.np_
        self.desc = d
        self.h = C.c_void_p()
        rc = lib().orc_scene_create(C.byref(d), C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"orc_scene_create failed: {rc}")

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            lib().orc_scene_destroy(self.h)
            self.h = None

    def set_density(self, drho):
        drho = np.ascontiguousarray(drho, np.float32)
        assert lib().orc_scene_set_density(self.h, _p(drho)) == 0

    def step(self, n):
        out = np.zeros((n, self.np_), np.float64)
        assert lib().orc_scene_step(self.h, n, _p(out)) == 0
        return out

    def phase(self, ph):
        assert lib().orc_scene_step_phase(self.h, ph) == 0

    def state(self):
        g = np.zeros((self.N, self.Q)); r = np.zeros(self.N)
        assert lib().orc_scene_read_state(self.h, _p(g), _p(r)) == 0
        return g, r

    def write_state(self, g):
        g = np.ascontiguousarray(g, np.float64)
        assert lib().orc_scene_write_state(self.h, _p(g)) == 0

    def set_sources(self, nodes, values):
        """Density sources: values [n_steps][len(nodes)] (dimensional
        density, float32 max = no term that step)."""
        nodes = np.ascontiguousarray(nodes, np.int64)
        values = np.ascontiguousarray(values, np.float32).reshape(-1, len(nodes))
        assert lib().orc_scene_set_sources(self.h, _p(nodes), len(nodes), _p(values), values.shape[0]) == 0

    def pml_state(self):
        q1 = np.zeros((self.N, self.Q)); q2 = np.zeros((self.N, self.Q))
        assert lib().orc_scene_pml_state(self.h, _p(q1), _p(q2)) == 0
        return q1, q2

    def tables(self):
        d = self.desc
        k, kb, kp, dim = d.k, d.k_boundary, d.k_probe, self.dim
        idx = np.zeros((self.N, k), np.uint32); W = np.zeros((self.N, k, dim))
        fw = np.zeros((self.N, k)); bidx = np.zeros((d.n_boundary, kb), np.uint32)
        bw = np.zeros((d.n_boundary, kb)); pidx = np.zeros((self.np_, kp), np.uint32)
        pw = np.zeros((self.np_, kp))
        assert lib().orc_scene_tables(self.h, _p(idx), _p(W), _p(fw), _p(bidx), _p(bw), _p(pidx),
                                      _p(pw)) == 0
        return dict(idx=idx, W=W, fw=fw, bidx=bidx, bw=bw, pidx=pidx, pw=pw)

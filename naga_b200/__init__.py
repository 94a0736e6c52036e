"""naga_b200: B200-native nonlocal lattice-Boltzmann acoustics step.

Python binding of the C ABI in include/naga_b200.h (libnaga_b200.so, built
in-tree by naga_b200/_build.py). The names follow NAGA's C++ API
(NAGAGroup/NAGA, fluids/nonlocal_lattice_boltzmann/simulation_engine.cuh):
a `Scene` is one simulation_engine with its domain and density observers; a
`Batch` steps many scenes per launch. There is no CPU fallback: every call
goes to the CUDA library, and importing this module without the built
library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = [
    "NagaError", "lib", "build", "GridSpec", "SceneDesc", "generate_grid", "gaussian_pulse",
    "Scene", "Batch", "knn", "knn_clouds", "batched_inverse_f64", "batched_inverse_f32r",
    "rbf_weights", "divergence_build", "profile", "Q_OF", "lattice_weights", "divergence_build_f32",
    "divergence_apply", "rbf_weights_f32", "rbf_interpolate", "cubic_segmentation",
]

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libnaga_b200.so")

NAGA_OK, NAGA_EINVAL, NAGA_ENOMEM, NAGA_ECUDA = 0, 1, 2, 3
NAGA_ENOCONVERGE, NAGA_ETIMEOUT, NAGA_ESINGULAR, NAGA_ENODEVICE = 4, 5, 6, 7
Q_OF = {2: 9, 3: 27}


class NagaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"naga error {code}: {msg}")
        self.code = code


class GridSpec(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_layers", C.c_int), ("n_side", C.c_int64),
                ("jitter", C.c_double), ("sigma_peak", C.c_double), ("seed", C.c_uint64)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("k", C.c_int), ("k_boundary", C.c_int), ("k_probe", C.c_int),
        ("shape", C.c_int), ("pml_indexing", C.c_int), ("weight_precision", C.c_int),
        ("n_probes", C.c_int),
        ("n_bulk", C.c_int64), ("n_layer", C.c_int64), ("n_boundary", C.c_int64),
        ("n_ghost", C.c_int64),
        ("nodal_spacing", C.c_double), ("viscosity", C.c_double), ("rho0", C.c_double),
        ("time_step", C.c_double), ("speed_of_sound", C.c_double),
        ("points", C.c_void_p), ("normals", C.c_void_p), ("sigma", C.c_void_p),
        ("probes", C.c_void_p), ("probe_capacity", C.c_int),
    ]


_lib = None
_SIGS = {
    "naga_last_error": ([], C.c_char_p),
    "naga_version": ([], C.c_int),
    "naga_grid_counts": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_grid_generate": ([C.c_void_p] * 5, C.c_int),
    "naga_box_grid_counts": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_box_grid_generate": ([C.c_void_p] * 5, C.c_int),
    "naga_gaussian_pulse": ([C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_double, C.c_double,
                             C.c_void_p], C.c_int),
    "naga_knn": ([C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                  C.c_void_p, C.c_void_p], C.c_int),
    "naga_knn_noalloc": ([C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                          C.c_void_p, C.c_void_p], C.c_int),
    "naga_knn_clouds": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                         C.c_void_p], C.c_int),
    "naga_batched_inverse_f64": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p],
                                 C.c_int),
    "naga_batched_inverse_f32r": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_int, C.c_double,
                                   C.c_void_p, C.c_void_p], C.c_int),
    "naga_rbf_weights": ([C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int64,
                          C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "naga_refinement_fallbacks": ([], C.c_int64),
    "naga_divergence_build": ([C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_divergence_apply": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                               C.c_float, C.c_void_p, C.c_void_p], C.c_int),
    "naga_divergence_apply_f64": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                                   C.c_double, C.c_void_p, C.c_void_p], C.c_int),
    "naga_divergence_build_f32": ([C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_rbf_weights_f32": ([C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int64,
                              C.c_int, C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "naga_rbf_interpolate": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_int64,
                              C.c_int, C.c_float, C.c_void_p, C.c_void_p], C.c_int),
    "naga_segmentation_shape": ([C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_segmentation_build": ([C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_float,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_create": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_destroy": ([C.c_void_p], C.c_int),
    "naga_scene_stream": ([C.c_void_p], C.c_void_p),
    "naga_scene_set_density": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_step": ([C.c_void_p, C.c_int], C.c_int),
    "naga_scene_sync": ([C.c_void_p], C.c_int),
    "naga_scene_step_count": ([C.c_void_p], C.c_int64),
    "naga_scene_read_probes": ([C.c_void_p, C.c_int64, C.c_int64, C.c_void_p], C.c_int),
    "naga_scene_read_state": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_write_state": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_read_tables": ([C.c_void_p] * 8, C.c_int),
    "naga_scene_device_bytes": ([C.c_void_p], C.c_int64),
    "naga_scene_size": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_batch_create": ([C.c_int, C.c_void_p], C.c_int),
    "naga_batch_create_with_priority": ([C.c_int, C.c_int, C.c_void_p], C.c_int),
    "naga_selftest_wait_timeout": ([C.c_int], C.c_int),
    "naga_scene_set_params": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double], C.c_int),
    "naga_scene_init_domain": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_set_initial_condition": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_add_probe": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_scene_read_macros": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_lattice": ([C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_batch_destroy": ([C.c_void_p], C.c_int),
    "naga_batch_add": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_batch_remove": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_batch_size": ([C.c_void_p], C.c_int),
    "naga_batch_stream": ([C.c_void_p], C.c_void_p),
    "naga_batch_step": ([C.c_void_p, C.c_int], C.c_int),
    "naga_batch_prepare": ([C.c_void_p], C.c_int),
    "naga_batch_sync": ([C.c_void_p], C.c_int),
    "naga_scene_estimate_bytes": ([C.c_void_p], C.c_int64),
    "naga_server_create": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_server_destroy": ([C.c_void_p], C.c_int),
    "naga_server_submit": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p], C.c_int),
    "naga_server_tick": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "naga_server_request_state": ([C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p], C.c_int),
    "naga_server_result": ([C.c_void_p, C.c_int64, C.c_void_p], C.c_int),
    "naga_server_read_stats": ([C.c_void_p, C.c_void_p], C.c_int),
    "naga_profile_enable": ([C.c_int], C.c_int),
    "naga_tuning_report": ([C.c_char_p, C.c_int64], C.c_int64),
    "naga_scene_snapshot_bytes": ([C.c_void_p], C.c_int64),
    "naga_scene_set_density_source": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64],
                                      C.c_int),
    "naga_scene_save": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "naga_scene_load": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "naga_scene_read_probes_async": ([C.c_void_p, C.c_int64, C.c_int64, C.c_void_p], C.c_int),
    "naga_profile_reset": ([], C.c_int),
    "naga_profile_read": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
}


def build(verbose: bool = False) -> str:
    from . import _build

    return _build.build(verbose=verbose)


def lib():
    """The loaded libnaga_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run naga_b200._build.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != NAGA_OK:
        raise NagaError(rc, lib().naga_last_error().decode())


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lattice(dim: int):
    """(weights [Q] float32, velocities [Q, dim] int32) in the library's
    population order (naga_lattice)."""
    q = C.c_int()
    _check(lib().naga_lattice(dim, C.byref(q), None, None))
    w = np.zeros(q.value, np.float32)
    c = np.zeros((q.value, dim), np.int32)
    _check(lib().naga_lattice(dim, C.byref(q), _p(w), _p(c)))
    return w, c


def lattice_weights(dim: int) -> np.ndarray:
    if dim == 2:
        return np.array([4 / 9, 1 / 36, 1 / 9, 1 / 36, 1 / 9, 1 / 36, 1 / 9, 1 / 36, 1 / 9])
    return np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)


# ------------------------------------------------------------ synthetic input
def generate_grid(dim: int, n_side: int, n_layers: int, seed: int, jitter: float = 0.25,
                  sigma_peak: float = 0.1) -> dict:
    """Jittered unit-grid scene (see naga_grid_generate in include/naga_b200.h)."""
    sp = GridSpec(dim, n_layers, n_side, jitter, sigma_peak, seed)
    nb, nl, nbd = C.c_int64(), C.c_int64(), C.c_int64()
    _check(lib().naga_grid_counts(C.byref(sp), C.byref(nb), C.byref(nl), C.byref(nbd)))
    n = nb.value + nl.value + nbd.value
    pts = np.zeros((n, dim), np.float32)
    nrm = np.zeros((nbd.value, dim), np.float32)
    sig = np.zeros(nl.value, np.float32)
    h = C.c_double()
    _check(lib().naga_grid_generate(C.byref(sp), _p(pts), _p(nrm), _p(sig), C.byref(h)))
    return dict(dim=dim, points=pts, n_bulk=nb.value, n_layer=nl.value, n_boundary=nbd.value,
                normals=nrm, sigma=sig, h=h.value)


class BoxGridSpec(C.Structure):
    _fields_ = [("dim", C.c_int), ("morton", C.c_int), ("min", C.c_double * 3), ("max", C.c_double * 3),
                ("spacing", C.c_double), ("layer_thickness", C.c_double), ("peak_absorption", C.c_double)]


def box_grid(lo, hi, spacing: float, layer_thickness: float = 0.0, peak_absorption: float = 0.0,
             morton: bool = True) -> dict:
    """NAGA's uniform_grid_provider(min, max, grid_spacing, layer_thickness,
    peak_absorption_rate): see naga_box_grid_generate in include/naga_b200.h."""
    dim = len(lo)
    sp = BoxGridSpec()
    sp.dim, sp.morton = dim, int(bool(morton))
    for d in range(3):
        sp.min[d] = float(lo[d]) if d < dim else 0.0
        sp.max[d] = float(hi[d]) if d < dim else 1.0
    sp.spacing, sp.layer_thickness, sp.peak_absorption = spacing, layer_thickness, peak_absorption
    nb, nl, nbd = C.c_int64(), C.c_int64(), C.c_int64()
    _check(lib().naga_box_grid_counts(C.byref(sp), C.byref(nb), C.byref(nl), C.byref(nbd)))
    n = nb.value + nl.value + nbd.value
    pts = np.zeros((n, dim), np.float32)
    nrm = np.zeros((nbd.value, dim), np.float32)
    sig = np.zeros(nl.value, np.float32)
    h = C.c_double()
    _check(lib().naga_box_grid_generate(C.byref(sp), _p(pts), _p(nrm), _p(sig), C.byref(h)))
    return dict(dim=dim, points=pts, n_bulk=nb.value, n_layer=nl.value, n_boundary=nbd.value,
                normals=nrm, sigma=sig, h=h.value)


def gaussian_pulse(points: np.ndarray, center, amplitude: float, width: float) -> np.ndarray:
    pts = np.ascontiguousarray(points, np.float32)
    c = np.ascontiguousarray(center, np.float64)
    out = np.zeros(pts.shape[0], np.float32)
    _check(lib().naga_gaussian_pulse(_p(pts), pts.shape[0], pts.shape[1], _p(c), amplitude, width,
                                     _p(out)))
    return out


# ---------------------------------------------------------------- scenes
class Scene:
    """One acoustic scene: NAGA's simulation_engine<Lattice> after
    set_problem_parameters + init_domain, with density observers (probes)."""

    def __init__(self, grid: dict, *, k: int, k_boundary: int | None = None,
                 k_probe: int | None = None, shape: int = 1, pml_indexing: int = 0,
                 weight_precision: int = 0, viscosity: float = 1e-5, rho0: float = 1.0,
                 time_step: float | None = None, speed_of_sound: float = 1.0, probes=None,
                 probe_capacity: int = 4096, n_ghost: int = 0):
        dim = grid["dim"]
        self.dim, self.Q = dim, Q_OF[dim]
        self._keep = [np.ascontiguousarray(grid["points"], np.float32),
                      np.ascontiguousarray(grid["normals"], np.float32),
                      np.ascontiguousarray(grid["sigma"], np.float32),
                      np.ascontiguousarray(probes if probes is not None else np.zeros((0, dim)),
                                           np.float32)]
        self.N = self._keep[0].shape[0]
        self.n_probes = self._keep[3].shape[0]
        d = SceneDesc()
        d.dim, d.k = dim, k
        d.k_boundary = k_boundary or k
        d.k_probe = k_probe or k
        d.shape, d.pml_indexing, d.weight_precision = shape, pml_indexing, weight_precision
        d.n_probes = self.n_probes
        d.n_bulk, d.n_layer, d.n_boundary = grid["n_bulk"], grid["n_layer"], grid["n_boundary"]
        d.n_ghost = n_ghost
        d.nodal_spacing = grid["h"]
        d.viscosity, d.rho0, d.speed_of_sound = viscosity, rho0, speed_of_sound
        d.time_step = time_step if time_step is not None else 0.5 * grid["h"] / speed_of_sound
        d.points, d.normals, d.sigma, d.probes = (_p(a) for a in self._keep)
        d.probe_capacity = probe_capacity
        self.desc = d
        self.h = C.c_void_p()
        _check(lib().naga_scene_create(C.byref(d), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().naga_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_density(self, drho=None):
        if drho is None:
            _check(lib().naga_scene_set_density(self.h, None))
        else:
            drho = np.ascontiguousarray(drho, np.float32)
            assert drho.shape == (self.N,)
            _check(lib().naga_scene_set_density(self.h, _p(drho)))

    def set_initial_condition(self, drho=None):
        """naga_scene_set_initial_condition (the same as set_density)."""
        drho = None if drho is None else np.ascontiguousarray(drho, np.float32)
        _check(lib().naga_scene_set_initial_condition(self.h, _p(drho)))

    def set_params(self, viscosity: float, rho0: float, time_step: float, speed_of_sound: float):
        """simulation_engine::set_problem_parameters on the existing scene."""
        _check(lib().naga_scene_set_params(self.h, viscosity, rho0, time_step, speed_of_sound))

    def init_domain(self, grid: dict, **kw):
        """simulation_engine::init_domain on this handle (rebuilt from grid)."""
        d, keep = scene_desc(grid, **kw)
        _check(lib().naga_scene_init_domain(self.h, C.byref(d)))
        self._keep, self.desc = keep, d
        self.dim, self.Q = grid["dim"], Q_OF[grid["dim"]]
        self.N = keep[0].shape[0]
        self.n_probes = d.n_probes

    def macros(self):
        """(density [N], velocity [N, dim]) as NAGA's solution() holds them
        (dimensional; computed at the start of the last step)."""
        rho = np.zeros(self.N, np.float32)
        u = np.zeros((self.N, self.dim), np.float32)
        _check(lib().naga_scene_read_macros(self.h, _p(rho), _p(u)))
        return rho, u

    def add_probe(self, xyz) -> int:
        """Attach one more density probe; returns its index."""
        x = np.ascontiguousarray(xyz, np.float32).reshape(self.dim)
        idx = C.c_int()
        _check(lib().naga_scene_add_probe(self.h, _p(x), C.byref(idx)))
        self.n_probes += 1
        return idx.value

    def step(self, n: int = 1):
        _check(lib().naga_scene_step(self.h, n))

    def sync(self):
        _check(lib().naga_scene_sync(self.h))

    @property
    def step_count(self) -> int:
        return lib().naga_scene_step_count(self.h)

    @property
    def stream(self) -> int:
        return lib().naga_scene_stream(self.h) or 0

    def probes(self, first: int = 0, count: int | None = None) -> np.ndarray:
        if count is None:
            count = self.step_count - first
        out = np.zeros((count, self.n_probes), np.float32)
        _check(lib().naga_scene_read_probes(self.h, first, count, _p(out)))
        return out

    def set_density_source(self, nodes, values, first_step: int = 0) -> None:
        """Density sources: values [n_steps][len(nodes)] (dimensional density,
        float32 max = no term that step) for steps first_step, first_step + 1,
        ...; see naga_scene_set_density_source."""
        nodes = np.ascontiguousarray(nodes, np.int64)
        values = np.ascontiguousarray(values, np.float32).reshape(-1, max(len(nodes), 1))
        _check(lib().naga_scene_set_density_source(self.h, _p(nodes), len(nodes), _p(values), first_step,
                                                   values.shape[0] if len(nodes) else 0))

    def save(self) -> bytes:
        """Snapshot of the dynamic state (naga_scene_save)."""
        n = lib().naga_scene_snapshot_bytes(self.h)
        buf = C.create_string_buffer(int(n))
        _check(lib().naga_scene_save(self.h, buf, n))
        return buf.raw

    def load(self, snapshot: bytes) -> None:
        """Resume from a snapshot of a scene with the same description."""
        _check(lib().naga_scene_load(self.h, snapshot, len(snapshot)))

    def probes_async(self, first: int, count: int, out) -> None:
        """Enqueue the copy of steps [first, first + count) to host address
        `out` (>= count * n_probes floats, ideally page-locked, kept alive
        until the next sync); returns at once."""
        _check(lib().naga_scene_read_probes_async(self.h, first, count, C.c_void_p(int(out))))

    def state(self):
        g = np.zeros((self.N, self.Q), np.float32)
        r = np.zeros(self.N, np.float32)
        _check(lib().naga_scene_read_state(self.h, _p(g), _p(r)))
        return g, r

    def write_state(self, g):
        g = np.ascontiguousarray(g, np.float32)
        _check(lib().naga_scene_write_state(self.h, _p(g)))

    def tables(self) -> dict:
        d = self.desc
        k, kb, kp, dim = d.k, d.k_boundary, d.k_probe, self.dim
        out = dict(idx=np.zeros((self.N, k), np.uint32), W=np.zeros((self.N, k, dim), np.float32),
                   fw=np.zeros((self.N, k), np.float32),
                   bidx=np.zeros((d.n_boundary, kb), np.uint32),
                   bw=np.zeros((d.n_boundary, kb), np.float32),
                   pidx=np.zeros((self.n_probes, kp), np.uint32),
                   pw=np.zeros((self.n_probes, kp), np.float32))
        _check(lib().naga_scene_read_tables(self.h, *(_p(out[n]) for n in
                                                      ("idx", "W", "fw", "bidx", "bw", "pidx", "pw"))))
        return out

    @property
    def device_bytes(self) -> int:
        return lib().naga_scene_device_bytes(self.h)


class Batch:
    """Many scenes of one lattice, stepped together (one launch per kernel)."""

    def __init__(self, dim: int, priority: int = 0):
        self.h = C.c_void_p()
        self.scenes: list[Scene] = []
        _check(lib().naga_batch_create_with_priority(dim, priority, C.byref(self.h)))

    def add(self, s: Scene):
        _check(lib().naga_batch_add(self.h, s.h))
        self.scenes.append(s)

    def remove(self, s: Scene):
        _check(lib().naga_batch_remove(self.h, s.h))
        self.scenes.remove(s)

    def prepare(self):
        """Apply membership changes now (rebuild, shape tuning, graph capture)."""
        _check(lib().naga_batch_prepare(self.h))

    def step(self, n: int = 1):
        _check(lib().naga_batch_step(self.h, n))

    def sync(self):
        _check(lib().naga_batch_sync(self.h))

    @property
    def stream(self) -> int:
        return lib().naga_batch_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().naga_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- serving
class ServerConfig(C.Structure):
    _fields_ = [("dim", C.c_int), ("steps_per_tick", C.c_int), ("max_active", C.c_int),
                ("step_priority", C.c_int), ("memory_budget", C.c_int64), ("target_step_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("ticks", C.c_int64), ("steps", C.c_int64), ("node_updates", C.c_int64),
                ("busy_ms", C.c_double), ("p50_step_ms", C.c_double), ("p99_step_ms", C.c_double),
                ("bytes_in_use", C.c_int64), ("peak_bytes", C.c_int64), ("done", C.c_int64),
                ("failed", C.c_int64), ("active", C.c_int), ("queued", C.c_int),
                ("prepare_ms", C.c_double), ("admit_ms", C.c_double), ("wait_ms", C.c_double),
                ("retire_ms", C.c_double), ("p50_request_ms", C.c_double), ("p99_request_ms", C.c_double),
                ("p50_queue_ms", C.c_double), ("admitted", C.c_int64)]


def scene_desc(grid: dict, *, k: int, k_boundary=None, k_probe=None, shape=1, pml_indexing=0,
               weight_precision=0, viscosity=1e-5, rho0=1.0, time_step=None, speed_of_sound=1.0,
               probes=None, probe_capacity=4096, n_ghost=0):
    """A naga_scene_desc for `grid`; returns (desc, arrays it points into)."""
    dim = grid["dim"]
    keep = [np.ascontiguousarray(grid["points"], np.float32),
            np.ascontiguousarray(grid["normals"], np.float32),
            np.ascontiguousarray(grid["sigma"], np.float32),
            np.ascontiguousarray(probes if probes is not None else np.zeros((0, dim)), np.float32)]
    d = SceneDesc()
    d.dim, d.k = dim, k
    d.k_boundary = k_boundary or k
    d.k_probe = k_probe or k
    d.shape, d.pml_indexing, d.weight_precision = shape, pml_indexing, weight_precision
    d.n_probes = keep[3].shape[0]
    d.n_bulk, d.n_layer, d.n_boundary = grid["n_bulk"], grid["n_layer"], grid["n_boundary"]
    d.n_ghost = n_ghost
    d.nodal_spacing = grid["h"]
    d.viscosity, d.rho0, d.speed_of_sound = viscosity, rho0, speed_of_sound
    d.time_step = time_step if time_step is not None else 0.5 * grid["h"] / speed_of_sound
    d.points, d.normals, d.sigma, d.probes = (_p(a) for a in keep)
    d.probe_capacity = probe_capacity
    return d, keep


class Server:
    """Continuous-batching request loop (naga_server_* in include/naga_b200.h)."""

    QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, dim: int, memory_budget: int, steps_per_tick: int = 50, max_active: int = 0,
                 step_priority: int = 0, target_step_ms: float = 0.0):
        self.h = C.c_void_p()
        cfg = ServerConfig(dim, steps_per_tick, max_active, step_priority, memory_budget, target_step_ms)
        _check(lib().naga_server_create(C.byref(cfg), C.byref(self.h)))
        self.n_probes = {}

    def submit(self, grid: dict, drho, steps: int, **kw) -> int:
        d, keep = scene_desc(grid, **kw)
        rid = C.c_int64()
        drho = None if drho is None else np.ascontiguousarray(drho, np.float32)
        _check(lib().naga_server_submit(self.h, C.byref(d), _p(drho), steps, C.byref(rid)))
        self.n_probes[rid.value] = (d.n_probes, steps)
        return rid.value

    def tick(self):
        a, q = C.c_int(), C.c_int()
        _check(lib().naga_server_tick(self.h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def state(self, rid: int):
        st, done = C.c_int(), C.c_int64()
        _check(lib().naga_server_request_state(self.h, rid, C.byref(st), C.byref(done)))
        return st.value, done.value

    def result(self, rid: int) -> np.ndarray:
        np_, steps = self.n_probes.pop(rid)
        out = np.zeros((steps, np_), np.float32)
        _check(lib().naga_server_result(self.h, rid, _p(out)))
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().naga_server_read_stats(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().naga_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------- primitives
# Device buffers are torch CUDA tensors (plumbing only); results are torch
# tensors on the same device.
def _torch():
    import torch

    return torch


def _dptr(t):
    return C.c_void_p(t.data_ptr())


def _stream_ptr():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def knn(src, qry, k: int):
    """Exact kNN (device tensors [n][dim] float32) -> (idx int32 [nq][k], d2)."""
    torch = _torch()
    src = src.contiguous().float()
    qry = qry.contiguous().float()
    idx = torch.empty((qry.shape[0], k), dtype=torch.int32, device=src.device)
    d2 = torch.empty((qry.shape[0], k), dtype=torch.float32, device=src.device)
    _check(lib().naga_knn(_dptr(src), src.shape[0], _dptr(qry), qry.shape[0], src.shape[1], k,
                          _dptr(idx), _dptr(d2), _stream_ptr()))
    return idx, d2


def knn_clouds(pts, offsets, k: int):
    torch = _torch()
    pts = pts.contiguous().float()
    off = np.ascontiguousarray(offsets, np.int64)
    idx = torch.empty((pts.shape[0], k), dtype=torch.int32, device=pts.device)
    d2 = torch.empty((pts.shape[0], k), dtype=torch.float32, device=pts.device)
    _check(lib().naga_knn_clouds(_dptr(pts), _p(off), len(off) - 1, pts.shape[1], k, _dptr(idx),
                                 _dptr(d2), _stream_ptr()))
    return idx, d2


def batched_inverse_f64(A):
    """A: device float64 [batch][n][n] with element (i, j) at A[b, j, i]."""
    torch = _torch()
    A = A.contiguous()
    out = torch.empty_like(A)
    info = torch.empty(A.shape[0], dtype=torch.int32, device=A.device)
    _check(lib().naga_batched_inverse_f64(_dptr(A), _dptr(out), A.shape[1], A.shape[0], _dptr(info),
                                          _stream_ptr()))
    return out, info


def batched_inverse_f32r(A, max_iter: int = 20, rel_tol: float = 1e-14):
    torch = _torch()
    A = A.contiguous()
    out = torch.empty_like(A)
    info = torch.empty(A.shape[0], dtype=torch.int32, device=A.device)
    _check(lib().naga_batched_inverse_f32r(_dptr(A), _dptr(out), A.shape[1], A.shape[0], max_iter,
                                           rel_tol, _dptr(info), _stream_ptr()))
    return out, info


def rbf_weights(src, support, qry, group: int, spacing: float, shape: int, precision: int = 0):
    torch = _torch()
    src = src.contiguous().float()
    support = support.contiguous().to(torch.int32)
    qry = qry.contiguous().double()
    ng, k = support.shape
    w = torch.empty((ng * group, k), dtype=torch.float64, device=src.device)
    _check(lib().naga_rbf_weights(_dptr(src), src.shape[0], src.shape[1], _dptr(support), k,
                                  _dptr(qry), ng, group, spacing, shape, precision, _dptr(w),
                                  _stream_ptr()))
    return w


def refinement_fallbacks() -> int:
    """Systems of this thread's last refined-precision solve re-done in FP64."""
    return int(lib().naga_refinement_fallbacks())


def divergence_build(pts, k: int, shape: int, precision: int = 0):
    torch = _torch()
    pts = pts.contiguous().float()
    n, dim = pts.shape
    idx = torch.empty((n, k), dtype=torch.int32, device=pts.device)
    W = torch.empty((n, k, dim), dtype=torch.float64, device=pts.device)
    delta = torch.empty(n, dtype=torch.float64, device=pts.device)
    _check(lib().naga_divergence_build(_dptr(pts), n, dim, k, shape, precision, _dptr(idx), _dptr(W),
                                       _dptr(delta), _stream_ptr()))
    return idx, W, delta


def divergence_build_f32(pts, k: int, shape: int, precision: int = 0):
    """The stencil with FP32 outputs: (idx int32 [n][k], W float32 [n][k][dim],
    delta float32 [n])."""
    torch = _torch()
    pts = pts.contiguous().float()
    n, dim = pts.shape
    idx = torch.empty((n, k), dtype=torch.int32, device=pts.device)
    W = torch.empty((n, k, dim), dtype=torch.float32, device=pts.device)
    delta = torch.empty(n, dtype=torch.float32, device=pts.device)
    _check(lib().naga_divergence_build_f32(_dptr(pts), n, dim, k, shape, precision, _dptr(idx), _dptr(W),
                                           _dptr(delta), _stream_ptr()))
    return idx, W, delta


def divergence_apply(W, idx, field, centering_offset: float = 0.0):
    """divergence_operator::apply: result_i = sum_s sum_d W[i, s, d]
    (field[idx[i, s], d] - offset); FP32 or FP64 by W's dtype."""
    torch = _torch()
    W = W.contiguous()
    idx = idx.contiguous().to(torch.int32)
    field = field.contiguous().to(W.dtype)
    n, k, dim = W.shape
    out = torch.empty(n, dtype=W.dtype, device=W.device)
    fn = lib().naga_divergence_apply_f64 if W.dtype == torch.float64 else lib().naga_divergence_apply
    _check(fn(_dptr(W), _dptr(idx), n, dim, k, _dptr(field), centering_offset, _dptr(out), _stream_ptr()))
    return out


def rbf_weights_f32(src, support, qry, group: int, spacing: float, shape: int, precision: int = 0):
    """RBF weights with FP32 queries and outputs (FP64 solves)."""
    torch = _torch()
    src = src.contiguous().float()
    support = support.contiguous().to(torch.int32)
    qry = qry.contiguous().float()
    ng, k = support.shape
    w = torch.empty((ng * group, k), dtype=torch.float32, device=src.device)
    _check(lib().naga_rbf_weights_f32(_dptr(src), src.shape[0], src.shape[1], _dptr(support), k, _dptr(qry),
                                      ng, group, spacing, shape, precision, _dptr(w), _stream_ptr()))
    return w


def rbf_interpolate(weights, support, field, group: int = 1, centering_offset: float = 0.0):
    """radial_point_method::interpolate: field [n_src] or [n_src][c] float32
    -> [nq] or [nq][c]."""
    torch = _torch()
    weights = weights.contiguous().float()
    support = support.contiguous().to(torch.int32)
    one = field.dim() == 1
    f = field.contiguous().float().reshape(field.shape[0], -1)
    nq, k = weights.shape
    out = torch.empty((nq, f.shape[1]), dtype=torch.float32, device=f.device)
    _check(lib().naga_rbf_interpolate(_dptr(weights), _dptr(support), nq, group, k, _dptr(f), f.shape[0],
                                      f.shape[1], centering_offset, _dptr(out), _stream_ptr()))
    return out[:, 0] if one else out


def cubic_segmentation(pts, approx_partition_size: int) -> dict:
    """NAGA's nd_cubic_segmentation of a device point cloud [n][dim]: bounds,
    width, shape and (device) partition sizes, offsets and indices."""
    torch = _torch()
    pts = pts.contiguous().float()
    n, dim = pts.shape
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    w = C.c_float()
    shape = np.zeros(3, np.int64)
    _check(lib().naga_segmentation_shape(_dptr(pts), n, dim, approx_partition_size, _p(lo), _p(hi), C.byref(w),
                                         _p(shape), _stream_ptr()))
    cells = int(np.prod(shape[:dim]))
    sizes = torch.empty(cells, dtype=torch.int32, device=pts.device)
    offsets = torch.empty(cells, dtype=torch.int32, device=pts.device)
    indices = torch.empty(n, dtype=torch.int32, device=pts.device)
    _check(lib().naga_segmentation_build(_dptr(pts), n, dim, _p(lo), _p(hi), w.value, _p(shape), _dptr(sizes),
                                         _dptr(offsets), _dptr(indices), _stream_ptr()))
    return dict(lower=lo[:dim].copy(), upper=hi[:dim].copy(), width=w.value, shape=shape[:dim].copy(),
                sizes=sizes, offsets=offsets, indices=indices)


class profile:
    """Per-kernel CUDA-event timing of the step kernels (context manager)."""

    def __enter__(self):
        _check(lib().naga_profile_enable(1))
        _check(lib().naga_profile_reset())
        return self

    def __exit__(self, *exc):
        self.result = read_profile()
        lib().naga_profile_enable(0)
        return False


def read_profile() -> dict:
    n = C.c_int(64)
    names = (C.c_char_p * 64)()
    launches = np.zeros(64, np.int64)
    ms = np.zeros(64, np.float64)
    _check(lib().naga_profile_read(C.byref(n), names, _p(launches), _p(ms)))
    return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(n.value)}


def selftest_wait_timeout(polls: int = 0) -> int:
    """Runs the step kernels' bounded device wait on a barrier that nothing
    completes (0 polls = their own limit); returns the status, NAGA_ETIMEOUT
    when the wait gave up and was reported."""
    return int(lib().naga_selftest_wait_timeout(int(polls)))


def tuning_report() -> str:
    """The launch-shape tuner's log (one line per tuned batch shape)."""
    n = lib().naga_tuning_report(None, 0)
    buf = C.create_string_buffer(int(n) + 1)
    lib().naga_tuning_report(buf, n + 1)
    return buf.value.decode()

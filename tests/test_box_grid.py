"""NAGA's uniform_grid_provider restated (naga_box_grid_generate): the box
grid, node classes, inward normals and absorption profile against a NumPy
restatement of node_providers/uniform_grid_provider.cuh:53-161,
detail/uniform_grid_provider.inl:38-171 and ranges/uniform_grid.cuh:58-64,
243-293 in FP32. Host code only: no GPU."""
import numpy as np
import pytest

f32 = np.float32


def reference_box(lo, hi, h, L, peak):
    """[bulk, layer, boundary] in grid order (x fastest), FP32."""
    dim = len(lo)
    lo = np.array(lo, f32)
    ext = np.array(hi, f32) - lo
    n = (np.ceil(ext / f32(h)) + 1).astype(np.int64)
    sp = (ext / (n - 1).astype(f32)).astype(f32)
    idx = np.arange(int(np.prod(n)))
    grid = np.zeros((idx.size, dim), np.int64)
    r = idx.copy()
    for d in range(dim):
        grid[:, d] = r % n[d]
        r //= n[d]
    x = (lo + grid.astype(f32) * sp).astype(f32)
    top = (lo + (n - 1).astype(f32) * sp).astype(f32)
    bnd = ((grid == 0) | (grid == n - 1)).any(1)
    d2 = np.minimum((x - lo) * (x - lo), (x - top) * (x - top)).astype(f32).min(1)
    layer = (~bnd) & (f32(L) > 0) & (d2 <= f32(L) * f32(L))
    bulk = (~bnd) & (~layer)
    nv = np.where(grid == 0, f32(-1), np.where(grid == n - 1, f32(1), f32(0))).astype(f32)
    nn = np.sqrt((nv * nv).sum(1)).astype(f32)
    normals = -(nv / np.where(nn == 0, f32(1), nn)[:, None]).astype(f32)
    dl = np.sqrt(d2[layer]).astype(f32)
    sigma = (f32(peak) * ((f32(L) - dl) / f32(L)) ** 2).astype(f32)
    pts = np.concatenate([x[bulk], x[layer], x[bnd]])
    return dict(points=pts, n_bulk=int(bulk.sum()), n_layer=int(layer.sum()), n_boundary=int(bnd.sum()),
                normals=normals[bnd], sigma=sigma)


CASES = [([0.0, 0.0], [1.0, 0.7], 0.05, 0.2, 0.1),
         ([-0.5, 0.25], [0.5, 1.0], 0.033, 0.1, 0.3),
         ([0.0, 0.0, 0.0], [1.0, 0.6, 0.8], 0.07, 0.21, 0.1),
         ([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], 0.1, 0.0, 0.0)]


@pytest.mark.parametrize("lo,hi,h,L,peak", CASES)
def test_box_grid_grid_order_matches_reference(naga, lo, hi, h, L, peak):
    got = naga.box_grid(lo, hi, h, L, peak, morton=False)
    ref = reference_box(lo, hi, h, L, peak)
    for key in ("n_bulk", "n_layer", "n_boundary"):
        assert got[key] == ref[key], key
    assert np.array_equal(got["points"], ref["points"])
    assert np.array_equal(got["normals"], ref["normals"])
    assert np.array_equal(got["sigma"], ref["sigma"])
    assert got["h"] == pytest.approx(h)


@pytest.mark.parametrize("lo,hi,h,L,peak", CASES)
def test_box_grid_morton_order_is_a_permutation_within_classes(naga, lo, hi, h, L, peak):
    got = naga.box_grid(lo, hi, h, L, peak)
    ref = reference_box(lo, hi, h, L, peak)
    nb, nl = ref["n_bulk"], ref["n_layer"]
    cls = [(0, nb), (nb, nb + nl), (nb + nl, len(ref["points"]))]

    def rows(a, b, arr, extra=None):
        m = arr[a:b] if extra is None else np.concatenate([arr[a:b], extra], 1)
        return m[np.lexsort(m.T[::-1])]

    for c, (a, b) in enumerate(cls):
        ex_g = ex_r = None
        if c == 1:
            ex_g, ex_r = got["sigma"][:, None], ref["sigma"][:, None]
        if c == 2:
            ex_g, ex_r = got["normals"], ref["normals"]
        assert np.array_equal(rows(a, b, got["points"], ex_g), rows(a, b, ref["points"], ex_r))


def test_box_grid_rejects_degenerate_boxes(naga):
    with pytest.raises(naga.NagaError):
        naga.box_grid([0.0, 0.0], [0.0, 1.0], 0.1)
    with pytest.raises(naga.NagaError):
        naga.box_grid([0.0, 0.0], [1.0, 1.0], -0.1)


def test_facade_uniform_grid_provider_compiles():
    import os
    import shutil
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = ("#include <naga/naga.hpp>\nusing namespace naga::fluids::nonlocal_lbm;\n"
           "int main() { uniform_grid_provider<d3q27_lattice<float>> p({0.f, 0.f, 0.f}, {1.f, 0.5f, 1.f}, "
           "0.05f, 0.2f, 0.1f); return p.get().num_layer_points > 0 ? 0 : 1; }\n")
    gxx = shutil.which("g++-13") or shutil.which("g++")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-x", "c++", "-", f"-I{root}/include",
                        "-I/usr/local/cuda/include"], input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

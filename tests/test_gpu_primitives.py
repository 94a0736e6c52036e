"""GPU set-up primitives through the C ABI against the CPU oracle:
bit-exact kNN, batched inverses, RBF weights and the divergence stencil."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _np(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def _cloud(dim, seed):
    rng = np.random.default_rng(seed)
    m = 9 if dim == 3 else 30
    lat = np.stack(np.meshgrid(*[np.arange(m)] * dim, indexing="ij"), -1).reshape(-1, dim) / m
    pts = np.concatenate([lat, rng.random((3000, dim)), lat[:20]]).astype(np.float32)
    qry = np.concatenate([pts[::5], rng.random((300, dim)) * 1.4 - 0.2]).astype(np.float32)
    return pts, qry


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("k", [1, 16, 32, 48, 64])
def test_knn_bit_exact(naga, oracle, dim, k):
    pts, qry = _cloud(dim, 10 + dim)
    idx, d2 = naga.knn(_t(pts), _t(qry), k)
    oi, od = oracle.knn(pts, qry, k)
    assert np.array_equal(_np(idx).view(np.uint32), oi)
    assert np.array_equal(_np(d2), od)


def test_knn_golden_validation_grid(naga, golden_dir):
    g = json.load(open(os.path.join(golden_dir, "knn_validation_3d.json")))
    n1, h, k = g["grid_size"], np.float32(g["spacing"]), g["k"]
    i = np.arange(n1 ** 3)
    grid = np.stack([(i % n1).astype(np.float32) * h, ((i // n1) % n1).astype(np.float32) * h,
                     (i // n1 // n1).astype(np.float32) * h], 1).astype(np.float32)
    idx, _ = naga.knn(_t(grid), _t(np.array(g["queries"], np.float32)), k)
    assert np.array_equal(_np(idx), np.array(g["neighbours"], np.int32))


def test_knn_clouds_batched(naga, oracle):
    rng = np.random.default_rng(5)
    sizes = [40, 500, 3000, 64, 1200]
    clouds = [rng.random((n, 3)).astype(np.float32) for n in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)])
    idx, d2 = naga.knn_clouds(_t(np.concatenate(clouds)), off, 32)
    idx, d2 = _np(idx), _np(d2)
    for c, pts in enumerate(clouds):
        oi, od = oracle.knn(pts, pts, 32)
        assert np.array_equal(idx[off[c]:off[c + 1]].view(np.uint32), oi)
        assert np.array_equal(d2[off[c]:off[c + 1]], od)


def test_inverse_golden(naga, golden_dir):
    g = json.load(open(os.path.join(golden_dir, "inverse_3x3.json")))
    A = np.repeat(np.array(g["A"]).T[None], 1000, 0)
    out, info = naga.batched_inverse_f64(_t(A))
    out = _np(out)
    assert (_np(info) == 0).all()
    assert np.abs(out.transpose(0, 2, 1) - np.array(g["A_inv"])[None]).max() <= g["tol"]


def _rbf_systems(n_sys, seed=0):
    """36 x 36 augmented PHS r^3 moment matrices of random k = 32 stencils in
    a jittered cube, centred and scaled as the library assembles them."""
    rng = np.random.default_rng(seed)
    pts = rng.random((20000, 3)).astype(np.float32)
    from oracle import oracle as O

    centres = rng.integers(0, len(pts), n_sys)
    idx, _ = O.knn(pts, pts[centres], 32)
    X = pts.astype(np.float64)[idx] - pts.astype(np.float64)[centres][:, None]
    X /= np.abs(X).max(axis=(1, 2), keepdims=True)
    r = np.sqrt(((X[:, :, None] - X[:, None]) ** 2).sum(-1))
    G = np.zeros((n_sys, 36, 36))
    G[:, :32, :32] = r ** 3
    G[:, :32, 32] = G[:, 32, :32] = 1
    G[:, :32, 33:] = X
    G[:, 33:, :32] = X.transpose(0, 2, 1)
    return G  # symmetric: column-major storage equals row-major


def _assert_inverse_close(out, ref, A):
    """A stable inverse is accurate to a small multiple of eps * cond(A)
    (relative, max-norm). The GPU kernels (LU for most sizes, register
    Gauss-Jordan for the stencil sizes) and the oracle's LU round
    differently, so they agree to that bound rather than bit for bit; the
    largest ratio seen over these batches is about 0.6."""
    kappa = np.linalg.cond(A)
    err = np.abs(out - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))
    assert (err <= 4 * np.finfo(np.float64).eps * kappa).all(), float((err / kappa).max())


@pytest.mark.parametrize("n", [3, 19, 20, 35, 36, 64])
def test_inverse_matches_oracle(naga, oracle, n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((300, n, n)) + 3 * np.eye(n)
    out, info = naga.batched_inverse_f64(_t(A))
    ref, rinfo = oracle.batched_inverse(A)
    assert (_np(info) == 0).all()
    _assert_inverse_close(_np(out), ref, A)


def test_inverse_rbf_systems_f64_and_refined(naga, oracle):
    A = _rbf_systems(500)
    ref, _ = oracle.batched_inverse(A)
    out, info = naga.batched_inverse_f64(_t(A))
    e64 = np.abs(_np(out) - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))
    assert (_np(info) == 0).all() and e64.max() < 1e-9
    outr, infor = naga.batched_inverse_f32r(_t(A), max_iter=30, rel_tol=1e-14)
    er = np.abs(_np(outr) - ref).max(axis=(1, 2)) / np.abs(ref).max(axis=(1, 2))
    # kappa ~ 1e4: FP32 LU + FP64 residuals converges to the FP64 floor
    assert (_np(infor) == 0).all()
    assert er.max() < 1e-10


def test_inverse_refined_flags_hopeless_systems(naga):
    """Condition ~1e12 is beyond FP32 refinement: flagged (-1), not silent."""
    rng = np.random.default_rng(1)
    n = 12
    U, _ = np.linalg.qr(rng.standard_normal((n, n)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (U @ np.diag(np.logspace(0, -12, n)) @ V.T)[None].repeat(4, 0)
    _, info = naga.batched_inverse_f32r(_t(A.transpose(0, 2, 1).copy()), max_iter=10)
    assert (_np(info) == -1).all()


@pytest.mark.parametrize("dim,shape,precision", [(2, 0, 0), (2, 1, 0), (3, 0, 0), (3, 1, 0), (3, 1, 1)])
def test_rbf_weights_match_oracle(naga, oracle, dim, shape, precision):
    rng = np.random.default_rng(dim * 10 + shape)
    m = 14 if dim == 3 else 40
    h = 1.0 / (m - 1)
    g = np.stack(np.meshgrid(*[np.arange(m) * h] * dim, indexing="ij"), -1).reshape(-1, dim)
    pts = (g + rng.uniform(-0.25 * h, 0.25 * h, g.shape)).astype(np.float32)
    k = 32 if dim == 3 else 16
    qry = rng.random((400, dim)) * 0.9 + 0.05
    sup, _ = oracle.knn(pts, qry.astype(np.float32), k)
    w = _np(naga.rbf_weights(_t(pts), _t(sup.astype(np.int32)), _t(qry), 1, h, shape, precision))
    ref = oracle.rbf_weights(pts, sup, qry, 1, h, shape)
    err = np.abs(w - ref).max() / np.abs(ref).max()
    assert err < 1e-10
    if precision == 1:
        # refined FP32 solves converge here; none needed the FP64 fallback
        assert naga.refinement_fallbacks() == 0


@pytest.mark.parametrize("dim,shape", [(2, 1), (3, 0), (3, 1)])
def test_divergence_stencil_matches_oracle(naga, oracle, dim, shape):
    m = 14 if dim == 3 else 40
    rng = np.random.default_rng(7)
    h = 1.0 / (m - 1)
    g = np.stack(np.meshgrid(*[np.arange(m) * h] * dim, indexing="ij"), -1).reshape(-1, dim)
    pts = (g + rng.uniform(-0.25 * h, 0.25 * h, g.shape)).astype(np.float32)
    k = 32 if dim == 3 else 16
    idx, W, delta = naga.divergence_build(_t(pts), k, shape)
    oi, oW, od = oracle.divergence_stencil(pts, k, shape)
    assert np.array_equal(_np(idx).view(np.uint32), oi)
    err = np.abs(_np(W) - oW).max() / np.abs(oW).max()
    assert err < 1e-9
    assert np.abs(_np(delta) - od).max() / od.max() < 1e-14


@pytest.mark.parametrize("dim", [2, 3])
def test_knn_edge_sizes(naga, oracle, dim):
    """No queries; a source cloud smaller than k (the slots past the n
    sources hold index 0xffffffff and d2 = +inf, as the oracle; NAGA warns
    and leaves them unset, nearest_neighbors.cuh:421-425); one source."""
    import torch

    rng = np.random.default_rng(dim)
    pts = rng.random((500, dim)).astype(np.float32)
    idx, d2 = naga.knn(_t(pts), torch.empty((0, dim), device="cuda"), 16)
    assert tuple(idx.shape) == (0, 16) and tuple(d2.shape) == (0, 16)
    for n, k in ((5, 16), (1, 4), (16, 16)):
        src, qry = pts[:n], rng.random((40, dim)).astype(np.float32)
        idx, d2 = naga.knn(_t(src), _t(qry), k)
        oi, od = oracle.knn(src, qry, k)
        assert np.array_equal(_np(idx).view(np.uint32), oi)
        assert np.array_equal(_np(d2), od)
        assert (oi[:, n:] == 0xFFFFFFFF).all() and np.isinf(od[:, n:]).all()


def test_nonfinite_coordinates_are_rejected(naga):
    """NaN or infinite point coordinates are an input error (NAGA_EINVAL)
    found at the kNN's bounding box, before any search or stencil kernel
    sees them: plain and batched kNN, the divergence build and scene
    creation; the context stays usable."""
    rng = np.random.default_rng(5)
    pts = rng.random((2000, 3)).astype(np.float32)
    for bad in (np.nan, np.inf, -np.inf):
        p = pts.copy()
        p[123, 1] = bad
        with pytest.raises(naga.NagaError, match="non-finite"):
            naga.knn(_t(p), _t(pts[:10]), 8)
        with pytest.raises(naga.NagaError, match="non-finite"):
            naga.knn_clouds(_t(np.concatenate([pts[:500], p[:300]])), np.array([0, 500, 800]), 8)
        with pytest.raises(naga.NagaError, match="non-finite"):
            naga.divergence_build(_t(p), 32, 0)
    g = naga.generate_grid(2, 30, 4, 0)
    g["points"][7, 0] = np.nan
    with pytest.raises(naga.NagaError, match="non-finite"):
        naga.Scene(g, k=16)
    idx, _ = naga.knn(_t(pts), _t(pts[:10]), 8)
    assert (_np(idx)[:, 0] == np.arange(10)).all()


def test_knn_clouds_ragged(naga, oracle):
    """Clouds back to back with an empty cloud and clouds smaller than k
    between full ones: each equals its own search."""
    rng = np.random.default_rng(11)
    sizes = [300, 0, 7, 1, 900, 0, 40]
    clouds = [rng.random((n, 3)).astype(np.float32) for n in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)])
    idx, d2 = naga.knn_clouds(_t(np.concatenate(clouds)), off, 32)
    idx, d2 = _np(idx), _np(d2)
    for c, pts in enumerate(clouds):
        if len(pts) == 0:
            continue
        oi, od = oracle.knn(pts, pts, 32)
        assert np.array_equal(idx[off[c]:off[c + 1]].view(np.uint32), oi)
        assert np.array_equal(d2[off[c]:off[c + 1]], od)


def test_inverse_singular_and_empty(naga, oracle):
    """A matrix with an exactly zero column reports the LAPACK info (the
    1-based column of the zero pivot) like the oracle; its neighbours in
    the batch are unaffected; an empty batch is a no-op."""
    import torch

    rng = np.random.default_rng(3)
    n = 9
    A = rng.standard_normal((6, n, n)) + 3 * np.eye(n)
    A[2, 4, :] = 0.0  # column 5 of matrix 2 (element (i, j) at A[b, j, i])
    out, info = naga.batched_inverse_f64(_t(A))
    ref, rinfo = oracle.batched_inverse(A)
    info = _np(info)
    assert info[2] == rinfo[2] and info[2] > 0
    ok = [b for b in range(6) if b != 2]
    assert (info[ok] == 0).all()
    assert np.abs(_np(out)[ok] - ref[ok]).max() / np.abs(ref[ok]).max() < 1e-12
    out0, info0 = naga.batched_inverse_f64(torch.empty((0, n, n), dtype=torch.float64, device="cuda"))
    assert tuple(out0.shape) == (0, n, n) and tuple(info0.shape) == (0,)


@pytest.mark.parametrize("n", [9, 36])
def test_inverse_nan_matrices_leave_the_batch_intact(naga, oracle, n):
    """Matrices with NaN entries (all of them, or one) in the middle of a
    batch: their results are not finite and their neighbours still match
    the oracle, on the shared-memory LU (n = 9) and the register
    Gauss-Jordan kernel (n = 36)."""
    rng = np.random.default_rng(n + 1)
    A = rng.standard_normal((5, n, n)) + 3 * np.eye(n)
    A[1] = np.nan
    A[3, 2, 5] = np.nan
    out, info = naga.batched_inverse_f64(_t(A))
    out, info = _np(out), _np(info)
    ok = [0, 2, 4]
    ref, _ = oracle.batched_inverse(A[ok])
    assert (info[ok] == 0).all()
    _assert_inverse_close(out[ok], ref, A[ok])
    assert not np.isfinite(out[1]).any() and not np.isfinite(out[3]).all()


@pytest.mark.parametrize("n", [19, 36])
def test_inverse_register_sizes_singular_and_ties(naga, oracle, n):
    """The stencil sizes take the register Gauss-Jordan kernel: a zero
    column reports getrf's info; integer matrices (many equal |a| pivot
    candidates) and a batch that is not a multiple of the warps per block
    still match the oracle."""
    rng = np.random.default_rng(n)
    A = rng.standard_normal((7, n, n)) + 3 * np.eye(n)
    A[2, n // 2, :] = 0.0  # column n/2 + 1 of matrix 2
    A[4] = np.round(2 * A[4])
    A[5] = rng.integers(-2, 3, (n, n)) + 6 * np.eye(n)
    out, info = naga.batched_inverse_f64(_t(A))
    ref, rinfo = oracle.batched_inverse(A)
    info = _np(info)
    assert info[2] == rinfo[2] == n // 2 + 1
    ok = [b for b in range(7) if b != 2]
    assert (info[ok] == 0).all()
    _assert_inverse_close(_np(out)[ok], ref[ok], A[ok])


def _jittered_box(dim, m, L, seed=0):
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(m)] * dim, indexing="ij"), -1).reshape(-1, dim).astype(np.float64)
    h = L / (m - 1)
    pts = g * h + rng.uniform(-0.25 * h, 0.25 * h, g.shape)
    return pts.astype(np.float32), h


@pytest.mark.parametrize("dim,shape", [(2, 1), (3, 0)])
def test_divergence_apply_matches_oracle_and_analytic_fields(naga, oracle, dim, shape):
    """naga_divergence_apply (FP32) and naga_divergence_apply_f64 against the
    FP64 oracle's stencil applied in FP64, on NAGA's known-answer field
    (examples/nonlocal_divergence_3d.cu:40-51: F = (sin x, 0, cos z), div F =
    cos x - sin z; 2-D: F = (sin x, cos y)) over a jittered grid of
    [0, 2 pi]^dim; the FP32 stencil comes from naga_divergence_build_f32."""
    L = 2 * np.pi
    m = 16 if dim == 3 else 40
    k = 32 if dim == 3 else 16
    pts, h = _jittered_box(dim, m, L)
    P = pts.astype(np.float64)
    if dim == 3:
        F = np.stack([np.sin(P[:, 0]), 0 * P[:, 0], np.cos(P[:, 2])], -1)
        exact = np.cos(P[:, 0]) - np.sin(P[:, 2])
    else:
        F = np.stack([np.sin(P[:, 0]), np.cos(P[:, 1])], -1)
        exact = np.cos(P[:, 0]) - np.sin(P[:, 1])
    oi, oW, _ = oracle.divergence_stencil(pts, k, shape)
    ref = np.einsum("nsd,nsd->n", oW, F[oi])
    scale = np.abs(ref).max()
    # FP32 stencil and FP32 apply
    idx, W, delta = naga.divergence_build_f32(_t(pts), k, shape)
    assert np.array_equal(_np(idx).view(np.uint32), oi)
    assert np.abs(_np(W) - oW).max() <= 1e-6 * np.abs(oW).max()
    got = _np(naga.divergence_apply(W, idx, _t(F.astype(np.float32))))
    assert np.abs(got - ref).max() <= 2e-5 * scale
    inner = np.all((P > 3 * h) & (P < L - 3 * h), axis=1)
    err = np.linalg.norm(got[inner] - exact[inner]) / np.linalg.norm(exact[inner])
    assert err < 0.08
    # the oracle's FP64 stencil through the FP64 apply
    got64 = _np(naga.divergence_apply(_t(oW), _t(oi.view(np.int32)), _t(F)))
    assert np.abs(got64 - ref).max() <= 1e-12 * scale
    # centring offset: apply(F, c) == apply(F - c)
    c = 0.75
    a = _np(naga.divergence_apply(_t(oW), _t(oi.view(np.int32)), _t(F), centering_offset=c))
    b = _np(naga.divergence_apply(_t(oW), _t(oi.view(np.int32)), _t(F - c)))
    assert np.abs(a - b).max() <= 1e-12 * scale
    assert np.abs(a - np.einsum("nsd,nsd->n", oW, F[oi] - c)).max() <= 1e-12 * scale


def test_divergence_apply_summation_order(naga):
    """The FP32 apply sums the per-support terms by NAGA's pairwise tree
    (divergence.cuh:452-468), not left to right: checked on values whose
    FP32 sum depends on the order, k = 32 and k = 20."""
    rng = np.random.default_rng(5)
    for k in (32, 20):
        n = 64
        W = np.zeros((n, k, 3), np.float32)
        W[:, :, 0] = rng.choice([1.0, 1e8, -1e8, 3.0], size=(n, k)).astype(np.float32)
        idx = np.zeros((n, k), np.int32)
        F = np.ones((1, 3), np.float32)
        got = _np(naga.divergence_apply(_t(W), _t(idx), _t(F)))
        t = W[:, :, 0].copy()
        s = 1
        while s < k:
            for j in range(0, k, 2 * s):
                if j + s < k:
                    t[:, j] = t[:, j] + t[:, j + s]
            s *= 2
        assert np.array_equal(got, t[:, 0].astype(np.float32)), k


def test_rbf_weights_f32_and_interpolate(naga, oracle):
    """radial_point_method<float>: weights from FP32 queries, and interpolate
    (one field and three components, with a centring offset) against the FP64
    oracle, on NAGA's known-answer field (examples/
    radial_point_interpolation_3d.cu:48-50: sin x cos y z over [0, 2 pi]^3)."""
    L = 2 * np.pi
    src, h = _jittered_box(3, 14, L, seed=3)
    rng = np.random.default_rng(4)
    qry = (rng.random((2000, 3)) * (L - 2 * h) + h).astype(np.float32)
    sup, _ = naga.knn(_t(src), _t(qry), 32)
    sup_np = _np(sup).view(np.uint32)
    for shape in (0, 1):
        w32 = naga.rbf_weights_f32(_t(src), sup, _t(qry), 1, h, shape)
        ow = oracle.rbf_weights(src, sup_np, qry.astype(np.float64), 1, h, shape)
        assert np.abs(_np(w32) - ow).max() <= 1e-6 * np.abs(ow).max()
        S = src.astype(np.float64)
        f = np.sin(S[:, 0]) * np.cos(S[:, 1]) * S[:, 2]
        ref = np.einsum("qs,qs->q", ow, f[sup_np])
        got = _np(naga.rbf_interpolate(w32, sup, _t(f.astype(np.float32))))
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(f).max()
        Q = qry.astype(np.float64)
        exact = np.sin(Q[:, 0]) * np.cos(Q[:, 1]) * Q[:, 2]
        assert np.sqrt(np.mean((got - exact) ** 2)) < 0.05 * np.abs(exact).max()
        F3 = np.stack([f, 2 * f, f + 1.0], -1)
        got3 = _np(naga.rbf_interpolate(w32, sup, _t(F3.astype(np.float32)), centering_offset=1.0))
        ref3 = np.einsum("qs,qsc->qc", ow, F3[sup_np] - 1.0) + 1.0
        assert np.abs(got3 - ref3).max() <= 2e-5 * np.abs(F3).max()


def test_rbf_interpolate_groups(naga, oracle):
    """group_size > 1: queries q share the support list of group q / group."""
    src, h = _jittered_box(2, 30, 1.0, seed=6)
    rng = np.random.default_rng(7)
    centres = (rng.random((50, 2)) * 0.8 + 0.1).astype(np.float32)
    sup, _ = naga.knn(_t(src), _t(centres), 16)
    qry = (np.repeat(centres, 4, 0) + rng.normal(0, 0.2 * h, (200, 2))).astype(np.float32)
    w32 = naga.rbf_weights_f32(_t(src), sup, _t(qry), 4, h, 1)
    sup_np = _np(sup).view(np.uint32)
    ow = oracle.rbf_weights(src, sup_np, qry.astype(np.float64), 4, h, 1)
    assert np.abs(_np(w32) - ow).max() <= 1e-6 * np.abs(ow).max()
    f = src[:, 0].astype(np.float64) ** 2 - src[:, 1]
    got = _np(naga.rbf_interpolate(w32, sup, _t(f.astype(np.float32)), group=4))
    ref = np.einsum("qs,qs->q", ow, f[np.repeat(sup_np, 4, 0)])
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(f).max()


def _seg_clouds():
    rng = np.random.default_rng(8)
    flat = rng.random((3000, 3)).astype(np.float32)
    flat[:, 2] = 0.25  # a plane: the thin axis is widened to 1e-3
    shifted = (rng.random((4000, 2)) * 7.0 - 3.0).astype(np.float32)
    return [("grid3", _jittered_box(3, 20, 1.0, seed=9)[0], 32), ("rand2", shifted, 16),
            ("flat3", flat, 32), ("one", shifted, 1), ("big", shifted, 1000),
            ("single", shifted[:1].copy(), 8)]


@pytest.mark.parametrize("case", range(6))
def test_cubic_segmentation_matches_oracle(naga, oracle, case):
    """NAGA's nd_cubic_segmentation on the device against its FP32
    restatement on the CPU: bounds, width, shape, partition sizes, offsets
    and the grouped indices, bit for bit."""
    name, pts, approx = _seg_clouds()[case]
    g = naga.cubic_segmentation(_t(pts), approx)
    o = oracle.cubic_segmentation(pts, approx)
    for key in ("lower", "upper", "shape"):
        assert np.array_equal(g[key], o[key]), (name, key)
    assert np.float32(g["width"]) == np.float32(o["width"]), name
    assert np.array_equal(_np(g["sizes"]).view(np.uint32), o["sizes"]), name
    assert np.array_equal(_np(g["offsets"]).view(np.uint32), o["offsets"]), name
    assert np.array_equal(_np(g["indices"]).view(np.uint32), o["indices"]), name

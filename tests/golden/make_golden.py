"""Generates the golden fixtures in tests/golden/ from NAGA's known-answer
programs. Run where the reference tree is available, giving its path:

    python tests/golden/make_golden.py <path-to-NAGA-checkout>

Fixtures written:
  inverse_3x3.json     the 3x3 matrix and its hard-coded inverse from
                       examples/batched_matrix_inversion.cu:47-70 (tol 1e-6)
  knn_validation_3d.json
                       the 20^3 grid (spacing 0.1) and the 30 query points of
                       examples/knn_validation_3d.cu:36-83, reproduced with a
                       restatement of thrust's minstd_rand (x <- 48271 x mod
                       2^31 - 1, seed 1, discard(i)) and uniform_real_distribution
                       ((x - 1) / 2^31 scaled to [0, 1.9)), plus their exact
                       k = 64 neighbour sets by brute force under the
                       (dist^2, index) order (the program checks set equality
                       against a KD-tree, :84-139)
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _floats(txt: str) -> list[float]:
    return [float(v) for v in re.findall(r"-?\d+\.\d*(?:e-?\d+)?|-?\d+\.", txt)]


def inverse_fixture(ref: str) -> dict:
    src = open(os.path.join(ref, "examples", "batched_matrix_inversion.cu")).read()
    a = src[src.index("float A[3][3]"):src.index("float A_inv_check")]
    b = src[src.index("float A_inv_check"):src.index("// clang-format on")]
    A = np.array(_floats(a.split("=", 1)[1])).reshape(3, 3)
    Ainv = np.array(_floats(b.split("=", 1)[1])).reshape(3, 3)
    tol = float(re.search(r"float tol\s*=\s*([0-9.e-]+)", src).group(1))
    return {"source": "examples/batched_matrix_inversion.cu:47-70", "A": A.tolist(),
            "A_inv": Ainv.tolist(), "tol": tol}


def minstd_uniform(idx: int, n: int, lo: np.float32, hi: np.float32) -> list[np.float32]:
    """thrust::default_random_engine rng; rng.discard(idx); n draws of
    uniform_real_distribution<float>(lo, hi)."""
    m = 2147483647
    x = pow(48271, idx, m)  # seed 1, then discard(idx)
    out = []
    for _ in range(n):
        x = (48271 * x) % m
        r = np.float32(x - 1) / (np.float32(1) + np.float32(m - 1 - 1))
        out.append(np.float32(r * (hi - lo) + lo))
    return out


def d2_ref(q: np.ndarray, p: np.ndarray) -> np.ndarray:
    """FP32 squared distances, highest dimension added last."""
    d = (q[None, :] - p).astype(np.float32)
    sq = (d * d).astype(np.float32)
    s = sq[:, 0]
    for k in range(1, sq.shape[1]):
        s = (sq[:, k] + s).astype(np.float32)
    return s


def knn_fixture(ref: str) -> dict:
    src = open(os.path.join(ref, "examples", "knn_validation_3d.cu")).read()
    grid_size = int(re.search(r"size_t grid_size\s*=\s*(\d+)", src).group(1))
    spacing = np.float32(float(re.search(r"float grid_spacing\s*=\s*([0-9.]+)", src).group(1)))
    k = int(re.search(r"uint k\s*=\s*(\d+)", src).group(1))
    nq = int(re.search(r"size_t num_query_points\s*=\s*(\d+)", src).group(1))
    n = grid_size ** 3
    i = np.arange(n)
    grid = np.stack([(i % grid_size).astype(np.float32) * spacing,
                     ((i // grid_size) % grid_size).astype(np.float32) * spacing,
                     (i // grid_size // grid_size).astype(np.float32) * spacing], 1).astype(np.float32)
    hi = np.float32(spacing * np.float32(grid_size - 1))
    # rng.discard(idx) then three draws: the stream position of query t is t
    qry = np.array([minstd_uniform(t, 3, np.float32(0), hi) for t in range(nq)], np.float32)
    idx = []
    for q in qry:
        d2 = d2_ref(q, grid)
        order = np.lexsort((np.arange(n), d2))[:k]
        idx.append(order.tolist())
    return {"source": "examples/knn_validation_3d.cu:36-141", "grid_size": grid_size,
            "spacing": float(spacing), "k": k, "queries": qry.tolist(), "neighbours": idx}


def main(ref: str) -> None:
    with open(os.path.join(HERE, "inverse_3x3.json"), "w") as f:
        json.dump(inverse_fixture(ref), f, indent=1)
    with open(os.path.join(HERE, "knn_validation_3d.json"), "w") as f:
        json.dump(knn_fixture(ref), f)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path-to-NAGA-checkout>")
    main(sys.argv[1])

"""Generates the FP64-oracle probe trace of the 3-D benchmark scene.

    python tests/golden/make_config2_trace.py [--steps 1000] [--threads N]

Scene: 63^3 = 250,047 points in the unit cube (regular grid, h = 1/62,
interior coordinates jittered by U(-h/4, h/4), seed 1), 8-layer PML
(sigma_peak 0.1), k = 32, multiquadric RBF, FP64 weight solves, Gaussian
pulse of amplitude 1e-3 and width 0.05 at the centre, u = 0,
nu = 1e-5, rho0 = 1, c = 1, dt = 0.5 h / c, 8 probes at the corners of
[0.35, 0.65]^3. The CPU oracle (oracle/, FP64 throughout) steps it and
records the probe densities (rho - rho0) sampled at the start of every step.

Written: tests/golden/trace_d3q27_63.npz with
  probes   [steps][8] float64   the oracle's trace
  sha256   hex digest of the scene inputs (points, normals, sigma, pulse),
           so a test can check that it builds the same scene
  desc     a one-line description of the configuration

The grid comes from the oracle's own generator (orc_grid_generate), which
the CPU tests check bit for bit against the library's naga_grid_generate.
This takes about half an hour on 8 cores.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

PROBES3 = np.array([[x, y, z] for z in (0.35, 0.65) for y in (0.35, 0.65) for x in (0.35, 0.65)],
                   np.float32)
OUT = os.path.join(HERE, "trace_d3q27_63.npz")
DESC = ("D3Q27 63^3 jittered grid seed 1, 8-layer PML sigma_peak 0.1, k=32, MQ RBF, FP64 weights, "
        "pulse 1e-3 width 0.05 at the centre, nu=1e-5, rho0=1, c=1, dt=0.5h, 8 probes, FP64 oracle")


def scene_hash(g: dict, drho: np.ndarray) -> str:
    h = hashlib.sha256()
    for a in (g["points"], g["normals"], g["sigma"], drho):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    h.update(np.array([g["n_bulk"], g["n_layer"], g["n_boundary"]], np.int64).tobytes())
    return h.hexdigest()


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args()
    if args.threads:
        os.environ["OMP_NUM_THREADS"] = str(args.threads)
    from oracle import oracle

    g = oracle.generate_grid(3, 63, 8, 1)
    drho = oracle.gaussian_pulse(g["points"], [0.5, 0.5, 0.5], 1e-3, 0.05)
    digest = scene_hash(g, drho)
    t0 = time.time()
    S = oracle.Scene(3, g["points"], g["n_bulk"], g["n_layer"], g["n_boundary"], g["normals"],
                     g["sigma"], g["h"], k=32, shape=0, precision=0, probes=PROBES3)
    S.set_density(drho)
    print(f"set-up {time.time() - t0:.1f} s, {S.N} nodes", flush=True)
    out = np.zeros((args.steps, len(PROBES3)))
    done = 0
    while done < args.steps:
        n = min(50, args.steps - done)
        out[done:done + n] = S.step(n)
        done += n
        print(f"{done} steps, {time.time() - t0:.0f} s, max |probe| {np.abs(out[:done]).max():.3e}",
              flush=True)
    np.savez_compressed(args.out, probes=out, sha256=np.array(digest), desc=np.array(DESC))
    print(f"wrote {args.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Micro-benchmark of ws_render_particles (WaterScene.updateParticles,
js/scene.js:1595-1922) on seeded particles shaped like the 128^3 planet's:
n particles spread over a 128^3 box in cell order, every flag class or
liquid only, the lit-planet scene in beads mode with the camera two box
widths out. Prints one JSON line: time per call (the four kernels, the count
read-back and the synchronisation), points drawn and the algorithmic bytes
per second (26 bytes read per particle, 36 written per drawn point).

    python watersim-v1_b200/render_bench.py [--particles N] [--mix] [--calls K]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from fluid_solver import FluidSolver, render_opts  # noqa: E402


def particles(n, W, mix, seed=3):
    r = np.random.default_rng(seed)
    px, py, pz = (r.uniform(0, W, n).astype(np.float32) for _ in range(3))
    o = np.lexsort((px, py, pz))                      # cell order, like the solver's particles
    flags = r.integers(0, 6, n) if mix else np.zeros(n)
    return {"px": px[o], "py": py[o], "pz": pz[o], "pflag": flags.astype(np.uint8),
            "pT": r.uniform(0, 1, n).astype(np.float32), "pLight": r.uniform(0, 1, n).astype(np.float32),
            "pDepth": r.integers(0, 5, n).astype(np.uint8), "pPh": r.uniform(-3, 3, n).astype(np.float32)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=1856640)
    ap.add_argument("--mix", action="store_true", help="all six flag classes instead of liquid only")
    ap.add_argument("--calls", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    n, W = a.particles, 128.0
    fs = FluidSolver(nx=128, ny=128, nz=128, dx=1.0, coreR=40, targetParticles=1000, capacity=n + 64)
    fs.set_scalars(nP=n)
    fs.upload_state(particles(n, W, a.mix), count=n)
    opts = render_opts(beadsMode=1, cam=(0.5 * W, 0.5 * W, -2.0 * W), sunDir=(0.6, 0.0, 0.8))
    for _ in range(a.warmup):
        fs.render_particles(opts, download=False)
    t0 = time.perf_counter()
    for _ in range(a.calls):
        counts, pts = fs.render_particles(opts, download=False)
    ms = (time.perf_counter() - t0) / a.calls * 1000
    algo = 26 * n + 36 * pts
    print(json.dumps({"particles": n, "points": pts, "counts": counts, "mix": a.mix, "ms_per_call": ms,
                      "algorithmic_bytes": algo, "achieved_gbs": algo / (ms * 1e6)}))


if __name__ == "__main__":
    main()

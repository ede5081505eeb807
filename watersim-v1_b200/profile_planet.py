"""Runs the 128^3 benchmark planet (1.86M particles) through a few substeps,
for capturing one kernel under a profiler with few launches before it and
about 1.5 GB on the device:

    python watersim-v1_b200/profile_planet.py [--substeps N] [--learned]

--learned records two (input, converged q) pairs, takes one Adam step and
then runs the substeps with the learned warm start, so its convolutions run
in every substep. Prints the SOR iterations and fluid cells of the last
substep.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
import bench  # noqa: E402  (the benchmark planet and its knobs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--substeps", type=int, default=3)
    ap.add_argument("--learned", action="store_true")
    a = ap.parse_args()
    fs = bench.make_solver(0)
    if a.learned:
        fs.unet_init(7)
        fs.unet_collect(2)
        fs._substep(bench.DT)
        fs._substep(bench.DT)
        fs.unet_collect(0)
        fs.unet_train(1, 1, 1e-3, 1)
        fs.unet_enable(1)
    for _ in range(a.substeps):
        fs._substep(bench.DT)
    fs.synchronize()
    s = fs.scalars
    print("substeps %d learned %d sor_iterations %d fluid_cells %d" % (a.substeps, a.learned, s.sorIters, s.nFluid))


if __name__ == "__main__":
    main()

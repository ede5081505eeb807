"""The colour-list solve on a grid too large for the temporal-blocked one
(256^3 planet, sea-level radius 110, ocean 12 deep: about 680k fluid cells,
more than one cell per thread and colour). There each CTA sweeps a
contiguous range of each colour list and, between half-sweeps, waits only for
the CTAs owning other-colour cells within one z-plane of its range. Its q after
a fixed number of iterations must equal, bit for bit, the same red-black
iterations run as separate colour launches (one kernel per half-sweep, so
every half-sweep sees the whole previous one): the same cells, the same
update arithmetic, the same order of colours."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ITERS = 24


def test_list_solve_with_neighbour_waits_planet256():
    from fluid_solver import FluidSolver
    fs = FluidSolver(nx=256, ny=256, nz=256, dx=1.0, coreR=98.0, terrainSeed=20260114,
                     targetParticles=4.0e6, capacity=4_300_000)
    fs.generateTerrain(20260114, 110.0)
    fs.resetWater(12.0)
    fs.set_params(pic=0.05, omega=1.7, maxSpeed=3.2, cfl=3.0, viscosity=5e-4, thermalOn=0,
                  sorTol=0.0, pressureIters=ITERS)
    fs.set_scalars(gRamp=1.5)
    fs._substep(0.01)
    for st in ("CLEAR_RASTER", "MARK_FLUID", "P2G"):
        fs.stage(st)
    fs.stage("FORCES", 0.01)
    q0 = fs.q.copy()
    q0[fs.cellType != 1] = 0.0           # as the pressure setup leaves q off the fluid
    fs.stage("PRESSURE")                 # setup + the list solve
    s = fs.scalars
    assert s.sorPath == 1                # the grid-wide list solve
    assert s.nFluid > 2 * 148 * 1024     # more cells per colour than threads: the range-per-CTA loop
    assert s.sorIters == ITERS
    q_list = fs.q.copy()
    fs.upload("q", q0)
    fs.time_kernel(0, ITERS)             # ITERS red-black iterations, one launch per colour
    q_colour = fs.q.copy()
    assert np.all(np.isfinite(q_list))
    assert np.any(q_list != q0)
    assert np.array_equal(q_list.view(np.uint32), q_colour.view(np.uint32))
    fs.close()

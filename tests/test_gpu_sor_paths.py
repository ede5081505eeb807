"""The pressure solve's paths against each other and against the oracle.

Default path (sorPath 3): the temporal-blocked solve on every SM (ws_sor_tb.cu):
each CTA keeps a shared-memory region of its owned bricks plus a four-cell
halo and runs two iterations between exchanges with its neighbours. Its
iterates must be bitwise those of the colour-list solves (sorPath 1 grid-wide,
2 cluster-resident), which ws_time_kernel id 7 runs on the same system.
When a region does not fit in shared memory the same launch falls back to
red-black sweeps over the owned bricks in global memory (sorPath 4): the deep
128^3 ocean below (240k fluid cells) takes it.

Bars: q bitwise equal between paths after a fixed number of iterations; after
one substep against the oracle (device order), cell types bit-exact, q and
face velocities within 1e-5 relative."""
import numpy as np
import pytest

from helpers import planet, to_device, rel_err, DEVICE_ORDER, PLAIN32
from oracle.oracle import make_planet

pytestmark = pytest.mark.gpu


def _system(fs, dt=0.01):
    """Stages up to the pressure solve: the solve's inputs are then fixed."""
    for st in ("CLEAR_RASTER", "MARK_FLUID", "P2G"):
        fs.stage(st)
    fs.stage("FORCES", dt)


def _paths_bitwise(fs, iters):
    fs.set_params(sorTol=0.0, pressureIters=iters)
    _system(fs)
    q0 = fs.q.copy()
    q0[fs.cellType != 1] = 0.0           # as the pressure setup leaves q off the fluid
    fs.stage("PRESSURE")
    path = fs.scalars.sorPath
    q_default = fs.q.copy()
    fs.upload("q", q0)
    fs.time_kernel(7, 1)                 # the colour-list solve of the same system
    q_lists = fs.q.copy()
    assert np.all(np.isfinite(q_default))
    assert np.array_equal(q_default.view(np.uint32), q_lists.view(np.uint32))
    return path


@pytest.mark.parametrize("iters", [1, 7, 40])
def test_temporal_blocked_equals_cluster_solve_planet32(iters):
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    fs._substep(0.01)                     # a warm q to start from
    assert _paths_bitwise(fs, iters) == 3
    fs.close()


def test_temporal_blocked_equals_cluster_solve_planet128():
    o = planet("planet128", pic=0.05, omega=1.7, maxSpeed=3.2, cfl=3.0, thermalOn=0)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    fs.stir_gaussian(4.0, 2.0)
    fs._substep(0.01)
    assert _paths_bitwise(fs, 40) == 3
    fs.close()


def test_deep_ocean_fallback_matches_oracle_and_lists():
    o = make_planet(128, R=56.0, depth=24.0, particles=1200000)
    o.set(**DEVICE_ORDER)
    o.set(**PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    o.substep(0.01)
    fs._substep(0.01)
    s = fs.scalars
    assert s.sorPath in (3, 4)
    assert s.nFluid == o.scalars.nFluid and s.nFluid > 2 * 16 * 4095
    assert np.array_equal(fs.cellType, o.cellType)
    assert rel_err(fs.q, o.q) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_err(fs.download(k), o.arr(k)) <= 1e-5, k
    _paths_bitwise(fs, 40)               # grid-wide list solve (more fluid than one cluster holds)
    fs.close()

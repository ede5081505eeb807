"""Balls (addBall, js/solver.js:3910) on the device against the oracle's
restatement of the reference's ball coupling: the moving-solid raster
(_rasterizeStatic :918-938), solid-velocity boundary faces (_applyBC
:1153-1170), particle push-out (_pushBallsChunk :1009-1026) and the ball
integration (_updateBalls :2344-2564, _ballVsTerrain :2299-2342).

After one substep from the same state: cell types and particle flags
bit-exact, particle and grid state within the substep bar (1e-5), ball
positions within 1e-6 of the box and ball velocities within 1e-4 relative
(they integrate forces from the FP32 grid). After ten substeps the balls stay
within 1e-4 of the box. Run level: a light ball floats part-submerged, a
heavy ball sinks."""
import math

import numpy as np
import pytest

from fluid_solver import WsError
from helpers import planet, to_device, rel_err, PLAIN32

pytestmark = pytest.mark.gpu


def ocean_dirs(o, count):
    """Unit directions whose sea-level point lies over deep ocean."""
    c = o.nx * o.dx / 2
    R = o.scalars.oceanR
    out = []
    r = np.random.default_rng(2)
    while len(out) < count:
        v = r.normal(size=3)
        v /= np.linalg.norm(v)
        if o.terrain_radius_at(c + v[0] * R, c + v[1] * R, c + v[2] * R) < R - 2.5:
            out.append(v)
    return c, R, out


def ball_set(o):
    c, R, d = ocean_dirs(o, 4)
    t = np.cross(d[3], [0.0, 1.0, 0.0]); t /= np.linalg.norm(t)
    p4 = c + d[3] * (R + 0.5)
    return [
        (*(c + d[0] * R), 1.2, 500.0),            # light: floats half out
        (*(c + d[1] * (R - 1.5)), 1.0, 2500.0),   # heavy: underwater, sinks
        (*(c + d[2] * (R + 2.0)), 1.0, 900.0),    # above the water, falls in
        (*p4, 0.9, 700.0),                        # an overlapping pair: ball-ball contact
        (*(p4 + t * 1.5), 0.9, 1100.0),
    ]


def with_balls():
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    for b in ball_set(o):
        o.add_ball(*b)
        fs.add_ball(*b)
    return o, fs


def compare_balls(o, fs, pos_tol, vel_tol):
    a, b = fs.balls, o.balls()
    assert a.shape == b.shape
    W = o.nx * o.dx
    assert np.max(np.abs(a[:, :3] - b[:, :3])) <= pos_tol * W
    for k in range(3, 6):
        assert abs(a[:, k] - b[:, k]).max() <= vel_tol * max(np.abs(b[:, 3:6]).max(), 1e-3), k
    assert np.array_equal(a[:, 6:8], b[:, 6:8])
    assert np.max(np.abs(a[:, 8] - b[:, 8])) <= 1e-4


@pytest.mark.parametrize("cell_order", [0, 1])
def test_balls_one_substep(cell_order):
    """cell_order 1 also covers the cell-ordered P2G's direct path for the
    particles a ball pushed out of the cell they were binned in."""
    o, fs = with_balls()
    fs.set_params(p2gCellOrder=cell_order)
    o.substep(0.01)
    fs._substep(0.01)
    assert np.array_equal(fs.cellType, o.cellType)
    nP = o.nP
    assert np.array_equal(fs.download("pflag"), o.arr("pflag")[:nP])
    W = o.nx * o.dx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(fs.download(k).astype(np.float64) - o.arr(k)[:nP])) <= 1e-5 * W, k
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-5, k
    for k in ("u", "v", "w"):
        assert rel_err(fs.download(k), o.arr(k)) <= 1e-5, k
    compare_balls(o, fs, 1e-6, 1e-4)


def test_balls_ten_substeps():
    o, fs = with_balls()
    for _ in range(10):
        o.substep(0.01)
        fs._substep(0.01)
    compare_balls(o, fs, 1e-4, 1e-2)
    assert np.count_nonzero(fs.cellType != o.cellType) <= 16


def test_balls_float_and_sink():
    o, fs = with_balls()
    c = o.nx * o.dx / 2
    r0 = np.linalg.norm(fs.balls[:, :3] - c, axis=1)
    for _ in range(80):
        fs._substep(0.01)
    b = fs.balls
    r1 = np.linalg.norm(b[:, :3] - c, axis=1)
    assert 0.02 < b[0, 8] < 0.98                          # light ball floats part-submerged
    assert r1[1] < r0[1] - 0.05                           # heavy ball sinks toward the floor
    assert np.all(np.isfinite(b))


def test_ball_api():
    o = planet("planet32", **PLAIN32)
    fs = to_device(o)
    assert fs.balls.shape == (0, 9)
    rows = np.array([[16, 28, 16, 0.1, 0, 0, 1.0, 600, 0.0], [10, 16, 16, 0, 0, 0, 0.8, 1200, 0.0]])
    fs.set_balls(rows)
    assert np.array_equal(fs.balls, rows)
    with pytest.raises(WsError):
        fs.add_ball(16, 16, 16, -1.0, 500)
    fs.set_balls(np.zeros((0, 9)))
    for i in range(64):
        fs.add_ball(16 + 0.01 * i, 28, 16, 0.5, 500)
    with pytest.raises(WsError):
        fs.add_ball(16, 28, 16, 0.5, 500)
    fs.resetWater(o.scalars.oceanR - o.scalars.coreR)     # resetWater drops the balls
    assert fs.balls.shape == (0, 9)
    fs._substep(0.01)                                     # the solid-velocity field is cleared once
    fs._substep(0.01)


def test_snapshot_carries_balls():
    o, a = with_balls()
    a._substep(0.01)
    blob = a.snapshot()
    s = o.scalars
    from fluid_solver import FluidSolver
    b = FluidSolver(nx=o.nx, ny=o.ny, nz=o.nz, dx=o.dx, coreR=s.coreR, terrainSeed=s.terrainSeed,
                    bumpiness=s.bumpiness, targetParticles=s.targetParticles, capacity=s.nP + 8192)
    b.restore(blob)
    assert np.array_equal(a.balls, b.balls)
    assert np.array_equal(b.snapshot(), blob)
    a._substep(0.01)
    b._substep(0.01)
    assert np.array_equal(a.cellType, b.cellType)
    assert np.max(np.abs(a.balls - b.balls)) <= 1e-6 * max(1.0, np.abs(a.balls).max())

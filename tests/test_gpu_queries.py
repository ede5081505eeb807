"""The FluidSolver helpers on the device against the oracle: waveImpulse,
dryLandFraction, sampleVel, terrainRadiusAt, oceanPoint (js/solver.js
:3866-3892, :3593-3623, :811-854, :512-535, :591-608), through the C ABI.

waveImpulse and oceanPoint draw from the seeded stir stream on both sides
(the reference's Math.random() is unseeded), so the stream state must come
out equal. Bars: velocities after waveImpulse within 1e-7 relative (the
direction's sin/cos/acos are host libm on both sides; the per-particle
arithmetic is FP64 with one float store); sampled velocities and radii
within 1e-12 relative (FP64 sums of float data in the same order);
oceanPoint within 1e-12; dryLandFraction within one of its 1200 rays (the
ray directions use the device's cos/sin, which may differ from the host's in
the last bit and move a ray across a voxel boundary)."""
import numpy as np
import pytest

from helpers import planet, to_device, rel_err, DEVICE_ORDER

pytestmark = pytest.mark.gpu

THERMAL64 = dict(pic=0.05, omega=1.7, maxSpeed=3.2, sorTol=1e-5, sorCheckEvery=10, sorMaxIters=3000)


def _state():
    o = planet("planet64", **THERMAL64)
    o.set_scalars(gRamp=1.5)
    o.stir_gaussian(4.0, 2.0)
    o.substep(0.01)
    o.substep(0.01)
    return o


def test_wave_impulse_parity():
    o = _state()
    fs = to_device(o, with_grid=True)
    nP = o.nP
    before = o.arr("pvx")[:nP].copy()
    o.wave_impulse(0.8)
    fs.waveImpulse(0.8)
    assert fs.scalars.stirS == o.scalars.stirS
    assert np.count_nonzero(o.arr("pvx")[:nP] != before) > nP // 4
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-7, k


def test_dry_land_fraction_parity():
    o = _state()
    fs = to_device(o, with_grid=True)
    g, c = fs.dryLandFraction(), o.dry_land_fraction()
    assert 0.05 < c < 0.6
    assert abs(g - c) <= 1.0 / 1200 + 1e-15


def test_sample_vel_and_terrain_radius_parity():
    o = _state()
    fs = to_device(o, with_grid=True)
    rng = np.random.default_rng(4)
    pts = rng.uniform(0.5, o.nx * o.dx - 0.5, (5000, 3))
    uvw = fs.sample_vel(pts)
    ref = np.array([o.sample_vel(*p) for p in pts])
    assert np.abs(ref).max() > 1e-3
    assert rel_err(uvw, ref) <= 1e-12
    R = fs.terrain_radius_at(pts)
    refR = np.array([o.terrain_radius_at(*p) for p in pts])
    assert rel_err(R, refR) <= 1e-12
    x, y, z = pts[7]
    assert fs.sampleVel(x, y, z) == tuple(uvw[7])


@pytest.mark.parametrize("min_depth", [0.0, 2.0, 50.0])
def test_ocean_point_parity(min_depth):
    o = _state()
    fs = to_device(o, with_grid=True)
    for _ in range(3):                  # consecutive calls walk the stream alike
        pg, po = fs.oceanPoint(min_depth), o.ocean_point(min_depth)
        assert np.max(np.abs(np.array(pg) - np.array(po))) <= 1e-12 * o.nx
        assert fs.scalars.stirS == o.scalars.stirS
    c = o.nx * o.dx / 2
    r = np.linalg.norm(np.array(pg) - c)
    assert r <= o.scalars.oceanR + 1e-9

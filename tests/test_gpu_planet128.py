"""Parity at the headline size: one substep of the 128^3 planet (sea-level
radius 52, ocean 8 deep, 1,856,640 particles) on the device against the
oracle in the reference's arithmetic (double arithmetic over float storage,
the device order of the three order-dependent passes), from the same state.

The state is made on the oracle: a seeded Gaussian stir kick (sigma 4 cells,
2 m/s peak) and two substeps of dt = 0.01 with SOR to a 1e-5 relative
residual (checked every 10 iterations), so velocities and the warm-start q
are far from zero. Both sides then take one more substep.

Bars: cell types, particle phases, pcool, per-phase counts, the fluid cell
count and the SOR iteration count bit-exact; q, u/v/w and particle
velocities within 1e-5 relative (L-infinity); positions within 1e-5 of the
box width. The oracle's substep at this size takes about half a second on
one core; the fill about ten.
"""
import numpy as np
import pytest

from helpers import planet, to_device, rel_err

pytestmark = pytest.mark.gpu

BENCH128 = dict(pic=0.05, omega=1.7, maxSpeed=3.2, cfl=3.0, viscosity=5e-4, thermalOn=0,
                sorTol=1e-5, sorCheckEvery=10, sorMaxIters=5000, pressureIters=40)
TOL = 1e-5


def test_substep_parity_planet128():
    o = planet("planet128", **BENCH128)
    o.set_scalars(gRamp=1.5)
    o.stir_gaussian(4.0, 2.0)
    o.substep(0.01)
    o.substep(0.01)
    fs = to_device(o)
    nP = o.nP
    assert nP > 1800000
    o.substep(0.01)
    fs._substep(0.01)
    so, sg = o.scalars, fs.scalars
    assert np.array_equal(fs.cellType, o.cellType)
    assert sg.nFluid == so.nFluid
    assert sg.sorIters == so.sorIters and so.sorIters >= 10
    assert sg.sorRelRes <= 1e-5
    fl = fs.download("pflag")
    assert np.array_equal(fl, o.arr("pflag")[:nP])
    assert np.array_equal(np.bincount(fl, minlength=6), np.bincount(o.arr("pflag")[:nP], minlength=6))
    assert np.array_equal(fs.download("pcool"), o.arr("pcool")[:nP])
    assert rel_err(fs.q, o.q) <= TOL
    for k in ("u", "v", "w"):
        e = rel_err(fs.download(k), o.arr(k))
        assert e <= TOL, "%s rel err %.3g" % (k, e)
    for k in ("pvx", "pvy", "pvz"):
        e = rel_err(fs.download(k), o.arr(k)[:nP])
        assert e <= TOL, "%s rel err %.3g" % (k, e)
    W = o.nx * o.dx
    for k in ("px", "py", "pz"):
        err = np.max(np.abs(fs.download(k).astype(np.float64) - o.arr(k)[:nP]))
        assert err <= TOL * W, "%s max abs err %.3g" % (k, err)
    fs.close()

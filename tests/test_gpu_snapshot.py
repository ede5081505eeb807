"""ws_snapshot / ws_restore and ws_unet_save / ws_unet_load: a restored handle
holds exactly the saved state (it snapshots back to the same bytes) and steps
like the original; malformed or mismatched blobs are refused."""
import numpy as np
import pytest

from helpers import planet, to_device, PLAIN32, PFIELDS
from fluid_solver import FluidSolver, WsError

pytestmark = pytest.mark.gpu


def _fresh(o):
    s = o.scalars
    return FluidSolver(nx=o.nx, ny=o.ny, nz=o.nz, dx=o.dx, coreR=s.coreR, terrainSeed=s.terrainSeed,
                       bumpiness=s.bumpiness, targetParticles=s.targetParticles, capacity=s.nP + 8192)


def test_snapshot_round_trip_planet32():
    o = planet("planet32", **PLAIN32)
    a = to_device(o)
    for _ in range(3):
        a._substep(0.01)
    blob = a.snapshot()
    b = _fresh(o)
    b.restore(blob)
    assert np.array_equal(b.snapshot(), blob)          # every stored byte came back
    nP = a.scalars.nP
    for k in PFIELDS:
        assert np.array_equal(a.download(k, nP), b.download(k, nP)), k
    assert np.array_equal(a.download("q"), b.download("q"))
    for k in ("evS", "cfS", "bfS", "stirS", "nP", "gRamp", "dtLast", "oceanR"):
        assert getattr(a.scalars, k) == getattr(b.scalars, k), k
    a._substep(0.01)
    b._substep(0.01)
    assert np.array_equal(a.download("pflag", nP), b.download("pflag", nP))
    assert np.array_equal(a.download("cellType"), b.download("cellType"))
    W = o.nx * o.dx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(a.download(k, nP).astype(np.float64) - b.download(k, nP))) <= 1e-5 * W, k


def test_snapshot_rejects_bad_blobs():
    o = planet("planet32", **PLAIN32)
    a = to_device(o)
    blob = a.snapshot()
    b = _fresh(o)
    with pytest.raises(WsError):
        b.restore(blob[:-1])                           # truncated
    # cut inside the knobs and scalars that follow the header: refused before
    # they are read (the header alone is valid)
    for cut in (100, 200, 400):
        with pytest.raises(WsError):
            b.restore(blob[:cut].copy())
    bad = blob.copy()
    bad[0] ^= 0xFF
    with pytest.raises(WsError):
        b.restore(bad)                                 # not a snapshot
    other = FluidSolver(nx=24, ny=24, nz=24, dx=1.0, coreR=8.0, targetParticles=1000, capacity=4096)
    with pytest.raises(WsError):
        other.restore(blob)                            # another grid


def test_unet_save_load():
    o = planet("planet32", **PLAIN32)
    a = to_device(o)
    a.set_params(sorTol=1e-5, sorCheckEvery=10, sorMaxIters=4000)
    a.unet_init(1)
    a.unet_collect(2)
    a._substep(0.01)
    a._substep(0.01)
    a.unet_collect(0)
    a.unet_train(3, 1, 1e-3, 5)
    blob = a.unet_save()
    b = to_device(o)
    b.unet_init(2)
    assert not np.array_equal(a.unet_weights(), b.unet_weights())
    b.unet_load(blob)
    assert np.array_equal(a.unet_weights(), b.unet_weights())
    assert a.unet_info()["gain"] == b.unet_info()["gain"]
    r0n, types, target = a.unet_pair(1)
    b.unet_put_pair(r0n, types, target)
    np.testing.assert_array_equal(a.unet_forward_pair(1), b.unet_forward_pair(0))
    with pytest.raises(WsError):
        b.unet_load(blob[:-4])

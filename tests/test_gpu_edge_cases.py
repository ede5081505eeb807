"""Edge cases of the substep against the oracle, through the C ABI.

Ragged grid: a 35^3 planet (sea level 15.5, ocean 4 deep), so the last 4^3
brick along every axis holds three cells and the warm-start network's last
8 x 16 x 8 tile along every axis is partial (levels of 35, 18, 9 and 5
voxels). Fluid reaches those partial bricks. The substep checks are those of
the 32^3 planet (cell types and flags bit-exact, fields within 1e-5).

Empty ocean: a planet with no particle. The reference's solve then returns
before its first sweep (js/solver.js:1330): no fluid cell, q zero, no
iteration."""
import numpy as np
import pytest

from helpers import snapshot, restore, to_device, rel_err, DEVICE_ORDER, PLAIN32, planet
from oracle import unet_oracle as U

pytestmark = pytest.mark.gpu

TOL = 1e-5
RAGGED = dict(n=35, R=15.5, depth=4.0)
_SNAP = {}


def ragged(**params):
    """A fresh oracle copy of the 35^3 planet in device order."""
    if "r35" not in _SNAP:
        from oracle.oracle import make_planet
        _SNAP["r35"] = snapshot(make_planet(RAGGED["n"], R=RAGGED["R"], depth=RAGGED["depth"]))
    o = restore(_SNAP["r35"])
    o.set(**DEVICE_ORDER)
    o.set(**params)
    return o


def _partial_bricks_hold_fluid(o):
    n = o.nx
    ct = o.cellType.reshape(n, n, n)                 # (z, y, x)
    lo = (n // 4) * 4
    return (ct[:, :, lo:] == 1).any() and (ct[:, lo:, :] == 1).any() and (ct[lo:] == 1).any()


def _compare_particles(o, fs, label):
    nP = o.nP
    assert fs.scalars.nP == nP
    W = o.nx * o.dx
    for k in ("pflag", "pcool"):
        bad = np.nonzero(fs.download(k) != o.arr(k)[:nP])[0]
        assert bad.size == 0, "%s %s differs at %d particles" % (label, k, bad.size)
    for k in ("px", "py", "pz"):
        err = np.max(np.abs(fs.download(k).astype(np.float64) - o.arr(k)[:nP]))
        assert err <= TOL * W, "%s %s max abs err %.3g" % (label, k, err)
    for k in ("pvx", "pvy", "pvz"):
        e = rel_err(fs.download(k), o.arr(k)[:nP])
        assert e <= TOL, "%s %s rel err %.3g" % (label, k, e)


@pytest.mark.parametrize("cell_order", [0, 1])
def test_ragged_substep_parity(cell_order):
    o = ragged(**PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    fs.set_params(p2gCellOrder=cell_order)
    o.substep(0.01)
    fs._substep(0.01)
    assert _partial_bricks_hold_fluid(o)
    assert np.array_equal(fs.cellType, o.cellType)
    assert fs.scalars.nFluid == o.scalars.nFluid
    assert rel_err(fs.q, o.q) <= TOL
    for k in ("u", "v", "w"):
        e = rel_err(fs.download(k), o.arr(k))
        assert e <= TOL, "%s rel err %.3g" % (k, e)
    _compare_particles(o, fs, "ragged")
    assert abs(fs.scalars.umax - o.scalars.umax) <= TOL * o.scalars.umax
    assert fs.scalars.airborneCount == o.scalars.airborneCount
    fs.close()


def test_ragged_tolerance_mode_and_ten_substeps():
    """SOR to 1e-5 (check every 5): the same iteration count each substep;
    after ten substeps the cell types still agree and the velocities stay
    at the FP32 rounding level."""
    o = ragged(**PLAIN32, sorTol=1e-5, sorCheckEvery=5, sorMaxIters=2000)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    for _ in range(10):
        o.substep(0.01)
        fs._substep(0.01)
        assert fs.scalars.sorIters == o.scalars.sorIters
        assert fs.scalars.sorRelRes <= 1e-5
    assert np.array_equal(fs.cellType, o.cellType)
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:o.nP]) <= 1e-4, k
    fs.close()


@pytest.mark.parametrize("levels", [3, 4])
def test_ragged_network_forward_and_gradients(levels):
    """The tensor-core convolutions, pooling and upsampling on levels whose
    sizes are neither multiples of the tile nor even; same tolerances as on
    the 32^3 planet (forward 3%, gradients 6% at 3 levels and 10% at 4)."""
    o = ragged(**PLAIN32, sorTol=1e-5, sorCheckEvery=10, sorMaxIters=4000)
    fs = to_device(o)
    fs.unet_init(7, levels)
    fs.unet_collect(2)
    for _ in range(2):
        fs._substep(0.01)
    fs.unet_collect(0)
    assert fs.unet_info()["pairs_stored"] == 2
    dims = (o.nx, o.ny, o.nz)
    w = fs.unet_weights()
    r0n, types, target = fs.unet_pair(1)
    fl = types == 1
    gpu = fs.unet_forward_pair(1)
    cpu = U.forward(dims, w, r0n, types, rounding=True, levels=levels)
    assert np.all(gpu[cpu == 0] == 0)
    assert np.linalg.norm(gpu[fl] - cpu[fl]) < 3e-2 * np.linalg.norm(cpu[fl])
    gain = float(np.sqrt(np.mean(target[fl].astype(np.float64) ** 2)))
    fs.unet_set_gain(gain)
    g_gpu, loss_gpu = fs.unet_grad_pair(1)
    loss_cpu, g_cpu = U.loss_grad(dims, w, r0n, types, target / np.float32(gain), rounding=True, levels=levels)
    assert abs(loss_gpu - loss_cpu) <= 2e-2 * loss_cpu
    tol = {3: 6e-2, 4: 1e-1}[levels]
    for name, (ws, bs) in U.slices(levels).items():
        for sl in (ws, bs):
            err = np.linalg.norm(np.asarray(g_gpu[sl], np.float64) - g_cpu[sl]) / max(np.linalg.norm(g_cpu[sl]), 1e-30)
            assert err < tol, (name, err)
    fs.close()


@pytest.mark.parametrize("tol_mode", [False, True])
def test_empty_ocean(tol_mode):
    """No particle: every cell is air or solid, the solve runs no sweep and
    q stays zero; the face velocities (gravity on the empty faces, boundary
    conditions, extrapolation) match the oracle's."""
    extra = dict(sorTol=1e-5, sorCheckEvery=5, sorMaxIters=2000) if tol_mode else {}
    o = planet("planet32", **PLAIN32, **extra)
    o.set_scalars(gRamp=1.5, nP=0)
    fs = to_device(o)
    for _ in range(2):
        o.substep(0.01)
        fs._substep(0.01)
        s = fs.scalars
        assert s.nP == 0 and s.nFluid == 0
        assert s.sorIters == o.scalars.sorIters == 0
        assert s.sorRelRes == 0.0
        assert s.airborneCount == 0
    assert np.array_equal(fs.cellType, o.cellType)
    assert not np.any(fs.cellType == 1)
    assert not np.any(fs.q)
    for k in ("u", "v", "w"):
        e = rel_err(fs.download(k), o.arr(k))
        assert e <= TOL, "%s rel err %.3g" % (k, e)
    fs.close()

"""ws_metaball_mesh against the metaball oracle (Metaballs.build,
js/surface.js:203-284). The corner field is compared with the oracle's
Float32 particle-order sum within that sum's own rounding bound (the device
accumulates in FP64 and rounds once): |gpu - oracle| <= 3e-5 x oracle +
1e-7. The mesh of the device's field is compared with the oracle mesher on
the same field: same vertex count, bit-identical float positions and normals
in emission order, the same FP64 volume (1e-12). Cases: the reference's own
7^3 and 11^3 particle blocks on the 16^3 stub (spacing dx/4) over tension and
the detail factor, mixed flags and strays, the 32^3 planet after a substep,
and 2M seeded particles on a 128^3 box."""
import math

import numpy as np
import pytest

from fluid_solver import FluidSolver
from helpers import planet, to_device, PLAIN32
from oracle.oracle import metaball_field, mt_mesh_field

pytestmark = pytest.mark.gpu

FIELD_REL, FIELD_ABS = 3e-5, 1e-7


def check(fs, f, nx, dx, spacing, tension, detail):
    vol, pos, nrm, field, m = fs.metaballs(tension, detail, field=True)
    ref, rm, mdx, iso, _ = metaball_field(f["px"], f["py"], f["pz"], f["pflag"], nx, dx, spacing, tension, detail)
    assert m == rm
    assert np.all(np.abs(field.astype(np.float64) - ref) <= FIELD_REL * np.abs(ref) + FIELD_ABS)
    v2, p2, n2 = mt_mesh_field(field, m, m, m, mdx, iso)
    assert len(pos) == len(p2)
    assert np.array_equal(pos, p2) and np.array_equal(nrm, n2)
    assert abs(vol - abs(v2)) <= 1e-12 * max(vol, 1e-30)
    return vol, len(pos)


def stub(px, py, pz, fl=None, n=16):
    dx = 1.0 / n
    fs = FluidSolver(nx=n, ny=n, nz=n, dx=dx, coreR=n * dx * 0.3, targetParticles=1000, capacity=len(px) + 64)
    fs.set_scalars(spacing=dx * 0.25, nP=len(px))
    f = {"px": np.asarray(px, np.float32), "py": np.asarray(py, np.float32), "pz": np.asarray(pz, np.float32),
         "pflag": np.zeros(len(px), np.uint8) if fl is None else np.asarray(fl, np.uint8)}
    if len(px):
        fs.upload_state(f, count=len(px))
    return fs, f


def block(side, n=16):
    sp = 0.25 / n
    g = np.arange(side) * sp + 0.5 - (side // 2) * sp
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    return x.ravel(), y.ravel(), z.ravel()


@pytest.mark.parametrize("side", [7, 11])
def test_reference_blocks(side):
    fs, f = stub(*block(side))
    for t in (0, 0.25, 0.5, 0.75, 1):
        for detail in (None, 0.6, 1.4, 999):
            vol, nv = check(fs, f, 16, 1.0 / 16, 0.25 / 16, t, detail)
            assert vol > 0 and nv % 3 == 0


def test_flags_empty_and_strays():
    x, y, z = block(7)
    fl = np.where(np.arange(len(x)) % 2 == 1, 2, 0)
    fs, f = stub(x, y, z, fl)
    check(fs, f, 16, 1.0 / 16, 0.25 / 16, 0.0, None)
    fs, f = stub(x, y, z, np.full(len(x), 2))
    assert check(fs, f, 16, 1.0 / 16, 0.25 / 16, 0.5, None)[1] == 0
    fs, f = stub([], [], [])
    assert check(fs, f, 16, 1.0 / 16, 0.25 / 16, 0.5, None)[1] == 0
    d = 1.0 / 16
    fs, f = stub([5 * d, -3 * d, 2.0, math.nan, 1e30], [5 * d] * 5, [5 * d] * 5)
    check(fs, f, 16, d, 0.25 * d, 0.5, None)


def test_planet32_after_substep():
    o = planet("planet32", **PLAIN32)
    fs = to_device(o)
    fs._substep(0.01)
    nP = fs.scalars.nP
    f = {k: fs.download(k, nP) for k in ("px", "py", "pz", "pflag")}
    for t, detail in ((0.5, None), (0.0, 1.6), (1.0, 0.5)):
        vol, nv = check(fs, f, fs.nx, fs.dx, fs.scalars.spacing, t, detail)
        assert nv > 1000


def test_two_million_particles_128():
    n, N = 2_000_000, 128
    r = np.random.default_rng(5)
    fs = FluidSolver(nx=N, ny=N, nz=N, dx=1.0, coreR=40, targetParticles=1000, capacity=n + 64)
    c = np.array([64.0, 64.0, 64.0])
    # a shell of fluid between radius 30 and 50, sorted by cell like the solver's particles
    u = r.normal(size=(n, 3)); u /= np.linalg.norm(u, axis=1)[:, None]
    p = (c + u * r.uniform(30, 50, n)[:, None]).astype(np.float32)
    p = p[np.lexsort((p[:, 0], p[:, 1], p[:, 2]))]
    f = {"px": p[:, 0].copy(), "py": p[:, 1].copy(), "pz": p[:, 2].copy(),
         "pflag": (r.uniform(size=n) > 0.97).astype(np.uint8)}          # 3% spray, the rest liquid
    fs.set_scalars(nP=n)
    fs.upload_state(f, count=n)
    vol, nv = check(fs, f, N, 1.0, fs.scalars.spacing, 0.5, None)
    assert nv > 100000

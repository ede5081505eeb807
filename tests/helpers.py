"""Test helpers: oracle fixtures and their transfer onto the device.

The oracle (oracle/oracle.py) is the checker; these helpers only move its
inputs to the library under test so both start from identical state.
"""
import numpy as np

from oracle.oracle import make_planet, PLANETS

DEVICE_ORDER = dict(sorRedBlack=1, viscJacobi=1, extrapJacobi=1)
# the 32^3 workload: pic 0.05, omega 1.7, 40 iterations, thermal off
PLAIN32 = dict(pic=0.05, omega=1.7, pressureIters=40, maxSpeed=3.2, cfl=3.0, thermalOn=0)

_CACHE = {}


def planet(name, device_order=True, **params):
    """A fresh oracle planet; the expensive terrain+fill is cached as arrays."""
    key = name
    if key not in _CACHE:
        o = make_planet(name)
        _CACHE[key] = snapshot(o)
    o = restore(_CACHE[key])
    if device_order:
        o.set(**DEVICE_ORDER)
    if params:
        o.set(**params)
    return o


PFIELDS = ("px", "py", "pz", "pvx", "pvy", "pvz", "pT", "pAir", "pLight", "pWx", "pWy", "pWz", "pPh",
           "pflag", "pcool", "pDepth")
SCALARS = ("coreR", "oceanR", "spacing", "particleVolume", "iso", "waterTopY", "umax", "dtLast",
           "simTime", "gRamp", "heatAcc", "targetParticles", "landFrac", "bumpiness",
           "evS", "cfS", "bfS", "stirS", "terrainSeed", "nP")


def snapshot(o):
    s = o.scalars
    nP = s.nP
    snap = {"dims": (o.nx, o.ny, o.nz, o.dx), "terrain": o.terrain(),
            "scalars": {k: getattr(s, k) for k in SCALARS},
            "fields": {k: o.arr(k)[:nP].copy() for k in PFIELDS},
            "q": o.arr("q").copy(), "dens": o.arr("dens").copy()}
    return snap


def restore(snap, fp64=False):
    from oracle.oracle import Oracle
    nx, ny, nz, dx = snap["dims"]
    sc = snap["scalars"]
    o = Oracle(nx, ny, nz, dx, coreR=sc["coreR"], terrainSeed=sc["terrainSeed"],
               bumpiness=sc["bumpiness"], targetParticles=sc["targetParticles"], fp64=fp64)
    o.load_terrain(snap["terrain"])
    nP = sc["nP"]
    o.alloc_particles(nP + 8192)
    for k, v in snap["fields"].items():
        o.arr(k)[:nP] = v
    o.arr("q")[:] = snap["q"]
    o.arr("dens")[:] = snap["dens"]
    o.set_scalars(**sc)
    o.L.or_build_planet_gravity(o.h)
    return o


def to_device(o, capacity=None, with_grid=False):
    """A FluidSolver on cuda:0 holding exactly the oracle's state and knobs
    (with_grid: also the cell types and face velocities of the last substep)."""
    from fluid_solver import FluidSolver
    s = o.scalars
    nP = s.nP
    fs = FluidSolver(nx=o.nx, ny=o.ny, nz=o.nz, dx=o.dx, coreR=s.coreR, terrainSeed=s.terrainSeed,
                     bumpiness=s.bumpiness, targetParticles=s.targetParticles,
                     capacity=capacity or (nP + 8192))
    fs.upload_terrain(o.terrain())
    p = o.params
    kw = {f[0]: getattr(p, f[0]) for f in p._fields_ if f[0] not in ("sunPos",)}
    kw["sunPos"] = list(p.sunPos) if p.hasSun else None
    kw.pop("hasSun")
    fs.set_params(**kw)
    for k in PFIELDS:
        fs.upload(k, o.arr(k)[:nP])
    fs.upload("q", o.arr("q"))
    fs.upload("dens", o.arr("dens"))
    fs.set_scalars(**{k: getattr(s, k) for k in SCALARS}, nFluid=s.nFluid)
    if with_grid:
        for k in ("cellType", "u", "v", "w", "uO", "vO", "wO"):
            fs.upload(k, o.arr(k))
    return fs


def rel_err(a, b):
    """max |a - b| / max |b| (L-infinity relative error), 0 for an all-zero b."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if b.size else 0.0
    return num / den if den > 0 else num

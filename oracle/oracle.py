"""ctypes wrapper of the CPU oracle — TEST INFRASTRUCTURE ONLY.

The oracle restates WaterSim's FluidSolver (js/solver.js) in C (ws_oracle.c)
and is the parity checker for the CUDA library. Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg use this module; the
product path never imports it.

Two flavours: ``Oracle(..., fp64=False)`` stores float32 and computes in
double (the JavaScript semantics: Float32Array storage, double arithmetic);
``fp64=True`` stores double everywhere (the FP64 oracle).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


class OrParams(C.Structure):
    """Mirror of or_params (ws_oracle.h); same field order as ws_params."""
    _fields_ = [
        ("substeps", C.c_int32), ("pressureIters", C.c_int32),
        ("cfl", C.c_double), ("pic", C.c_double), ("gravity", C.c_double),
        ("viscosity", C.c_double), ("omega", C.c_double), ("maxSpeed", C.c_double),
        ("vorticity", C.c_double), ("currents", C.c_double), ("shadeCool", C.c_double),
        ("sunActivity", C.c_double), ("evapIntensity", C.c_double), ("atmosphereH", C.c_double),
        ("ceilReflect", C.c_int32), ("hasSun", C.c_int32), ("sunPos", C.c_double * 3),
        ("heatK", C.c_double), ("Tamb", C.c_double), ("cloudT", C.c_double),
        ("cloudP", C.c_double), ("rainT", C.c_double), ("rainLiftAge", C.c_double),
        ("snowT", C.c_double), ("meltT", C.c_double),
        ("spinOn", C.c_int32), ("thermalOn", C.c_int32),
        ("sorRedBlack", C.c_int32), ("sorCheckEvery", C.c_int32),
        ("sorTol", C.c_double), ("sorMaxIters", C.c_int32),
        ("viscJacobi", C.c_int32), ("extrapJacobi", C.c_int32),
        ("p2gCellOrder", C.c_int32),
    ]


class OrScalars(C.Structure):
    """Mirror of or_scalars (ws_oracle.h)."""
    _fields_ = [
        ("coreR", C.c_double), ("oceanR", C.c_double), ("spacing", C.c_double),
        ("particleVolume", C.c_double), ("iso", C.c_double), ("waterTopY", C.c_double),
        ("umax", C.c_double), ("dtLast", C.c_double), ("simTime", C.c_double),
        ("gRamp", C.c_double), ("heatAcc", C.c_double),
        ("targetParticles", C.c_double), ("landFrac", C.c_double), ("bumpiness", C.c_double),
        ("sorRelRes", C.c_double),
        ("evS", C.c_uint32), ("cfS", C.c_uint32), ("bfS", C.c_uint32), ("stirS", C.c_uint32),
        ("terrainSeed", C.c_uint32),
        ("nP", C.c_int32), ("capacity", C.c_int32),
        ("airborneCount", C.c_int32), ("vaporCount", C.c_int32), ("nightVaporCount", C.c_int32),
        ("evapCount", C.c_int32), ("substepsLast", C.c_int32), ("nFluid", C.c_int32),
        ("sorIters", C.c_int32), ("sorPath", C.c_int32),
    ]


def build():
    """Compile both oracle flavours with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(fp64):
    key = "f64" if fp64 else "js"
    if key in _LIBS:
        return _LIBS[key]
    path = os.path.join(_HERE, "liboracle_%s.so" % key)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, d, i32, u32, i64p = C.c_void_p, C.c_double, C.c_int, C.c_uint32, C.POINTER(C.c_int64)
    sigs = {
        "or_create": (vp, [i32, i32, i32, d, d, u32, d, d]),
        "or_destroy": (None, [vp]),
        "or_storage_bytes": (i32, []),
        "or_get_params": (None, [vp, C.POINTER(OrParams)]),
        "or_set_params": (None, [vp, C.POINTER(OrParams)]),
        "or_get_scalars": (None, [vp, C.POINTER(OrScalars)]),
        "or_set_scalars": (None, [vp, C.POINTER(OrScalars)]),
        "or_array": (vp, [vp, C.c_char_p, i64p, C.POINTER(C.c_int)]),
        "or_alloc_particles": (i32, [vp, i32]),
        "or_generate_terrain": (None, [vp, u32, d]),
        "or_load_terrain": (i32, [vp, i32, d, vp, vp, d, d, d, d]),
        "or_water_volume_mc": (d, [vp, d]),
        "or_reset_water": (None, [vp, d]),
        "or_build_planet_gravity": (None, [vp]),
        "or_step": (None, [vp, d]),
        "or_substep": (None, [vp, d]),
        "or_residual": (d, [vp]),
        "or_clamp_um": (d, [vp]),
        "or_mt_volume": (d, [vp, d, i64p]),
        "or_autotune_iso": (d, [vp]),
        "or_census": (None, [vp, C.POINTER(C.c_double)]),
        "or_kinetic_energy": (d, [vp]),
        "or_dry_land_fraction": (d, [vp]),
        "or_sample_vel": (None, [vp, d, d, d, C.POINTER(C.c_double)]),
        "or_sample_face": (d, [vp, i32, d, d, d]),
        "or_terrain_radius_at": (d, [vp, d, d, d]),
        "or_rock_cell_at": (i32, [vp, d, d, d]),
        "or_apply_impulse_sphere": (None, [vp, d, d, d, d, d, d, d]),
        "or_stir_at": (None, [vp, d, d, d, d, d, d, d, d]),
        "or_add_ball": (i32, [vp, d, d, d, d, d]),
        "or_get_balls": (i32, [vp, vp, i32]),
        "or_set_balls": (i32, [vp, vp, i32]),
        "or_push_balls": (None, [vp]),
        "or_update_balls": (None, [vp, d]),
        "or_stir_gaussian": (None, [vp, d, d]),
        "or_wave_impulse": (None, [vp, d]),
        "or_ocean_point": (None, [vp, d, C.POINTER(C.c_double)]),
        "or_mt_volume_field": (d, [vp, i32, i32, i32, d, d, i64p]),
        "or_mt_mesh_field": (d, [vp, i32, i32, i32, d, d, vp, vp, C.c_int64, i64p]),
        "or_metaball_field": (i32, [i32, vp, vp, vp, vp, i32, d, d, d, d, vp,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    }
    for stage in ("clear_faces", "rasterize_static", "mark_fluid", "p2g", "apply_bc",
                  "snapshot_old", "pressure_solve", "project", "extrapolate",
                  "vapor_collisions", "ice_contacts", "push_surface", "splat_density"):
        sigs["or_" + stage] = (None, [vp])
    for stage in ("viscosity", "planet_gravity", "vorticity", "g2p", "advect", "update_heat",
                  "update_evaporation", "update_phase", "update_currents"):
        sigs["or_" + stage] = (None, [vp, d])
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIBS[key] = L
    return L


_KIND = {0: np.uint8, 1: np.int32, 3: np.float64}


class Oracle:
    """One FluidSolver instance restated on the CPU (sphere-planet mode)."""

    def __init__(self, nx, ny, nz, dx=1.0, coreR=0.0, terrainSeed=20260114, bumpiness=1.0,
                 targetParticles=110000, fp64=False):
        self.fp64 = fp64
        self.L = _lib(fp64)
        self.h = self.L.or_create(nx, ny, nz, dx, coreR, terrainSeed, bumpiness, targetParticles)
        self.nx, self.ny, self.nz, self.dx = nx, ny, nz, dx
        self.real = np.float64 if fp64 else np.float32

    def __del__(self):
        try:
            if self.h:
                self.L.or_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # ---- knobs and scalars
    @property
    def params(self):
        p = OrParams()
        self.L.or_get_params(self.h, C.byref(p))
        return p

    def set(self, **kw):
        p = self.params
        for k, v in kw.items():
            if k == "sunPos":
                if v is None:
                    p.hasSun = 0
                else:
                    p.hasSun = 1
                    for i in range(3):
                        p.sunPos[i] = v[i]
            else:
                setattr(p, k, v)
        self.L.or_set_params(self.h, C.byref(p))

    @property
    def scalars(self):
        s = OrScalars()
        self.L.or_get_scalars(self.h, C.byref(s))
        return s

    def set_scalars(self, **kw):
        s = self.scalars
        for k, v in kw.items():
            setattr(s, k, v)
        self.L.or_set_scalars(self.h, C.byref(s))

    @property
    def nP(self):
        return self.scalars.nP

    # ---- arrays (numpy views into oracle memory)
    def arr(self, name):
        cnt, kind = C.c_int64(0), C.c_int(0)
        ptr = self.L.or_array(self.h, name.encode(), C.byref(cnt), C.byref(kind))
        if kind.value < 0:
            raise KeyError(name)
        dt = self.real if kind.value == 2 else _KIND[kind.value]
        if cnt.value == 0 or not ptr:
            return np.zeros(0, dt)
        buf = (C.c_char * (cnt.value * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt, count=cnt.value)

    def __getattr__(self, name):
        if name.startswith("_") or name in ("L", "h"):
            raise AttributeError(name)
        return self.arr(name)

    # ---- setup
    def generate_terrain(self, seed, seaLevel):
        self.L.or_generate_terrain(self.h, seed, seaLevel)

    def load_terrain(self, t):
        solid = np.ascontiguousarray(t["solid"], np.uint8)
        R = np.ascontiguousarray(t["R"], np.float32)
        self.L.or_load_terrain(self.h, int(t["n"]), float(t["dv"]), solid.ctypes.data,
                               R.ctypes.data, float(t["Rsl"]), float(t["Rlo"]),
                               float(t["Rhi"]), float(t["landFrac"]))

    def terrain(self):
        """The current terrain as plain arrays (float32 radius field)."""
        s = self.scalars
        n = round(len(self.arr("tsolid")) ** (1 / 3))
        return {"n": n, "dv": self.dx / 2, "solid": self.arr("tsolid").copy(),
                "R": self.arr("tR").astype(np.float32), "Rsl": self._terr_meta()[0],
                "Rlo": self._terr_meta()[1], "Rhi": self._terr_meta()[2],
                "landFrac": s.landFrac}

    def _terr_meta(self):
        # Rsl/Rlo/Rhi follow from coreR and the sea level (js/solver.js:280-282)
        s = self.scalars
        R1, Rsl = s.coreR, s.oceanR
        depthW = max(Rsl - R1, 1e-4)
        Rlo = max(R1 * 0.55, Rsl - 1.8889 * depthW)
        Rhi = Rsl + 0.7778 * depthW
        return Rsl, Rlo, Rhi

    def alloc_particles(self, cap):
        self.L.or_alloc_particles(self.h, cap)

    def water_volume_mc(self, depth):
        return self.L.or_water_volume_mc(self.h, depth)

    def reset_water(self, depth):
        self.L.or_reset_water(self.h, depth)

    # ---- drivers and stages
    def step(self, dtFrame):
        self.L.or_step(self.h, dtFrame)

    def substep(self, dt):
        self.L.or_substep(self.h, dt)

    def stage(self, name, *args):
        getattr(self.L, "or_" + name)(self.h, *args)

    def residual(self):
        return self.L.or_residual(self.h)

    def clamp_um(self):
        return self.L.or_clamp_um(self.h)

    def mt_volume(self, iso):
        cnt = C.c_int64(0)
        v = self.L.or_mt_volume(self.h, iso, C.byref(cnt))
        return v, cnt.value

    def autotune_iso(self):
        return self.L.or_autotune_iso(self.h)

    def census(self):
        out = (C.c_double * 3)()
        self.L.or_census(self.h, out)
        return tuple(out)

    def kinetic_energy(self):
        return self.L.or_kinetic_energy(self.h)

    def dry_land_fraction(self):
        return self.L.or_dry_land_fraction(self.h)

    def sample_vel(self, x, y, z):
        out = (C.c_double * 3)()
        self.L.or_sample_vel(self.h, x, y, z, out)
        return tuple(out)

    def sample_face(self, comp, x, y, z):
        return self.L.or_sample_face(self.h, comp, x, y, z)

    def terrain_radius_at(self, x, y, z):
        return self.L.or_terrain_radius_at(self.h, x, y, z)

    def rock_cell_at(self, x, y, z):
        return bool(self.L.or_rock_cell_at(self.h, x, y, z))

    def apply_impulse_sphere(self, *a):
        self.L.or_apply_impulse_sphere(self.h, *a)

    def stir_at(self, *a):
        self.L.or_stir_at(self.h, *a)

    def stir_gaussian(self, sigma, peak):
        self.L.or_stir_gaussian(self.h, sigma, peak)

    def wave_impulse(self, dvx):
        self.L.or_wave_impulse(self.h, dvx)

    def ocean_point(self, min_depth=0.0):
        out = (C.c_double * 3)()
        self.L.or_ocean_point(self.h, min_depth, out)
        return [out[0], out[1], out[2]]

    # balls: addBall (js/solver.js:3910); rows x y z vx vy vz r rho submerged
    def add_ball(self, x, y, z, r, rho):
        n = self.L.or_add_ball(self.h, x, y, z, r, rho)
        if n < 0:
            raise ValueError("too many balls")
        return n

    def balls(self):
        out = np.zeros((64, 9))
        n = self.L.or_get_balls(self.h, out.ctypes.data, 64)
        return out[:n].copy()

    def set_balls(self, rows):
        a = np.ascontiguousarray(rows, np.float64).reshape(-1, 9)
        if self.L.or_set_balls(self.h, a.ctypes.data, len(a)) < 0:
            raise ValueError("too many balls")


def mt_volume_field(dens, nx, ny, nz, dx, iso):
    """MarchingTetrahedra.build volume over an external float32 corner field."""
    L = _lib(False)
    d = np.ascontiguousarray(dens, np.float32)
    cnt = C.c_int64(0)
    v = L.or_mt_volume_field(d.ctypes.data, nx, ny, nz, dx, iso, C.byref(cnt))
    return v, cnt.value


def mt_mesh_field(dens, nx, ny, nz, dx, iso):
    """MarchingTetrahedra.build over an external float32 corner field: (volume,
    positions (V,3) float32, normals (V,3) float32), vertices in build order."""
    L = _lib(False)
    d = np.ascontiguousarray(dens, np.float32)
    cnt = C.c_int64(0)
    L.or_mt_mesh_field(d.ctypes.data, nx, ny, nz, dx, iso, None, None, 0, C.byref(cnt))
    n = cnt.value
    pos = np.zeros((max(n, 1), 3), np.float32)
    nrm = np.zeros((max(n, 1), 3), np.float32)
    v = L.or_mt_mesh_field(d.ctypes.data, nx, ny, nz, dx, iso, pos.ctypes.data, nrm.ctypes.data, n, C.byref(cnt))
    return v, pos[:n], nrm[:n]


def metaball_field(px, py, pz, pflag, nx, dx, spacing, tension, detail=None):
    """Metaballs.build's kernel field (js/surface.js:203-284) in the reference's
    Float32Array accumulation order: (field (m+1)^3 float32, m, mdx, iso, R)."""
    L = _lib(False)
    n = len(px)
    a = [np.ascontiguousarray(v, np.float32) for v in (px, py, pz)]
    f = np.ascontiguousarray(pflag, np.uint8)
    det = float("nan") if detail is None else float(detail)
    mdx, iso, R = C.c_double(), C.c_double(), C.c_double()
    m = L.or_metaball_field(n, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, f.ctypes.data, nx, dx, spacing,
                            tension, det, None, C.byref(mdx), C.byref(iso), C.byref(R))
    field = np.zeros((m + 1) ** 3, np.float32)
    L.or_metaball_field(n, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, f.ctypes.data, nx, dx, spacing,
                        tension, det, field.ctypes.data, C.byref(mdx), C.byref(iso), C.byref(R))
    return field, m, mdx.value, iso.value, R.value


# Planet workloads (grid n, sea-level radius R, ocean depth): coreR = R - depth,
# unit cells. "particles" is the reference's targetParticles knob; None fills
# at 8 particles per water cell (spacing dx/2).
PLANETS = {
    "planet32": dict(n=32, R=12.0, depth=3.0, particles=None),          # ~10k at 8 per cell
    "planet64": dict(n=64, R=26.0, depth=5.0, particles=220000),
    "planet128": dict(n=128, R=52.0, depth=8.0, particles=2000000),
    "planet256": dict(n=256, R=110.0, depth=12.0, particles=16000000),
}


def make_planet(name_or_n, R=None, depth=None, seed=20260114, fp64=False, per_cell=8.0, particles=None):
    """Build the seeded planet fixture: terrain, then the jittered lattice fill
    with targetParticles = particles (or 8 per water cell)."""
    if isinstance(name_or_n, str):
        cfg = PLANETS[name_or_n]
        n, R, depth, particles = cfg["n"], cfg["R"], cfg["depth"], cfg["particles"]
    else:
        n = name_or_n
    coreR = R - depth
    o = Oracle(n, n, n, 1.0, coreR=coreR, terrainSeed=seed, fp64=fp64)
    o.generate_terrain(seed, R)
    if particles is None:
        particles = float(round(o.water_volume_mc(depth) * per_cell))
    o.set_scalars(targetParticles=float(particles))
    o.reset_water(depth)
    return o

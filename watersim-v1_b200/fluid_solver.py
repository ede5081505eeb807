"""Host-side mirror of WaterSim's FluidSolver (js/solver.js) over libwatersim.

The reference's host code is JavaScript; this module stands in for it with
the same surface: constructor options, public knobs as attributes, the
typed-array fields, step(dtFrame) / _substep(dt), resetWater(depth),
generateTerrain(seed, seaLevel), splatDensity(), autotuneIso(), the
interaction helpers and kineticEnergy(). Everything computes on the GPU
through the C ABI of include/watersim.h; there is no CPU fallback — the
constructor raises if the CUDA library cannot be loaded or no device exists.

Differences from the reference object, all documented at the attribute:
  * typed-array fields are snapshots (numpy copies downloaded on access);
    assigning a numpy array to a field uploads it;
  * only the sphere-planet world is implemented (mode 'sphere');
  * pressure uses red-black SOR, viscosity and extrapolation Jacobi order.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libwatersim.so")
_lib = None


WS_BUSY = 1          # ws_step_async: previous frame still running, nothing started


class WsError(RuntimeError):
    """A ws_status < 0 from the library, with ws_last_error()'s message."""

    def __init__(self, code, msg):
        super().__init__("watersim error %d: %s" % (code, msg))
        self.code = code


class WsConfig(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("capacity", C.c_int32),
                ("dx", C.c_double), ("coreR", C.c_double), ("bumpiness", C.c_double),
                ("targetParticles", C.c_double), ("terrainSeed", C.c_uint32), ("device", C.c_int32)]


class WsParams(C.Structure):
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


class WsScalars(C.Structure):
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


class WsHostArrays(C.Structure):
    """ws_host_arrays: count plus one host pointer per particle field (NULL skips it)."""
    _fields_ = [("count", C.c_int64), ("field", C.c_void_p * 16)]


class WsUnetInfo(C.Structure):
    _fields_ = [("pairs_stored", C.c_int32), ("pairs_capacity", C.c_int32), ("train_steps", C.c_int64),
                ("num_weights", C.c_int64), ("gain", C.c_double), ("last_loss", C.c_double),
                ("enabled", C.c_int32), ("collecting", C.c_int32)]


class WsRenderOpts(C.Structure):
    """ws_render_opts: the scene state WaterScene.updateParticles reads
    (js/scene.js:1595-1922)."""
    _fields_ = [("show", C.c_int32), ("beadsMode", C.c_int32), ("metaballMode", C.c_int32),
                ("spinColor", C.c_int32), ("cloudSprite", C.c_int32), ("planetLit", C.c_int32),
                ("sortOn", C.c_int32), ("useLight", C.c_int32), ("useDepth", C.c_int32),
                ("useTemp", C.c_int32), ("waterOpa", C.c_double), ("pOpa", C.c_double),
                ("wScale", C.c_double), ("waterColor", C.c_double * 3), ("sunDir", C.c_double * 3),
                ("cam", C.c_double * 3)]


RENDER_CLASSES = ("beads", "spray", "vapor", "cloud", "snow")


def render_opts(**kw):
    """A WsRenderOpts with the scene's defaults (js/scene.js:780, 849, 895-896,
    981-983): liquid hidden (no beads mode), spray opacity 1, water opacity
    0.25, water hue #9fd4ee, solver mirrors present, sorted, lit."""
    o = WsRenderOpts()
    o.show, o.beadsMode, o.metaballMode, o.spinColor, o.cloudSprite = 1, 0, 0, 0, 0
    o.planetLit, o.sortOn, o.useLight, o.useDepth, o.useTemp = 1, 1, 1, 1, 1
    o.waterOpa, o.pOpa, o.wScale = 0.25, 1.0, 1.0
    o.waterColor[:] = (0x9f / 255, 0xd4 / 255, 0xee / 255)
    o.sunDir[:] = (1.0, 0.0, 0.0)
    o.cam[:] = (0.0, 0.0, 0.0)
    for k, v in kw.items():
        if k in ("waterColor", "sunDir", "cam"):
            getattr(o, k)[:] = tuple(float(x) for x in v)
        else:
            setattr(o, k, v)
    return o


class WsTerrain(C.Structure):
    _fields_ = [("n", C.c_int32), ("dv", C.c_double), ("Rsl", C.c_double), ("Rlo", C.c_double),
                ("Rhi", C.c_double), ("landFrac", C.c_double),
                ("solid", C.c_void_p), ("R", C.c_void_p)]


# field ids of include/watersim.h (ws_field), with element dtype
FIELDS = {
    "px": (0, np.float32), "py": (1, np.float32), "pz": (2, np.float32),
    "pvx": (3, np.float32), "pvy": (4, np.float32), "pvz": (5, np.float32),
    "pT": (6, np.float32), "pAir": (7, np.float32), "pLight": (8, np.float32),
    "pWx": (9, np.float32), "pWy": (10, np.float32), "pWz": (11, np.float32), "pPh": (12, np.float32),
    "pflag": (13, np.uint8), "pcool": (14, np.uint8), "pDepth": (15, np.uint8),
    "cellType": (16, np.uint8), "q": (17, np.float32), "rhs": (18, np.float32),
    "u": (19, np.float32), "v": (20, np.float32), "w": (21, np.float32),
    "uO": (22, np.float32), "vO": (23, np.float32), "wO": (24, np.float32),
    "uW": (25, np.float32), "vW": (26, np.float32), "wW": (27, np.float32),
    "validU": (28, np.uint8), "validV": (29, np.uint8), "validW": (30, np.uint8),
    "dens": (31, np.float32),
}
PARTICLE_FIELDS = ("px", "py", "pz", "pvx", "pvy", "pvz", "pT", "pAir", "pLight", "pWx", "pWy",
                   "pWz", "pPh", "pflag", "pcool", "pDepth")
STAGES = ["CLEAR_RASTER", "MARK_FLUID", "P2G", "FORCES", "PRESSURE", "PROJECT", "VORTICITY", "CLAMP",
          "EXTRAPOLATE", "G2P_ADVECT", "HEAT", "EVAPORATION", "PHASE", "PUSH_SURFACE", "SPLAT",
          "VAPOR_COLLISIONS", "ICE_CONTACTS", "CURRENTS"]
CEIL = {"linear": 0, "quadratic": 1, "exponential": 2}

# exported entry points of include/watersim.h
SYMBOLS = ["ws_create", "ws_destroy", "ws_last_error", "ws_version", "ws_set_params", "ws_get_params",
           "ws_default_params", "ws_set_scalars", "ws_get_scalars", "ws_generate_terrain",
           "ws_upload_terrain", "ws_download_terrain", "ws_water_volume", "ws_reset_water",
           "ws_upload_field", "ws_download_field", "ws_field_info", "ws_set_nparticles", "ws_step",
           "ws_substep", "ws_stage", "ws_residual", "ws_mt_volume", "ws_autotune_iso", "ws_census",
           "ws_kinetic_energy", "ws_apply_impulse_sphere", "ws_stir_at", "ws_stir_gaussian",
           "ws_wave_impulse", "ws_dry_land_fraction", "ws_sample_vel", "ws_terrain_radius_at", "ws_ocean_point",
           "ws_synchronize", "ws_get_stream", "ws_launch_count", "ws_time_kernel", "ws_probe_wait",
           "ws_residual_noalloc", "ws_upload_state", "ws_download_state",
           "ws_unet_init", "ws_unet_init_levels", "ws_unet_collect", "ws_unet_enable", "ws_unet_train", "ws_unet_get_info",
           "ws_unet_get_weights", "ws_unet_set_weights", "ws_unet_set_gain", "ws_unet_get_pair",
           "ws_unet_put_pair", "ws_unet_forward_pair", "ws_unet_grad_pair", "ws_unet_probe", "ws_unet_time",
           "ws_unet_accumulate", "ws_unet_grads", "ws_unet_apply", "ws_snapshot", "ws_restore",
           "ws_unet_save", "ws_unet_load", "ws_surface_mesh", "ws_surface_download", "ws_surface_device",
           "ws_render_particles", "ws_render_download", "ws_render_device",
           "ws_metaball_mesh", "ws_metaball_download", "ws_metaball_device", "ws_metaball_field",
           "ws_step_async", "ws_step_poll", "ws_step_wait", "ws_add_ball", "ws_get_balls", "ws_set_balls"]


def load_library(path=None):
    """Load libwatersim.so and declare its signatures (raises if missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or _LIB_PATH
    if not os.path.exists(p):
        raise OSError("libwatersim.so not built (%s); run watersim-v1_b200/build.py" % p)
    L = C.CDLL(p)
    h, vp, d, i32, u32, i64 = C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_uint32, C.c_int64
    sig = {
        "ws_create": [C.POINTER(WsConfig), C.POINTER(C.c_void_p)],
        "ws_destroy": [h], "ws_set_params": [h, C.POINTER(WsParams)],
        "ws_get_params": [h, C.POINTER(WsParams)], "ws_default_params": [C.POINTER(WsParams)],
        "ws_set_scalars": [h, C.POINTER(WsScalars)], "ws_get_scalars": [h, C.POINTER(WsScalars)],
        "ws_generate_terrain": [h, u32, d], "ws_upload_terrain": [h, C.POINTER(WsTerrain)],
        "ws_download_terrain": [h, vp, vp, C.POINTER(C.c_double)],
        "ws_water_volume": [h, d, C.POINTER(C.c_double)], "ws_reset_water": [h, d],
        "ws_upload_field": [h, i32, vp, i64], "ws_download_field": [h, i32, vp, i64],
        "ws_field_info": [h, i32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)],
        "ws_set_nparticles": [h, i32], "ws_step": [h, d], "ws_substep": [h, d],
        "ws_stage": [h, i32, d], "ws_residual": [h, C.POINTER(C.c_double)],
        "ws_mt_volume": [h, d, C.POINTER(C.c_double), C.POINTER(C.c_int64)],
        "ws_autotune_iso": [h, C.POINTER(C.c_double)], "ws_census": [h, C.POINTER(C.c_double)],
        "ws_kinetic_energy": [h, C.POINTER(C.c_double)],
        "ws_apply_impulse_sphere": [h, d, d, d, d, d, d, d],
        "ws_stir_at": [h, d, d, d, d, d, d, d, d], "ws_stir_gaussian": [h, d, d],
        "ws_wave_impulse": [h, d], "ws_dry_land_fraction": [h, C.POINTER(C.c_double)],
        "ws_sample_vel": [h, C.c_void_p, C.c_int64, C.c_void_p],
        "ws_terrain_radius_at": [h, C.c_void_p, C.c_int64, C.c_void_p],
        "ws_ocean_point": [h, d, C.POINTER(C.c_double)],
        "ws_synchronize": [h], "ws_get_stream": [h, C.POINTER(C.c_void_p)],
        "ws_launch_count": [h, C.POINTER(C.c_int64)],
        "ws_time_kernel": [h, i32, i32, C.POINTER(C.c_double)],
        "ws_probe_wait": [h, C.c_int64],
        "ws_upload_state": [h, C.POINTER(WsHostArrays)], "ws_download_state": [h, C.POINTER(WsHostArrays)],
        "ws_unet_init": [h, u32], "ws_unet_init_levels": [h, u32, i32], "ws_unet_collect": [h, i32], "ws_unet_enable": [h, i32],
        "ws_unet_train": [h, i32, i32, d, u32, C.POINTER(C.c_double)],
        "ws_unet_get_info": [h, C.POINTER(WsUnetInfo)],
        "ws_unet_get_weights": [h, vp, i64], "ws_unet_set_weights": [h, vp, i64], "ws_unet_set_gain": [h, d],
        "ws_unet_get_pair": [h, i32, vp, vp, vp], "ws_unet_put_pair": [h, vp, vp, vp],
        "ws_unet_forward_pair": [h, i32, vp], "ws_unet_grad_pair": [h, i32, vp, C.POINTER(C.c_double)],
        "ws_unet_probe": [h, C.POINTER(C.c_double), C.POINTER(C.c_double)],
        "ws_unet_time": [h, i32, i32, C.POINTER(C.c_double)],
        "ws_unet_accumulate": [h, i32, u32, C.POINTER(C.c_double)],
        "ws_unet_grads": [h, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)],
        "ws_unet_apply": [h, d, i32],
        "ws_snapshot": [h, vp, i64, C.POINTER(C.c_int64)], "ws_restore": [h, vp, i64],
        "ws_unet_save": [h, vp, i64, C.POINTER(C.c_int64)], "ws_unet_load": [h, vp, i64],
        "ws_surface_mesh": [h, d, C.POINTER(C.c_int64), C.POINTER(C.c_double)],
        "ws_surface_download": [h, vp, vp, i64],
        "ws_surface_device": [h, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64)],
        "ws_add_ball": [h, d, d, d, d, d],
        "ws_get_balls": [h, vp, i32, C.POINTER(C.c_int32)],
        "ws_set_balls": [h, vp, i32],
        "ws_step_async": [h, d],
        "ws_step_poll": [h, C.POINTER(C.c_int32)],
        "ws_step_wait": [h],
        "ws_metaball_mesh": [h, d, d, C.POINTER(C.c_int64), C.POINTER(C.c_double)],
        "ws_metaball_download": [h, vp, vp, i64],
        "ws_metaball_device": [h, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64)],
        "ws_metaball_field": [h, vp, i64, C.POINTER(C.c_int32)],
        "ws_render_particles": [h, C.POINTER(WsRenderOpts), C.POINTER(C.c_int32), C.POINTER(C.c_int64)],
        "ws_render_download": [h, vp, vp, vp, vp, vp, i64],
        "ws_render_device": [h] + [C.POINTER(C.c_void_p)] * 5 + [C.POINTER(C.c_int64)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int32
    L.ws_last_error.argtypes = [h]
    L.ws_last_error.restype = C.c_char_p
    L.ws_residual_noalloc.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp]
    L.ws_residual_noalloc.restype = C.c_int32
    L.ws_version.argtypes = []
    L.ws_version.restype = C.c_char_p
    if path is None:
        _lib = L
    return L


class FluidSolver:
    """The FluidSolver of js/solver.js:45-216 on a B200, sphere mode only.

    opts: nx, ny, nz, dx, coreR, terrainSeed, bumpiness, targetParticles,
    capacity (particle capacity; default targetParticles + 8192), device.
    """

    _KNOBS = {f[0] for f in WsParams._fields_} - {"sunPos", "hasSun", "ceilReflect"}

    def __init__(self, **opts):
        object.__setattr__(self, "_h", None)
        L = load_library()
        object.__setattr__(self, "_L", L)
        tp = float(opts.get("targetParticles", 110000))
        cfg = WsConfig(nx=int(opts["nx"]), ny=int(opts["ny"]), nz=int(opts["nz"]),
                       capacity=int(opts.get("capacity", tp + 8192)), dx=float(opts["dx"]),
                       coreR=float(opts.get("coreR", 0.0)), bumpiness=float(opts.get("bumpiness", 1.0)),
                       targetParticles=tp, terrainSeed=int(opts.get("terrainSeed", 20260114)),
                       device=int(opts.get("device", 0)))
        hh = C.c_void_p()
        rc = L.ws_create(C.byref(cfg), C.byref(hh))
        if rc:
            raise WsError(rc, "ws_create failed (no CUDA device or bad options)")
        object.__setattr__(self, "_h", hh)
        object.__setattr__(self, "nx", cfg.nx)
        object.__setattr__(self, "ny", cfg.ny)
        object.__setattr__(self, "nz", cfg.nz)
        object.__setattr__(self, "dx", cfg.dx)
        object.__setattr__(self, "mode", "sphere")
        object.__setattr__(self, "device", cfg.device)
        p = WsParams()
        self._check(L.ws_get_params(hh, C.byref(p)))
        object.__setattr__(self, "_p", p)
        if "vorticity" in opts:
            self.vorticity = opts["vorticity"]

    # ---- lifetime
    def close(self):
        if self._h:
            self._L.ws_destroy(self._h)
            object.__setattr__(self, "_h", None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- balls: addBall (js/solver.js:3910); rows x y z vx vy vz r rho submerged
    def addBall(self, x, y, z, r, rho):
        self._check(self._L.ws_add_ball(self._h, float(x), float(y), float(z), float(r), float(rho)))

    add_ball = addBall

    @property
    def balls(self):
        """(n, 9) float64: x y z vx vy vz r rho submerged of every ball."""
        cnt = C.c_int32()
        out = np.zeros((64, 9))
        self._check(self._L.ws_get_balls(self._h, out.ctypes.data, 64, C.byref(cnt)))
        return out[:cnt.value].copy()

    def set_balls(self, rows):
        a = np.ascontiguousarray(rows, np.float64).reshape(-1, 9)
        self._check(self._L.ws_set_balls(self._h, a.ctypes.data if len(a) else None, len(a)))

    def step_async(self, dtFrame):
        """Start step(dtFrame) on the handle's worker thread; False (nothing
        started) while the previous frame still runs, as GpuSim.step returns
        while busy (js/gpu/gpusim.js:328-339)."""
        rc = self._L.ws_step_async(self._h, float(dtFrame))
        if rc == WS_BUSY:
            return False
        self._check(rc)
        return True

    def step_poll(self):
        """True once the asynchronous frame has ended (raising its error, if any)."""
        done = C.c_int32()
        self._check(self._L.ws_step_poll(self._h, C.byref(done)))
        return bool(done.value)

    def step_wait(self):
        """Block until the asynchronous frame ends; raises its error, if any."""
        self._check(self._L.ws_step_wait(self._h))

    def _check(self, rc):
        if rc:
            raise WsError(rc, self._L.ws_last_error(self._h).decode(errors="replace"))

    # ---- knobs: attribute writes go straight to ws_set_params
    def __setattr__(self, k, v):
        if k in FluidSolver._KNOBS:
            setattr(self._p, k, v)
            self._check(self._L.ws_set_params(self._h, C.byref(self._p)))
        elif k == "sunPos":
            if v is None:
                self._p.hasSun = 0
            else:
                self._p.hasSun = 1
                for i in range(3):
                    self._p.sunPos[i] = float(v[i])
            self._check(self._L.ws_set_params(self._h, C.byref(self._p)))
        elif k == "ceilReflect":
            self._p.ceilReflect = CEIL[v] if isinstance(v, str) else int(v)
            self._check(self._L.ws_set_params(self._h, C.byref(self._p)))
        elif k in FIELDS:
            self.upload(k, v)
        elif k in {f[0] for f in WsScalars._fields_}:
            self.set_scalars(**{k: v})
        else:
            object.__setattr__(self, k, v)

    def __getattr__(self, k):
        if k.startswith("_"):
            raise AttributeError(k)
        if k in FluidSolver._KNOBS:
            return getattr(self._p, k)
        if k == "sunPos":
            return list(self._p.sunPos) if self._p.hasSun else None
        if k in FIELDS:
            return self.download(k)
        if k in {f[0] for f in WsScalars._fields_}:
            return getattr(self.scalars, k)
        raise AttributeError(k)

    def set_params(self, **kw):
        for k, v in kw.items():
            if k == "sunPos":
                if v is None:
                    self._p.hasSun = 0
                else:
                    self._p.hasSun = 1
                    for i in range(3):
                        self._p.sunPos[i] = float(v[i])
            elif k == "ceilReflect":
                self._p.ceilReflect = CEIL[v] if isinstance(v, str) else int(v)
            else:
                setattr(self._p, k, v)
        self._check(self._L.ws_set_params(self._h, C.byref(self._p)))

    @property
    def scalars(self):
        s = WsScalars()
        self._check(self._L.ws_get_scalars(self._h, C.byref(s)))
        return s

    def set_scalars(self, **kw):
        s = self.scalars
        for k, v in kw.items():
            setattr(s, k, v)
        self._check(self._L.ws_set_scalars(self._h, C.byref(s)))

    # ---- fields
    def field_size(self, name):
        cnt, elem = C.c_int64(), C.c_int32()
        self._check(self._L.ws_field_info(self._h, FIELDS[name][0], C.byref(cnt), C.byref(elem)))
        return cnt.value

    def download(self, name, count=None):
        fid, dt = FIELDS[name]
        if count is None:
            count = self.scalars.nP if name in PARTICLE_FIELDS else self.field_size(name)
        out = np.empty(count, dt)
        self._check(self._L.ws_download_field(self._h, fid, out.ctypes.data, count))
        return out

    def upload(self, name, arr):
        fid, dt = FIELDS[name]
        a = np.ascontiguousarray(arr, dt)
        self._check(self._L.ws_upload_field(self._h, fid, a.ctypes.data, a.size))

    def _host_arrays(self, arrays, count):
        a = WsHostArrays()
        a.count = int(count)
        keep = []
        for name, arr in arrays.items():
            fid, dt = FIELDS[name]
            if name not in PARTICLE_FIELDS:
                raise ValueError("%s is not a particle field" % name)
            if arr.dtype != dt or not arr.flags.c_contiguous or arr.size < count:
                raise ValueError("%s: need a contiguous %s array of >= %d elements" % (name, np.dtype(dt), count))
            a.field[fid] = arr.ctypes.data
            keep.append(arr)
        return a, keep

    def upload_state(self, arrays, count=None):
        """Copy several particle fields host -> device in one call (one synchronisation).
        arrays maps field name -> contiguous array of that field's dtype; pinned
        buffers copy at full link speed."""
        count = self.scalars.nP if count is None else count
        a, _keep = self._host_arrays(arrays, count)
        self._check(self._L.ws_upload_state(self._h, C.byref(a)))

    def download_state(self, arrays, count=None):
        """Copy several particle fields device -> host into the given arrays (one synchronisation)."""
        count = self.scalars.nP if count is None else count
        a, _keep = self._host_arrays(arrays, count)
        self._check(self._L.ws_download_state(self._h, C.byref(a)))

    # ---- learned warm start of the pressure solve (no reference counterpart)
    def unet_init(self, seed=1, levels=3):
        self._check(self._L.ws_unet_init_levels(self._h, int(seed), int(levels)))

    def unet_collect(self, capacity):
        self._check(self._L.ws_unet_collect(self._h, int(capacity)))

    def unet_enable(self, on=True):
        self._check(self._L.ws_unet_enable(self._h, 1 if on else 0))

    def unet_train(self, steps, batch=4, lr=1e-3, seed=1):
        loss = C.c_double()
        self._check(self._L.ws_unet_train(self._h, int(steps), int(batch), float(lr), int(seed), C.byref(loss)))
        return loss.value

    def unet_info(self):
        i = WsUnetInfo()
        self._check(self._L.ws_unet_get_info(self._h, C.byref(i)))
        return {f[0]: getattr(i, f[0]) for f in i._fields_}

    def unet_weights(self):
        n = self.unet_info()["num_weights"]
        w = np.empty(n, np.float32)
        self._check(self._L.ws_unet_get_weights(self._h, w.ctypes.data, n))
        return w

    def unet_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self._L.ws_unet_set_weights(self._h, w.ctypes.data, w.size))

    def unet_set_gain(self, g):
        self._check(self._L.ws_unet_set_gain(self._h, float(g)))

    def unet_pair(self, idx):
        N = self.nx * self.ny * self.nz
        r0n, types, target = np.empty(N, np.float32), np.empty(N, np.uint8), np.empty(N, np.float32)
        self._check(self._L.ws_unet_get_pair(self._h, int(idx), r0n.ctypes.data, types.ctypes.data,
                                             target.ctypes.data))
        return r0n, types, target

    def unet_put_pair(self, r0n, types, target):
        r0n = np.ascontiguousarray(r0n, np.float32)
        types = np.ascontiguousarray(types, np.uint8)
        target = np.ascontiguousarray(target, np.float32)
        self._check(self._L.ws_unet_put_pair(self._h, r0n.ctypes.data, types.ctypes.data, target.ctypes.data))

    def unet_forward_pair(self, idx):
        out = np.empty(self.nx * self.ny * self.nz, np.float32)
        self._check(self._L.ws_unet_forward_pair(self._h, int(idx), out.ctypes.data))
        return out

    def unet_grad_pair(self, idx):
        g = np.empty(self.unet_info()["num_weights"], np.float32)
        loss = C.c_double()
        self._check(self._L.ws_unet_grad_pair(self._h, int(idx), g.ctypes.data, C.byref(loss)))
        return g, loss.value

    def unet_probe(self):
        a, b = C.c_double(), C.c_double()
        self._check(self._L.ws_unet_probe(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def unet_time(self, what, reps=10):
        ms = C.c_double()
        self._check(self._L.ws_unet_time(self._h, int(what), int(reps), C.byref(ms)))
        return ms.value

    # data-parallel training pieces (watersim-v1_b200/dp_train.py drives them)
    def unet_accumulate(self, samples, seed):
        loss = C.c_double()
        self._check(self._L.ws_unet_accumulate(self._h, int(samples), int(seed) & 0xffffffff, C.byref(loss)))
        return loss.value

    def unet_grads(self):
        """The FP32 gradient buffer as a CUDA tensor sharing the library's memory."""
        import torch
        ptr, n = C.c_void_p(), C.c_int64()
        self._check(self._L.ws_unet_grads(self._h, C.byref(ptr), C.byref(n)))

        class _View:
            __cuda_array_interface__ = {"shape": (n.value,), "typestr": "<f4", "data": (ptr.value, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device="cuda:%d" % self.device)

    def unet_apply(self, lr, total_samples):
        self._check(self._L.ws_unet_apply(self._h, float(lr), int(total_samples)))

    # ---- surface mesh (marching tets of the splatted density)
    def surface_mesh(self, iso=None):
        """(volume, positions (V,3), normals (V,3)) of the iso-surface of the
        current density field (splat it first with stage('SPLAT'))."""
        n, vol = C.c_int64(), C.c_double()
        iso = self.scalars.iso if iso is None else iso
        self._check(self._L.ws_surface_mesh(self._h, float(iso), C.byref(n), C.byref(vol)))
        pos = np.empty((n.value, 3), np.float32)
        nrm = np.empty((n.value, 3), np.float32)
        self._check(self._L.ws_surface_download(self._h, pos.ctypes.data, nrm.ctypes.data, n.value))
        return vol.value, pos, nrm

    def metaballs(self, tension=0.5, detail=None, field=False):
        """Metaballs.build(solver, tension, detail): (volume, positions (V,3),
        normals (V,3)) of the metaball skin over the liquid particles; with
        field, also the (m+1)^3 corner field and m."""
        n, vol = C.c_int64(), C.c_double()
        det = float("nan") if detail is None else float(detail)
        self._check(self._L.ws_metaball_mesh(self._h, float(tension), det, C.byref(n), C.byref(vol)))
        pos = np.empty((n.value, 3), np.float32)
        nrm = np.empty((n.value, 3), np.float32)
        self._check(self._L.ws_metaball_download(self._h, pos.ctypes.data, nrm.ctypes.data, n.value))
        if not field:
            return vol.value, pos, nrm
        m = C.c_int32()
        self._check(self._L.ws_metaball_field(self._h, None, 0, C.byref(m)))
        f = np.empty((m.value + 1) ** 3, np.float32)
        self._check(self._L.ws_metaball_field(self._h, f.ctypes.data, f.size, C.byref(m)))
        return vol.value, pos, nrm, f, m.value

    # ---- render-side particle prep (WaterScene.updateParticles)
    def render_particles(self, opts=None, download=True, **kw):
        """Classify, colour and sort the particles far to near into the
        handle's draw list. Returns (counts dict by class, points) and, with
        download, a dict of host arrays pos (P,3), col (P,3), alpha, size,
        sprite. opts is a WsRenderOpts (render_opts(**kw) when None)."""
        o = opts if opts is not None else render_opts(**kw)
        cnt = (C.c_int32 * 5)()
        pts = C.c_int64()
        self._check(self._L.ws_render_particles(self._h, C.byref(o), cnt, C.byref(pts)))
        counts = dict(zip(RENDER_CLASSES, list(cnt)))
        if not download:
            return counts, pts.value
        n = pts.value
        out = {"pos": np.empty((n, 3), np.float32), "col": np.empty((n, 3), np.float32),
               "alpha": np.empty(n, np.float32), "size": np.empty(n, np.float32), "sprite": np.empty(n, np.float32)}
        self._check(self._L.ws_render_download(self._h, out["pos"].ctypes.data, out["col"].ctypes.data,
                                               out["alpha"].ctypes.data, out["size"].ctypes.data,
                                               out["sprite"].ctypes.data, n))
        return counts, n, out

    # ---- snapshot / restore (versioned host blobs)
    def snapshot(self):
        n = C.c_int64()
        self._check(self._L.ws_snapshot(self._h, None, 0, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(self._L.ws_snapshot(self._h, buf.ctypes.data, buf.size, C.byref(n)))
        return buf

    def restore(self, blob):
        blob = np.ascontiguousarray(blob, np.uint8)
        self._check(self._L.ws_restore(self._h, blob.ctypes.data, blob.size))

    def unet_save(self):
        n = C.c_int64()
        self._check(self._L.ws_unet_save(self._h, None, 0, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(self._L.ws_unet_save(self._h, buf.ctypes.data, buf.size, C.byref(n)))
        return buf

    def unet_load(self, blob):
        blob = np.ascontiguousarray(blob, np.uint8)
        self._check(self._L.ws_unet_load(self._h, blob.ctypes.data, blob.size))

    def set_nparticles(self, n):
        self._check(self._L.ws_set_nparticles(self._h, int(n)))

    # ---- world setup
    def generateTerrain(self, seed, seaLevel):
        self._check(self._L.ws_generate_terrain(self._h, int(seed), float(seaLevel)))

    def upload_terrain(self, t):
        solid = np.ascontiguousarray(t["solid"], np.uint8)
        R = np.ascontiguousarray(t["R"], np.float32)
        wt = WsTerrain(n=int(t["n"]), dv=float(t["dv"]), Rsl=float(t["Rsl"]), Rlo=float(t["Rlo"]),
                       Rhi=float(t["Rhi"]), landFrac=float(t["landFrac"]),
                       solid=solid.ctypes.data, R=R.ctypes.data)
        self._check(self._L.ws_upload_terrain(self._h, C.byref(wt)))

    def terrain(self):
        meta = (C.c_double * 4)()
        self._check(self._L.ws_download_terrain(self._h, None, None, meta))
        n = int(meta[0])
        solid = np.empty(n ** 3, np.uint8)
        R = np.empty(n ** 3, np.float32)
        self._check(self._L.ws_download_terrain(self._h, solid.ctypes.data, R.ctypes.data, meta))
        return {"n": n, "solid": solid, "R": R, "Rlo": meta[1], "Rhi": meta[2], "landFrac": meta[3]}

    def water_volume(self, depth):
        v = C.c_double()
        self._check(self._L.ws_water_volume(self._h, float(depth), C.byref(v)))
        return v.value

    def resetWater(self, depth):
        self._check(self._L.ws_reset_water(self._h, float(depth)))

    # ---- drivers
    def step(self, dtFrame):
        self._check(self._L.ws_step(self._h, float(dtFrame)))

    def _substep(self, dt):
        self._check(self._L.ws_substep(self._h, float(dt)))

    substep = _substep

    def stage(self, name, dt=0.0):
        self._check(self._L.ws_stage(self._h, STAGES.index(name), float(dt)))

    # ---- reductions and helpers
    def residual(self):
        r = C.c_double()
        self._check(self._L.ws_residual(self._h, C.byref(r)))
        return r.value

    def splatDensity(self):
        self.stage("SPLAT")

    def mt_volume(self, iso):
        v, n = C.c_double(), C.c_int64()
        self._check(self._L.ws_mt_volume(self._h, float(iso), C.byref(v), C.byref(n)))
        return v.value, n.value

    def autotuneIso(self):
        v = C.c_double()
        self._check(self._L.ws_autotune_iso(self._h, C.byref(v)))
        return v.value

    def census(self):
        out = (C.c_double * 3)()
        self._check(self._L.ws_census(self._h, out))
        return tuple(out)

    def kineticEnergy(self):
        v = C.c_double()
        self._check(self._L.ws_kinetic_energy(self._h, C.byref(v)))
        return v.value

    def applyImpulseSphere(self, cx, cy, cz, R, fx, fy, fz):
        self._check(self._L.ws_apply_impulse_sphere(self._h, cx, cy, cz, R, fx, fy, fz))

    def stirAt(self, cx, cy, cz, vx, vy, vz, R, dt):
        self._check(self._L.ws_stir_at(self._h, cx, cy, cz, vx, vy, vz, R, dt))

    def stir_gaussian(self, sigma, peak):
        self._check(self._L.ws_stir_gaussian(self._h, float(sigma), float(peak)))

    def waveImpulse(self, dvx):
        """waveImpulse (js/solver.js:3866), draws from the seeded stir stream."""
        self._check(self._L.ws_wave_impulse(self._h, float(dvx)))

    def dryLandFraction(self):
        v = C.c_double()
        self._check(self._L.ws_dry_land_fraction(self._h, C.byref(v)))
        return v.value

    def sample_vel(self, points):
        """sampleVel at an (n, 3) array of points -> (n, 3) float64."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.empty_like(pts)
        self._check(self._L.ws_sample_vel(self._h, pts.ctypes.data, pts.shape[0], out.ctypes.data))
        return out

    def sampleVel(self, x, y, z):
        return tuple(self.sample_vel([[x, y, z]])[0])

    def terrain_radius_at(self, points):
        """terrainRadiusAt at an (n, 3) array of points -> (n,) float64."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.empty(pts.shape[0], np.float64)
        self._check(self._L.ws_terrain_radius_at(self._h, pts.ctypes.data, pts.shape[0], out.ctypes.data))
        return out

    def terrainRadiusAt(self, x, y, z):
        return float(self.terrain_radius_at([[x, y, z]])[0])

    def oceanPoint(self, minDepth=0.0):
        """oceanPoint (js/solver.js:591), draws from the seeded stir stream."""
        out = (C.c_double * 3)()
        self._check(self._L.ws_ocean_point(self._h, float(minDepth), out))
        return [out[0], out[1], out[2]]

    def synchronize(self):
        self._check(self._L.ws_synchronize(self._h))

    def stream(self):
        s = C.c_void_p()
        self._check(self._L.ws_get_stream(self._h, C.byref(s)))
        return s.value

    def launch_count(self):
        n = C.c_int64()
        self._check(self._L.ws_launch_count(self._h, C.byref(n)))
        return n.value

    def probe_wait(self, polls):
        """One bounded device wait on a word nothing sets (ws_probe_wait):
        raises WsError with WS_ERR_TIMEOUT when it runs out, as a timed-out
        solve does; the handle stays usable."""
        self._check(self._L.ws_probe_wait(self._h, int(polls)))

    def time_kernel(self, kernel, reps=20):
        """Mean microseconds per launch of one kernel group (ws_time_kernel)."""
        us = C.c_double()
        self._check(self._L.ws_time_kernel(self._h, int(kernel), int(reps), C.byref(us)))
        return us.value

"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of liboracle_render.so, the CPU
restatement of WaterScene.updateParticles (js/scene.js:1595-1922) in
oracle/ws_render_oracle.c. Only tests/ (and the bench's CPU timing leg) load
it, as the checker of ws_render_particles."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_L = None
CLASSES = ("beads", "spray", "vapor", "cloud", "snow")


class OrRenderOpts(C.Structure):
    """Scene state read by updateParticles; laid out as ws_render_opts."""
    _fields_ = [("show", C.c_int32), ("beadsMode", C.c_int32), ("metaballMode", C.c_int32),
                ("spinColor", C.c_int32), ("cloudSprite", C.c_int32), ("planetLit", C.c_int32),
                ("sortOn", C.c_int32), ("useLight", C.c_int32), ("useDepth", C.c_int32),
                ("useTemp", C.c_int32), ("waterOpa", C.c_double), ("pOpa", C.c_double),
                ("wScale", C.c_double), ("waterColor", C.c_double * 3), ("sunDir", C.c_double * 3),
                ("cam", C.c_double * 3)]


def make_opts(**kw):
    """OrRenderOpts from keyword fields (unset ints 0, doubles 0)."""
    o = OrRenderOpts()
    for k, v in kw.items():
        if k in ("waterColor", "sunDir", "cam"):
            getattr(o, k)[:] = tuple(float(x) for x in v)
        else:
            setattr(o, k, v)
    return o


def _lib():
    global _L
    if _L is None:
        path = os.path.join(_HERE, "liboracle_render.so")
        if not os.path.exists(path):
            raise OSError("liboracle_render.so not built; run make -C oracle")
        L = C.CDLL(path)
        vp, d, i32 = C.c_void_p, C.c_double, C.c_int
        L.or_render_particles.restype = C.c_int64
        L.or_render_particles.argtypes = [vp, d, d, d, d, i32, i32] + [vp] * 11 + [vp] * 5 + [vp]
        _L = L
    return _L


def render_particles(opts, center, spacing, spin_on, f):
    """opts: a structure laid out as ws_render_opts; center: the box centre
    (W/2, H/2, D/2); f: dict of the particle arrays px py pz pflag pT pLight
    pDepth pPh pWx pWy pWz (first n entries used, n = len(f['px'])).
    Returns (counts by class, points, dict pos col alpha size sprite)."""
    L = _lib()
    n = len(f["px"])
    a = {k: np.ascontiguousarray(f[k], np.uint8 if k in ("pflag", "pDepth") else np.float32)
         for k in ("px", "py", "pz", "pflag", "pT", "pLight", "pDepth", "pPh", "pWx", "pWy", "pWz")}
    m = max(n, 1)
    out = {"pos": np.zeros((m, 3), np.float32), "col": np.zeros((m, 3), np.float32),
           "alpha": np.zeros(m, np.float32), "size": np.zeros(m, np.float32), "sprite": np.zeros(m, np.float32)}
    cnt = (C.c_int32 * 5)()
    pts = L.or_render_particles(C.addressof(opts), float(center[0]), float(center[1]), float(center[2]),
                                float(spacing), int(spin_on), n,
                                *[a[k].ctypes.data for k in ("px", "py", "pz", "pflag", "pT", "pLight", "pDepth",
                                                             "pPh", "pWx", "pWy", "pWz")],
                                *[out[k].ctypes.data for k in ("pos", "col", "alpha", "size", "sprite")], cnt)
    return dict(zip(CLASSES, list(cnt))), pts, {k: v[:pts] for k, v in out.items()}

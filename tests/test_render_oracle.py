"""The render-prep oracle (oracle/ws_render_oracle.c) against the reference's
own known answers for WaterScene.updateParticles (test/scene_fx.test.js:
111-283 and test/metaball.test.js:266-288): class routing, counts, per-class
sprite tiles, alphas and sizes, far-to-near order, bead modes, the night-side
interior cull, spin-velocity colours and the hidden cases."""
import ctypes as C
import math

import numpy as np

from oracle.render_oracle import make_opts, render_particles, OrRenderOpts

CAP = 6


def fx_solver(**extra):
    f = {"px": np.array([1, 2, 3, 4, 5, 6], np.float32), "py": np.zeros(CAP, np.float32),
         "pz": np.zeros(CAP, np.float32), "pflag": np.array([0, 1, 2, 3, 4, 5], np.uint8),
         "pT": np.full(CAP, 0.3, np.float32), "pLight": np.zeros(CAP, np.float32),
         "pDepth": np.zeros(CAP, np.uint8), "pPh": np.zeros(CAP, np.float32),
         "pWx": np.zeros(CAP, np.float32), "pWy": np.zeros(CAP, np.float32), "pWz": np.zeros(CAP, np.float32)}
    f.update(extra)
    return f


def fx_opts(**kw):
    # scene_fx.test.js:126-148: camera at x=30 in the planet frame, sorted,
    # unlit, no exposure or depth mirrors, water hue (0.2, 0.5, 0.9)
    base = dict(show=1, beadsMode=0, metaballMode=0, spinColor=0, cloudSprite=0, planetLit=0, sortOn=1,
                useLight=0, useDepth=0, useTemp=1, waterOpa=0.5, pOpa=1.0, wScale=1.0,
                waterColor=(0.2, 0.5, 0.9), sunDir=(0, 1, 0), cam=(30, 0, 0))
    base.update(kw)
    return make_opts(**base)


def run(opts, f, center=(float("nan"),) * 3, spacing=0.2, spin_on=0):
    return render_particles(opts, center, spacing, spin_on, f)


def test_classes_sprites_alpha_size_order():
    cnt, n, out = run(fx_opts(), fx_solver())
    assert n == 5
    assert [cnt[k] for k in ("beads", "spray", "vapor", "cloud", "snow")] == [0, 2, 1, 1, 1]
    assert list(out["sprite"]) == [1, 2, 3, 1, 4]
    spr, al, sz = out["sprite"], out["alpha"], out["size"]
    assert any(abs(a - 0.23) < 1e-6 for a, s in zip(al, spr) if s == 2)
    assert all(abs(a - 0.88) < 1e-6 for a, s in zip(al, spr) if s == 3)
    assert all(a == 1 for a, s in zip(al, spr) if s == 4)
    size_of = lambda t: sz[list(spr).index(t)]
    assert abs(size_of(4) - 0.2 * 3.4) < 1e-6
    assert size_of(3) > size_of(2)
    assert abs(out["pos"][0, 0] - 2) < 1e-6 and abs(out["pos"][4, 0] - 6) < 1e-6


def test_beads_and_metaball_modes():
    cnt, n, out = run(fx_opts(beadsMode=1), fx_solver())
    assert n == 6 and cnt["beads"] == 1
    i = list(out["sprite"]).index(0)
    assert abs(out["alpha"][i] - 0.5) < 1e-6
    cnt, n, _ = run(fx_opts(beadsMode=1, metaballMode=1), fx_solver())
    assert n == 5 and cnt["beads"] == 0
    cnt, n, _ = run(fx_opts(), fx_solver())
    assert n == 5


def test_night_side_interior_cull():
    depth = np.array([4, 4, 4, 4, 0, 2], np.uint8)
    c = (3.0, 3.0, 3.0)                                   # W = H = D = 6
    cnt, _, _ = run(fx_opts(beadsMode=1, planetLit=1, useDepth=1, sunDir=(1, 0, 0)), fx_solver(pDepth=depth), c)
    assert cnt["beads"] == 0
    cnt, _, out = run(fx_opts(beadsMode=1, planetLit=1, useDepth=1, sunDir=(-1, 0, 0)), fx_solver(pDepth=depth), c)
    assert cnt["beads"] == 1
    j = list(out["sprite"]).index(0)
    assert abs(out["col"][j, 0] - 0.2 * (0.9 + 0.1 * math.pow(0.3, 1.4))) < 0.01
    cnt, _, _ = run(fx_opts(beadsMode=1, planetLit=1, useDepth=0, sunDir=(1, 0, 0)), fx_solver(pDepth=depth), c)
    assert cnt["beads"] == 1


def test_spin_velocity_colours():
    f = fx_solver(pWx=np.array([-1, 0, 0.5, 1, 0, 2], np.float32), pWy=np.full(CAP, 2, np.float32),
                  pWz=np.array([0, 4, 1, 3, 2, 0], np.float32))
    _, n, out = run(fx_opts(beadsMode=1, spinColor=1), f)
    want = [(0, 0.5, 0), (1 / 3, 0.5, 1), (0.5, 0.5, 0.25), (2 / 3, 0.5, 0.75), (1 / 3, 0.5, 0.5), (1, 0.5, 0)]
    assert n == 6
    np.testing.assert_allclose(out["col"], np.array(want), atol=1e-6)


def test_hidden_cases():
    cnt, n, _ = run(fx_opts(pOpa=0.0), fx_solver())
    assert n == 0 and sum(cnt.values()) == 0
    cnt, n, _ = run(fx_opts(show=0, beadsMode=1), fx_solver())
    assert n == 0
    # metaball.test.js:266-288: one liquid particle, spray opacity 0
    one = {k: v[:1] for k, v in fx_solver(px=np.array([0.5] * 6, np.float32)).items()}
    kw = dict(beadsMode=1, pOpa=0.0, waterOpa=0.25, sortOn=0, sunDir=(0, 1, 0))
    _, n, _ = run(fx_opts(metaballMode=1, **kw), one, (0.5, 0.5, 0.5))
    assert n == 0
    _, n, _ = run(fx_opts(metaballMode=0, **kw), one, (0.5, 0.5, 0.5))
    assert n == 1


def test_opts_layout_matches_library():
    import fluid_solver
    assert [f[0] for f in fluid_solver.WsRenderOpts._fields_] == [f[0] for f in OrRenderOpts._fields_]
    assert C.sizeof(fluid_solver.WsRenderOpts) == C.sizeof(OrRenderOpts) == 40 + 12 * 8

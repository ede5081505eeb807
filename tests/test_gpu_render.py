"""ws_render_particles against the render-prep oracle (WaterScene.updateParticles,
js/scene.js:1595-1922) on the same particles and scene state: the same class
counts and point count, bit-identical positions, alphas, sizes and sprite
tiles in the same far-to-near order, and colours equal to the float ulp (the
oracle's pow/cos are the host's, the device's are CUDA's: 2.5e-7 absolute).
Cases: the reference's own fixture (test/scene_fx.test.js), every scene switch
on seeded random particles of all flags, ragged sizes around the 2048-particle
chunk, and the 2M-particle size of the 128^3 workload."""
import numpy as np
import pytest

from fluid_solver import FluidSolver, render_opts
from oracle.render_oracle import render_particles as oracle_render

pytestmark = pytest.mark.gpu

COL_TOL = 2.5e-7
FIELDS = ("px", "py", "pz", "pflag", "pT", "pLight", "pDepth", "pPh", "pWx", "pWy", "pWz")


def solver(n_cap, n=24, dx=1.0):
    return FluidSolver(nx=n, ny=n, nz=n, dx=dx, coreR=n * 0.3, targetParticles=1000, capacity=n_cap)


def random_particles(n, W, seed):
    r = np.random.default_rng(seed)
    f = {"px": r.uniform(0, W, n).astype(np.float32), "py": r.uniform(0, W, n).astype(np.float32),
         "pz": r.uniform(0, W, n).astype(np.float32), "pflag": r.integers(0, 7, n).astype(np.uint8),
         "pT": r.uniform(-0.2, 1.2, n).astype(np.float32), "pLight": r.uniform(-0.5, 1.5, n).astype(np.float32),
         "pDepth": r.integers(0, 5, n).astype(np.uint8), "pPh": r.uniform(-7, 7, n).astype(np.float32),
         "pWx": r.normal(0, 1, n).astype(np.float32), "pWy": r.normal(0, 2, n).astype(np.float32),
         "pWz": r.normal(0.5, 1, n).astype(np.float32)}
    f["pLight"][::97] = np.nan                            # the reference's !(expo > 0) path
    return f


def load(fs, f):
    n = len(f["px"])
    fs.set_scalars(nP=n)
    if n:
        fs.upload_state({k: np.ascontiguousarray(v) for k, v in f.items()}, count=n)


def compare(fs, f, opts):
    center = (fs.nx * fs.dx * 0.5, fs.ny * fs.dx * 0.5, fs.nz * fs.dx * 0.5)
    cnt, n, out = fs.render_particles(opts)
    rc, rn, ref = oracle_render(opts, center, fs.scalars.spacing, fs._p.spinOn, f)
    assert cnt == rc and n == rn
    for k in ("pos", "alpha", "size", "sprite"):
        assert np.array_equal(out[k], ref[k]), k
    if n:
        assert np.max(np.abs(out["col"].astype(np.float64) - ref["col"])) <= COL_TOL
    return cnt, n


def test_reference_fixture():
    fs = solver(64, n=24, dx=0.25)                        # box centre (3, 3, 3) as in the fixture
    fs.set_scalars(spacing=0.2)
    z = np.zeros(6, np.float32)
    f = {"px": np.arange(1, 7, dtype=np.float32), "py": z, "pz": z, "pflag": np.arange(6, dtype=np.uint8),
         "pT": np.full(6, 0.3, np.float32), "pLight": z, "pDepth": np.array([4, 4, 4, 4, 0, 2], np.uint8),
         "pPh": z, "pWx": np.array([-1, 0, 0.5, 1, 0, 2], np.float32), "pWy": np.full(6, 2, np.float32),
         "pWz": np.array([0, 4, 1, 3, 2, 0], np.float32)}
    load(fs, f)
    base = dict(waterOpa=0.5, waterColor=(0.2, 0.5, 0.9), sunDir=(0, 1, 0), cam=(30, 0, 0), planetLit=0,
                useLight=0, useDepth=0)
    cnt, n = compare(fs, f, render_opts(**base))
    assert n == 5 and [cnt[k] for k in ("beads", "spray", "vapor", "cloud", "snow")] == [0, 2, 1, 1, 1]
    _, _, out = fs.render_particles(render_opts(**base))
    assert list(out["sprite"]) == [1, 2, 3, 1, 4]
    assert compare(fs, f, render_opts(**dict(base, beadsMode=1)))[1] == 6
    assert compare(fs, f, render_opts(**dict(base, beadsMode=1, metaballMode=1)))[1] == 5
    night = dict(base, beadsMode=1, planetLit=1, useDepth=1, sunDir=(1, 0, 0))
    assert compare(fs, f, render_opts(**night))[0]["beads"] == 0
    assert compare(fs, f, render_opts(**dict(night, sunDir=(-1, 0, 0))))[0]["beads"] == 1
    cnt, n = compare(fs, f, render_opts(**dict(base, beadsMode=1, spinColor=1)))
    _, _, out = fs.render_particles(render_opts(**dict(base, beadsMode=1, spinColor=1)))
    np.testing.assert_allclose(out["col"], [(0, 0.5, 0), (1 / 3, 0.5, 1), (0.5, 0.5, 0.25), (2 / 3, 0.5, 0.75),
                                            (1 / 3, 0.5, 0.5), (1, 0.5, 0)], atol=1e-6)
    assert compare(fs, f, render_opts(**dict(base, pOpa=0.0)))[1] == 0


SWITCHES = [
    dict(),
    dict(beadsMode=1),
    dict(beadsMode=1, useLight=0),
    dict(beadsMode=1, useDepth=0, useTemp=0),
    dict(beadsMode=1, planetLit=0),
    dict(beadsMode=1, spinColor=1),
    dict(sortOn=0, beadsMode=1),
    dict(cloudSprite=1, pOpa=0.3, wScale=2.5),
    dict(beadsMode=1, waterOpa=0.005),
    dict(beadsMode=1, pOpa=0.0),
    dict(show=0, beadsMode=1),
]


@pytest.mark.parametrize("sw", range(len(SWITCHES)))
def test_scene_switches_random(sw):
    n = 50000
    fs = solver(n + 100)
    W = fs.nx * fs.dx
    f = random_particles(n, W, 11 + sw)
    load(fs, f)
    opts = render_opts(cam=(W * 0.5, W * 0.6, W * 0.4), sunDir=(0.6, 0.8, 0.0), **SWITCHES[sw])
    compare(fs, f, opts)
    fs.set_params(spinOn=1)                               # spin twinkle on the vapour and cloud colours
    compare(fs, f, opts)


@pytest.mark.parametrize("n", [0, 1, 2, 31, 2047, 2048, 2049, 3 * 2048 + 17])
def test_ragged_sizes(n):
    fs = solver(max(n, 1) + 64)
    W = fs.nx * fs.dx
    f = random_particles(n, W, 100 + n)
    load(fs, f)
    compare(fs, f, render_opts(beadsMode=1, cam=(-3 * W, 0.2 * W, 1.1 * W), sunDir=(0, 0, 1)))


def test_two_million_particles_camera_inside():
    n = 2_000_000
    fs = solver(n + 64, n=128, dx=1.0)
    W = fs.nx * fs.dx
    f = random_particles(n, W, 7)
    load(fs, f)
    cnt, pts = compare(fs, f, render_opts(beadsMode=1, cam=(W * 0.5, W * 0.5, W * 0.5), sunDir=(0.0, 0.6, 0.8)))
    assert pts > 1_500_000
    # a second call on the same buffers gives the same list
    assert fs.render_particles(render_opts(beadsMode=1, cam=(W * 0.5,) * 3, sunDir=(0.0, 0.6, 0.8)),
                               download=False) == (cnt, pts)

"""Parity of the per-frame passes (thermal tick, evaporation, phases,
rescue, density splat, FP64 reductions, impulses) and of the vapour branch
of advection against the oracle, on the 64^3 planet with the sun on.

Exactness: flags, depths, RNG states and counts are bit-exact; temperatures
and exposures within 1e-6 absolute (FP64 conduction sums are accumulated in a
different order, transcendental functions differ in the last ulp); the
marching-tets volume and the census in FP64 to 1e-9 relative.
"""
import math

import numpy as np
import pytest

from helpers import planet, to_device, rel_err, DEVICE_ORDER

pytestmark = pytest.mark.gpu

THERMAL64 = dict(pic=0.05, omega=1.7, maxSpeed=3.2, thermalOn=1, vorticity=0.05, sunActivity=0.6,
                 evapIntensity=0.05, sorTol=1e-5, sorCheckEvery=10, sorMaxIters=3000)
TILT = math.radians(23.4)


def _sun(o, dist=3.0):
    c = o.nx / 2
    R = o.scalars.oceanR * dist
    return [c + R * math.cos(TILT), c + R * math.sin(TILT), c]


def _state64():
    o = planet("planet64", **THERMAL64)
    o.set(sunPos=_sun(o))
    o.set_scalars(gRamp=1.5)
    o.substep(0.01)
    o.substep(0.01)
    o.stage("splat_density")
    return o


def test_heat_tick_parity():
    o = _state64()
    fs = to_device(o, with_grid=True)
    o.stage("update_heat", 1 / 12)
    fs.stage("HEAT", 1 / 12)
    nP = o.nP
    assert np.array_equal(fs.pDepth, o.pDepth[:nP])
    assert np.max(np.abs(fs.pLight.astype(np.float64) - o.pLight[:nP])) <= 1e-6
    assert np.max(np.abs(fs.pT.astype(np.float64) - o.pT[:nP])) <= 1e-6
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-6, k


def test_evaporation_parity():
    o = _state64()
    o.set(sunActivity=2.0, evapIntensity=1.0)
    nP = o.nP
    rng = np.random.default_rng(7)
    o.pT[:nP] = rng.uniform(0.2, 1.0, nP).astype(np.float32)
    fs = to_device(o, with_grid=True)
    o.stage("update_evaporation", 1 / 12)
    fs.stage("EVAPORATION", 1 / 12)
    so, sg = o.scalars, fs.scalars
    assert sg.evapCount == so.evapCount and so.evapCount > 10
    assert sg.evS == so.evS
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-6, k


def _lcg_back(x, n):
    """The _evS state n draws before x (the generator is a bijection mod 2^32)."""
    a_inv = pow(1664525, -1, 2**32)
    for _ in range(n):
        x = (a_inv * (x - 1013904223)) % 2**32
    return x


@pytest.mark.parametrize("where", ["first", "second_window"])
def test_evaporation_irregular_kick(where):
    """A kick whose Box-Muller u1 draw is below 1e-9 takes an extra draw and
    shifts every later stream position (js/solver.js:3118-3125). With every
    candidate ejecting (prob capped at 1), candidate t decides on draw 7t + 1
    and draws its first u1 at 7t + 2; the start state is set so that this u1
    state is 3, i.e. u1 = 7e-10, at the first candidate or one in the second
    window of 4096 candidates."""
    def hot_state():
        o = _state64()
        o.set(sunActivity=2.0, evapIntensity=1.0)
        nP = o.nP
        o.pT[:nP] = np.random.default_rng(9).uniform(0.9, 1.0, nP).astype(np.float32)
        return o
    probe = hot_state()
    probe.stage("update_evaporation", 1 / 12)
    nC = probe.scalars.evapCount
    t = 0 if where == "first" else 4096 + 17
    if t >= nC:
        pytest.skip("fewer candidates than the second window needs")
    o = hot_state()
    o.set_scalars(evS=_lcg_back(3, 7 * t + 2))
    nP = o.nP
    fs = to_device(o, with_grid=True)
    o.stage("update_evaporation", 1 / 12)
    fs.stage("EVAPORATION", 1 / 12)
    so, sg = o.scalars, fs.scalars
    assert so.evapCount == nC and sg.evapCount == nC
    assert sg.evS == so.evS
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-6, k


def test_phase_parity():
    o = _state64()
    nP = o.nP
    rng = np.random.default_rng(11)
    fl = rng.choice([0, 0, 0, 1, 2, 3, 4, 5], nP).astype(np.uint8)
    o.pflag[:nP] = fl
    o.pT[:nP] = rng.uniform(0.0, 0.6, nP).astype(np.float32)
    o.pAir[:nP] = rng.uniform(0.0, 1.0, nP).astype(np.float32)
    fs = to_device(o, with_grid=True)
    o.stage("update_phase", 1 / 60)
    fs.stage("PHASE", 1 / 60)
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    assert np.array_equal(fs.pAir, o.pAir[:nP])
    for k in ("pvx", "pvy", "pvz"):
        assert np.array_equal(fs.download(k), o.arr(k)[:nP]), k


def test_vapor_advection_exact_streams():
    """Vapour parcels consume the serial _cfS/_bfS streams: the device pass
    reproduces every draw (states bit-exact after the substep)."""
    o = _state64()
    nP = o.nP
    rng = np.random.default_rng(3)
    c = o.nx / 2
    R = o.scalars.oceanR
    sel = rng.choice(nP, 3000, replace=False)
    d = rng.normal(size=(3000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = R + rng.uniform(-0.1, 0.4, 3000)
    o.px[sel] = c + d[:, 0] * r; o.py[sel] = c + d[:, 1] * r; o.pz[sel] = c + d[:, 2] * r
    o.pvx[sel] = rng.normal(0, 0.5, 3000); o.pvy[sel] = rng.normal(0, 0.5, 3000); o.pvz[sel] = rng.normal(0, 0.5, 3000)
    o.pflag[sel] = rng.choice([2, 3], 3000)
    o.pT[sel] = rng.uniform(0.1, 0.5, 3000)
    o.pAir[sel] = rng.uniform(0, 1, 3000)
    fs = to_device(o)
    o.substep(0.01)
    fs._substep(0.01)
    so, sg = o.scalars, fs.scalars
    assert (sg.cfS, sg.bfS) == (so.cfS, so.bfS)
    assert so.cfS != 0x2f6e2b1 and so.bfS != 0x7f4a7c15   # the streams were consumed
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    W = o.nx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(fs.download(k)[sel].astype(np.float64) - o.arr(k)[sel])) <= 1e-5 * W, k


def _jacobi_vapor_contacts(o, rad):
    """The device's vapour contact pass (js/solver.js:3345-3478 resolved from
    one snapshot, Jacobi order) restated with a k-d tree: position and
    velocity increments of every parcel, in FP64."""
    from scipy.spatial import cKDTree
    nP = o.nP
    f = o.pflag[:nP]
    X = np.stack([o.arr(k)[:nP].astype(np.float64) for k in ("px", "py", "pz")], 1)
    V = np.stack([o.arr(k)[:nP].astype(np.float64) for k in ("pvx", "pvy", "pvz")], 1)
    par = np.nonzero((f == 2) | (f == 3))[0]
    dpos = np.zeros((nP, 3))
    dvel = np.zeros((nP, 3))
    tp = cKDTree(X[par])
    pairs = np.array(sorted(tp.query_pairs(rad * 1.001)), dtype=np.int64).reshape(-1, 2)
    a, b = par[pairs[:, 0]], par[pairs[:, 1]]
    d = X[b] - X[a]
    d2 = (d * d).sum(1)
    keep = d2 < rad * rad
    a, b, d, d2 = a[keep], b[keep], d[keep], d2[keep]
    dd = np.sqrt(d2)
    dd[dd == 0] = 1e-9
    n = d / dd[:, None]
    vrel = ((V[a] - V[b]) * n).sum(1)
    dv = np.maximum(vrel, 0) + (rad - dd) * 2
    half = (rad - dd) * 0.5
    np.add.at(dpos, a, -n * half[:, None]); np.add.at(dpos, b, n * half[:, None])
    np.add.at(dvel, a, -n * dv[:, None]); np.add.at(dvel, b, n * dv[:, None])
    c = np.array([o.nx / 2, o.ny / 2, o.nz / 2], np.float64) * o.dx
    band = o.scalars.oceanR - o.dx * 2
    r2 = ((X - c) ** 2).sum(1)
    liq = np.nonzero(((f == 0) & (r2 >= band * band)) | (f == 1) | (f == 4))[0]
    tw = cKDTree(X[liq])
    hits = tw.query_ball_tree(tp, rad * 1.001)
    w = np.repeat(liq, [len(h) for h in hits])
    bp = par[np.concatenate([np.asarray(h, np.int64) for h in hits])] if len(w) else np.zeros(0, np.int64)
    d = X[bp] - X[w]
    d2 = (d * d).sum(1)
    keep = (d2 < rad * rad) & (d2 >= 1e-12)
    w, bp, d, d2 = w[keep], bp[keep], d[keep], d2[keep]
    dd = np.sqrt(d2)
    n = d / dd[:, None]
    vr = ((V[bp] - V[w]) * n).sum(1)
    ov = rad - dd
    dvl = ov * 2 - np.where(vr < 0, vr * 1.4, 0)
    np.add.at(dpos, bp, n * ov[:, None])
    np.add.at(dvel, bp, n * dvl[:, None])
    return X, V, dpos, dvel, len(a), len(w)


def test_vapor_contacts_jacobi():
    """Vapour-vapour and liquid-vapour contacts of 6000 parcels placed in the
    surface shell (steam and cloud), against a k-d tree restatement of the
    device's snapshot order: the same contact set, increments summed in FP32
    atomics on the device."""
    o = _state64()
    nP = o.nP
    rng = np.random.default_rng(21)
    c = o.nx / 2
    R = o.scalars.oceanR
    m = 6000
    sel = rng.choice(nP, m, replace=False)
    d = rng.normal(size=(m, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = R + rng.uniform(-0.6, 0.3, m)
    o.px[sel] = c + d[:, 0] * r; o.py[sel] = c + d[:, 1] * r; o.pz[sel] = c + d[:, 2] * r
    o.pvx[sel] = rng.normal(0, 0.5, m); o.pvy[sel] = rng.normal(0, 0.5, m); o.pvz[sel] = rng.normal(0, 0.5, m)
    o.pflag[sel] = rng.choice([2, 3], m)
    fs = to_device(o)
    rad = o.scalars.spacing * 0.6
    X, V, dpos, dvel, nvv, nvl = _jacobi_vapor_contacts(o, rad)
    assert nvv > 20 and nvl > 200
    fs.stage("VAPOR_COLLISIONS")
    assert fs.scalars.vaporCount == int(np.count_nonzero(o.pflag[:nP] == 2))
    gX = np.stack([fs.download(k).astype(np.float64) for k in ("px", "py", "pz")], 1)
    gV = np.stack([fs.download(k).astype(np.float64) for k in ("pvx", "pvy", "pvz")], 1)
    tol_x = 1e-5 + 1e-5 * np.abs(dpos).max()
    tol_v = 1e-5 + 1e-5 * np.abs(dvel).max()
    assert np.abs(gX - (X + dpos)).max() <= tol_x
    assert np.abs(gV - (V + dvel)).max() <= tol_v


def test_push_surface_parity():
    o = _state64()
    nP = o.nP
    rng = np.random.default_rng(5)
    sel = rng.choice(nP, 5000, replace=False)
    c = o.nx / 2
    for a in ("px", "py", "pz"):
        o.arr(a)[sel] = c + (o.arr(a)[sel] - c) * rng.uniform(0.7, 1.2, 5000)
    fs = to_device(o, with_grid=True)
    o.stage("push_surface")
    fs.stage("PUSH_SURFACE")
    W = o.nx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(fs.download(k).astype(np.float64) - o.arr(k)[:nP])) <= 1e-6 * W, k
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-6, k


def test_splat_volume_census_ke():
    o = _state64()
    fs = to_device(o, with_grid=True)
    o.stage("splat_density")
    fs.stage("SPLAT")
    assert rel_err(fs.dens, o.dens) <= 1e-6
    for iso in (0.8, 1.6):
        vg, ng = fs.mt_volume(iso)
        vo, no = o.mt_volume(iso)
        assert abs(vg - vo) <= 1e-6 * vo and abs(ng - no) <= max(3, 1e-4 * no)
    nP = o.nP
    fl = np.random.default_rng(2).choice([0, 1, 2, 3, 4, 5], nP).astype(np.uint8)
    o.pflag[:nP] = fl
    fs.upload("pflag", fl)
    assert np.allclose(fs.census(), o.census(), rtol=0, atol=1e-15)
    assert abs(fs.kineticEnergy() - o.kinetic_energy()) <= 1e-9 * o.kinetic_energy()


def test_impulses_parity():
    o = _state64()
    fs = to_device(o)
    c = o.nx / 2
    R = o.scalars.oceanR
    o.apply_impulse_sphere(c + R, c, c, 4.0, 0.5, -0.2, 0.1)
    fs.applyImpulseSphere(c + R, c, c, 4.0, 0.5, -0.2, 0.1)
    o.stir_at(c, c + R, c, 0.3, 0.0, -0.4, 5.0, 0.01)
    fs.stirAt(c, c + R, c, 0.3, 0.0, -0.4, 5.0, 0.01)
    o.stir_gaussian(4.0, 2.0)
    fs.stir_gaussian(4.0, 2.0)
    nP = o.nP
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-7, k
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    assert fs.scalars.stirS == o.scalars.stirS


def test_thermal_substep_parity_with_vorticity():
    o = planet("planet64", **THERMAL64)
    o.set(sunPos=_sun(o))
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    o.substep(0.01)
    fs._substep(0.01)
    nP = o.nP
    assert np.array_equal(fs.cellType, o.cellType)
    assert np.array_equal(fs.pflag, o.pflag[:nP])
    assert fs.scalars.sorIters == o.scalars.sorIters
    assert rel_err(fs.q, o.q) <= 1e-5
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-5, k


def test_frames_with_thermal_cycle():
    """Whole frames (thermal tick, evaporation, substeps, contacts, phases,
    rescue): counts and energy track the oracle. Vapour contacts are resolved
    in Jacobi order on the device, so this compares run-level observables."""
    o = planet("planet64", **THERMAL64)
    o.set(sunPos=_sun(o, 2.0), sunActivity=1.2, evapIntensity=0.5)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    for _ in range(6):
        o.step(1 / 60)
        fs.step(1 / 60)
    so, sg = o.scalars, fs.scalars
    assert sg.substepsLast == so.substepsLast
    assert abs(sg.evapCount - so.evapCount) <= max(2, 0.05 * so.evapCount)
    assert abs(sg.vaporCount - so.vaporCount) <= max(3, 0.05 * so.vaporCount)
    ko, kg = o.kinetic_energy(), fs.kineticEnergy()
    assert abs(kg - ko) <= 0.02 * ko


def test_currents_parity():
    """Subsurface currents (js/solver.js:3624-3782): the curl-noise lattice and
    the relaxation of deep fluid particles. The lattice uses cos; the device's
    and the host libm's may differ by an ulp, so velocities agree to 1e-6."""
    o = _state64()
    o.set(currents=0.6)
    o.set_scalars(simTime=3.7)
    fs = to_device(o)
    nP = o.nP
    before = o.arr("pvx")[:nP].copy()
    o.stage("update_currents", 1 / 12)
    fs.stage("CURRENTS", 1 / 12)
    assert np.abs(o.arr("pvx")[:nP] - before).max() > 1e-3          # the pass acts
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(fs.download(k), o.arr(k)[:nP]) <= 1e-6, k


def test_ice_contacts_parity():
    """_iceContacts (js/solver.js:3290-3324) on 4000 snow grains dropped in
    clumps at the sea surface, a third of them already stuck to the pack:
    the device's segmented serial sweep reproduces the reference's in-place
    sweep over the x-sorted list, so stuck flags and velocities are bit-exact."""
    o = _state64()
    nP = o.nP
    rng = np.random.default_rng(31)
    c = o.nx / 2
    R = o.scalars.oceanR
    m, clumps = 4000, 120
    sel = rng.choice(nP, m, replace=False)
    centres = rng.normal(size=(clumps, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    centres = c + centres * (R + 0.5)
    which = rng.integers(0, clumps, m)
    pos = centres[which] + rng.normal(0, 0.6 * o.scalars.spacing, (m, 3))
    for a, k in enumerate(("px", "py", "pz")):
        o.arr(k)[sel] = pos[:, a]
    for k in ("pvx", "pvy", "pvz"):
        o.arr(k)[sel] = rng.normal(0, 0.4, m)
    o.pflag[sel] = 5
    o.pAir[sel] = np.where(rng.random(m) < 0.33, 1.0, rng.uniform(0, 0.9, m)).astype(np.float32)
    fs = to_device(o)
    before_air = o.pAir[:nP].copy()
    before_v = o.arr("pvx")[:nP].copy()
    o.stage("ice_contacts")
    fs.stage("ICE_CONTACTS")
    newly_stuck = np.count_nonzero((o.pAir[:nP] == 1) & (before_air != 1))
    paired = np.count_nonzero((o.arr("pvx")[:nP] != before_v) & (o.pAir[:nP] != 1))
    assert newly_stuck > 50 and paired > 50            # both rules fire
    assert np.array_equal(fs.pAir, o.pAir[:nP])
    for k in ("pvx", "pvy", "pvz"):
        assert np.array_equal(fs.download(k), o.arr(k)[:nP]), k

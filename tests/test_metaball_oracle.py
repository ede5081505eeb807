"""The metaball oracle (or_metaball_field + the marching-tets mesher) against
the reference's own known answers for Metaballs.build (test/metaball.test.js:
26-160): a 7^3 particle block on a 16^3 stub solver (spacing dx/4) meshes into
whole triangles with unit outward normals, volume grows with tension, the iso
mapping clamps, the detail factor falls back and clamps, coarse and fine
lattices keep the volume within 15%, only liquid particles count, and stray
particles stay safe."""
import math

import numpy as np

from oracle.oracle import metaball_field, mt_mesh_field

N, DX = 16, 1.0 / 16
SP = DX * 0.25


def block(side):
    c = 0.5 - (side // 2) * SP
    g = np.arange(side) * SP + c
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    return [a.ravel().astype(np.float32) for a in (x, y, z)]


def build(px, py, pz, fl=None, tension=0.5, detail=None):
    fl = np.zeros(len(px), np.uint8) if fl is None else np.asarray(fl, np.uint8)
    field, m, mdx, iso, _ = metaball_field(px, py, pz, fl, N, DX, SP, tension, detail)
    vol, pos, nrm = mt_mesh_field(field, m, m, m, mdx, iso)
    return abs(vol), pos, nrm


def iso(t):
    return metaball_field(np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32),
                          np.zeros(0, np.uint8), N, DX, SP, t)[3]


P7 = block(7)
P11 = block(11)


def test_mesh_is_closed_with_outward_unit_normals():
    vol, pos, nrm = build(*P7, tension=0)
    assert len(pos) > 0 and len(pos) % 3 == 0 and vol > 0
    assert np.all(np.isfinite(pos)) and np.all(np.isfinite(nrm))
    assert np.all(np.abs(np.linalg.norm(nrm.astype(np.float64), axis=1) - 1) < 1e-5)
    assert np.all(np.sum((pos - 0.5) * nrm, axis=1) > -0.5)
    vol2, pos2, _ = build(*P7, tension=0)
    assert vol2 == vol and np.array_equal(pos2, pos)


def test_volume_grows_with_tension_and_iso_clamps():
    for detail in (None, 1.4):
        prev = -1
        for t in (0, 0.25, 0.5, 0.75, 1):
            vol = build(*P7, tension=t, detail=detail)[0]
            assert vol > 0 and vol > prev
            prev = vol
    assert iso(0) < iso(0.5) < iso(1)
    assert iso(1) == iso(2) and iso(0) == iso(-1)


def test_detail_fallback_and_clamps():
    v1, p1, _ = build(*P7)
    for d in (1, float("nan"), 0, -2):
        v, p, _ = build(*P7, detail=d)
        assert v == v1 and len(p) == len(p1)
    assert build(*P7, detail=999)[0] == build(*P7, detail=1.6)[0]
    assert build(*P7, detail=0.01)[0] == build(*P7, detail=0.5)[0]


def test_coarse_and_fine_lattices_keep_the_volume():
    vb, pb, _ = build(*P11, tension=1, detail=1)
    vc, pc, _ = build(*P11, tension=1, detail=0.6)
    vf, pf, nf = build(*P11, tension=1, detail=1.4)
    assert 0 < len(pc) < len(pb) and abs(vc - vb) / vb < 0.15
    assert len(pf) > len(pb) and abs(vf - vb) / vb < 0.15 and len(pf) % 3 == 0
    assert np.all(np.isfinite(pf)) and np.all(np.isfinite(nf))


def test_only_liquid_counts_and_strays_are_safe():
    n = len(P7[0])
    assert len(build(*P7, fl=np.full(n, 2))[1]) == 0
    half = np.where(np.arange(n) % 2 == 1, 2, 0)
    vh, ph, _ = build(*P7, fl=half, tension=0)
    assert len(ph) > 0 and vh < build(*P7, tension=0)[0]
    e = np.zeros(0, np.float32)
    assert len(build(e, e, e)[1]) == 0
    sx = np.array([5 * DX, -3 * DX, N * DX * 2, math.nan], np.float32)
    sy = np.full(4, 5 * DX, np.float32)
    _, ps, _ = build(sx, sy, sy)
    assert np.all(np.isfinite(ps))

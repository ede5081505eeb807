"""ws_surface_mesh against the oracle's MarchingTetrahedra.build
(js/surface.js:66-177) on the same density field: the same vertex count,
bit-identical float positions and normals in the same (cell, tet, case)
order, and the same FP64 volume (block-summed on the device: 1e-12)."""
import numpy as np
import pytest

from helpers import planet, to_device, PLAIN32
from oracle.oracle import mt_mesh_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["planet32", "planet64"])
def test_surface_mesh_matches_oracle(name):
    o = planet(name, **PLAIN32)
    fs = to_device(o)
    fs._substep(0.01)
    fs.stage("SPLAT")
    dens = fs.download("dens")
    iso = 1.0
    vol, pos, nrm = fs.surface_mesh(iso)
    vref, pref, nref = mt_mesh_field(dens, o.nx, o.ny, o.nz, o.dx, iso)
    assert len(pos) == len(pref) > 1000
    assert np.array_equal(pos, pref)
    assert np.array_equal(nrm, nref)
    assert abs(vol - vref) <= 1e-12 * vref
    # a second build at another iso reuses the buffer
    vol2, pos2, _ = fs.surface_mesh(1.4)
    vref2, pref2, _ = mt_mesh_field(dens, o.nx, o.ny, o.nz, o.dx, 1.4)
    assert np.array_equal(pos2, pref2) and abs(vol2 - vref2) <= 1e-12 * vref2
    # no straddling cell (iso above every corner, or below every corner): an empty mesh
    for iso3 in (float(dens.max()) + 1.0, float(dens.min()) - 1.0):
        vol3, pos3, nrm3 = fs.surface_mesh(iso3)
        vref3, pref3, _ = mt_mesh_field(dens, o.nx, o.ny, o.nz, o.dx, iso3)
        assert len(pos3) == len(pref3) == 0 and len(nrm3) == 0
        assert vol3 == 0.0 and vref3 == 0.0

"""The grid-wide SOR solve (k_sor_persistent: every SM, lists in global
memory, software grid barrier), which takes over when the interior fluid
cells of a colour exceed what one 16-CTA cluster holds (16 x 4095). A 128^3
planet with a 24-cell ocean (240k fluid cells) has almost twice that. After one substep from the
same state the device matches the oracle (device order) at the substep bar:
cell types bit-exact, q and face velocities within 1e-5 relative; a second
solve of the same system (ws_time_kernel) keeps q finite."""
import numpy as np
import pytest

from helpers import to_device, rel_err, DEVICE_ORDER, PLAIN32
from oracle.oracle import make_planet

pytestmark = pytest.mark.gpu


def test_grid_wide_solve_matches_oracle():
    o = make_planet(128, R=56.0, depth=24.0, particles=1200000)
    o.set(**DEVICE_ORDER)
    o.set(**PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    o.substep(0.01)
    fs._substep(0.01)
    s = fs.scalars
    assert s.sorPath == 1, "expected the grid-wide solve"
    assert s.nFluid == o.scalars.nFluid and s.nFluid > 2 * 16 * 4095
    assert np.array_equal(fs.cellType, o.cellType)
    assert rel_err(fs.q, o.q) <= 1e-5
    for k in ("u", "v", "w"):
        assert rel_err(fs.download(k), o.arr(k)) <= 1e-5, k
    fs.time_kernel(6, 2)
    assert np.all(np.isfinite(fs.q))

"""Device-side failure detection, made without faulting the GPU.

* A NaN planted on the host in one fluid particle's velocity: P2G leaves the
  particle out of the grid and latches the NaN bit; the next synchronising
  call returns WS_ERR_DEVICE. The handle stays usable: after a clean upload
  the next substep succeeds.
* A particle uploaded outside the domain box latches the range bit the same
  way when the next substep reads the positions (the reference's own passes
  keep every particle inside it).
* A bounded device wait that runs out (ws_probe_wait: a status word nothing
  sets, the same bounded wait the pressure solve's CTAs use between them)
  returns WS_ERR_TIMEOUT; the context stays usable.
"""
import numpy as np
import pytest

from helpers import planet, to_device, PLAIN32
from fluid_solver import WsError

pytestmark = pytest.mark.gpu

WS_ERR_DEVICE, WS_ERR_TIMEOUT = -5, -6


def _fluid_index(o):
    return int(np.nonzero(o.arr("pflag")[:o.nP] == 0)[0][100])


def test_nan_velocity_latched_and_recoverable():
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    clean = fs.snapshot()
    p = _fluid_index(o)
    bad = fs.download("pvx")
    bad[p] = np.nan
    fs.upload("pvx", bad)
    with pytest.raises(WsError) as ei:
        fs._substep(0.01)
        fs.synchronize()
    assert ei.value.code == WS_ERR_DEVICE
    assert "NaN" in str(ei.value)
    # usable afterwards: the clean state restored, the next substep succeeds
    fs.restore(clean)
    fs._substep(0.01)
    fs.synchronize()
    for k in ("px", "pvx"):
        assert np.all(np.isfinite(fs.download(k))), k
    fs.close()


def test_out_of_box_fluid_particle_latched():
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    p = _fluid_index(o)
    x = fs.download("px")
    x[p] = -3.0
    fs.upload("px", x)
    with pytest.raises(WsError) as ei:
        fs._substep(0.01)
        fs.synchronize()
    assert ei.value.code == WS_ERR_DEVICE
    assert "range" in str(ei.value)
    fs.close()


def test_bounded_wait_runs_out():
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    with pytest.raises(WsError) as ei:
        fs.probe_wait(200000)            # ~0.1-0.3 s of polls on a word nothing sets
    assert ei.value.code == WS_ERR_TIMEOUT
    fs._substep(0.01)                    # the context and the handle still work
    fs.synchronize()
    assert fs.scalars.sorIters > 0
    fs.close()

"""ws_upload_state / ws_download_state: the batched particle transfer that
GpuSim's frame readback needs (js/gpu/gpusim.js:568-650), checked against
the per-field transfer it replaces, then a substep fed through it against
the oracle."""
import numpy as np
import pytest

from helpers import planet, to_device, rel_err, PFIELDS, PLAIN32

pytestmark = pytest.mark.gpu


def test_state_round_trip_planet32():
    o = planet("planet32", **PLAIN32)
    fs = to_device(o)
    nP = o.nP
    rng = np.random.default_rng(7)
    host = {}
    for k in PFIELDS:
        dt = np.uint8 if k in ("pflag", "pcool", "pDepth") else np.float32
        host[k] = np.empty(nP, dt)
    fs.download_state(host, nP)
    for k in PFIELDS:
        assert np.array_equal(host[k], fs.download(k)), k
    # new values in, read back field by field
    new = {k: (rng.integers(0, 2, nP).astype(np.uint8) if v.dtype == np.uint8
               else rng.standard_normal(nP).astype(np.float32)) for k, v in host.items()}
    fs.upload_state(new, nP)
    for k in PFIELDS:
        assert np.array_equal(fs.download(k), new[k]), k
    # a subset moves only the named fields
    fs.upload_state({"px": host["px"]}, nP)
    assert np.array_equal(fs.download("px"), host["px"])
    assert np.array_equal(fs.download("py"), new["py"])
    cap = fs.scalars.capacity
    with pytest.raises(RuntimeError):
        fs.upload_state({"px": np.zeros(cap + 1, np.float32)}, cap + 1)
    with pytest.raises(ValueError):
        fs.download_state({"px": np.zeros(nP, np.float64)}, nP)


def test_substep_through_state_io_planet32():
    o = planet("planet32", **PLAIN32)
    fs = to_device(o)
    nP = o.nP
    fields = ("px", "py", "pz", "pvx", "pvy", "pvz", "pflag")
    host = {k: o.arr(k)[:nP].astype(np.uint8 if k == "pflag" else np.float32) for k in fields}
    fs.upload_state(host, nP)
    o.substep(0.01)
    fs._substep(0.01)
    fs.download_state(host, nP)
    assert np.array_equal(host["pflag"], o.arr("pflag")[:nP])
    W = o.nx * o.dx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(host[k].astype(np.float64) - o.arr(k)[:nP])) <= 1e-5 * W, k
    for k in ("pvx", "pvy", "pvz"):
        assert rel_err(host[k], o.arr(k)[:nP]) <= 1e-5, k

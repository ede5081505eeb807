"""ws_upload_state / ws_download_state with the substep-free fields (light,
depth, phase, and the temperature while no vapour exists) copied on a second
stream beside the substep: what comes back must be exactly what a field-by-
field download gives, and the free fields must be the uploaded values."""
import numpy as np
import pytest

from helpers import planet, to_device, PLAIN32

pytestmark = pytest.mark.gpu

FIELDS = {"px": np.float32, "py": np.float32, "pz": np.float32, "pvx": np.float32, "pvy": np.float32,
          "pvz": np.float32, "pT": np.float32, "pflag": np.uint8, "pLight": np.float32, "pDepth": np.uint8}


def _arrays(n):
    return {k: np.empty(n, dt) for k, dt in FIELDS.items()}


def test_free_fields_beside_substeps():
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    n = fs.scalars.nP
    host = _arrays(n)
    fs.download_state(host, n)
    rng = np.random.default_rng(3)
    host["pLight"][:] = rng.random(n, dtype=np.float32)
    host["pDepth"][:] = rng.integers(0, 255, n, dtype=np.uint8)
    host["pT"][:] = 280 + 10 * rng.random(n, dtype=np.float32)
    sent = {k: v.copy() for k, v in host.items()}
    for step in range(3):
        fs.upload_state(host, n)
        fs._substep(0.01)
        fs._substep(0.01)
        fs.download_state(host, n)
        for k in ("pLight", "pDepth", "pT"):
            assert np.array_equal(host[k], sent[k]), (step, k)
    # the substep's own fields against field-by-field downloads (a synchronising path)
    for k in ("px", "py", "pz", "pvx", "pvy", "pvz", "pflag", "pLight", "pDepth", "pT"):
        assert np.array_equal(host[k], fs.download(k)), k


def test_other_calls_see_the_uploaded_fields():
    """A call other than the substep right after an upload orders itself after
    the side copies: a field download returns the uploaded values."""
    o = planet("planet32", **PLAIN32)
    fs = to_device(o)
    n = fs.scalars.nP
    host = _arrays(n)
    fs.download_state(host, n)
    host["pLight"][:] = np.linspace(0, 1, n, dtype=np.float32)
    host["pDepth"][:] = np.arange(n, dtype=np.int64).astype(np.uint8)
    fs.upload_state(host, n)
    assert np.array_equal(fs.download("pLight"), host["pLight"])
    assert np.array_equal(fs.download("pDepth"), host["pDepth"])
    # and after a substep that was enqueued meanwhile
    fs.upload_state(host, n)
    fs._substep(0.01)
    assert np.array_equal(fs.download("pLight"), host["pLight"])

"""ws_step_async / ws_step_poll / ws_step_wait: GpuSim.step's non-blocking
contract (js/gpu/gpusim.js:328-339). A frame started asynchronously ends in
the same state as the same frame stepped synchronously on a twin handle (the
bar of the snapshot test: flags and cell types equal, positions within 1e-5 of
the box); a second start while the frame runs starts nothing (WS_BUSY), every
other call meanwhile returns WS_ERR_BUSY; a frame's error comes back through
poll/wait; destroying a handle waits for its frame."""
import time

import numpy as np
import pytest

from fluid_solver import FluidSolver, WsError
from helpers import planet, to_device

pytestmark = pytest.mark.gpu

WS_ERR_BUSY, WS_ERR_STATE = -8, -4


def test_async_frame_matches_sync_and_is_exclusive():
    o = planet("planet32")                               # thermal cycle on: every frame pass runs
    a, b = to_device(o), to_device(o)
    dt = 1 / 30
    a.step(dt)
    assert b.step_async(dt) is True
    assert b.step_async(dt) is False                     # busy: nothing started
    with pytest.raises(WsError) as e:
        b.download("px", 16)
    assert e.value.code == WS_ERR_BUSY
    polls = 0
    while not b.step_poll():
        polls += 1
        time.sleep(0.0005)
    assert polls > 0
    nP = a.scalars.nP
    assert b.scalars.nP == nP
    assert np.array_equal(a.download("pflag", nP), b.download("pflag", nP))
    assert np.array_equal(a.download("cellType"), b.download("cellType"))
    W = o.nx * o.dx
    for k in ("px", "py", "pz"):
        assert np.max(np.abs(a.download(k, nP).astype(np.float64) - b.download(k, nP))) <= 1e-5 * W, k
    # start / wait / start again; the synchronous API works between frames
    for _ in range(3):
        a.step(dt)
        assert b.step_async(dt)
        b.step_wait()
    assert a.scalars.substepsLast == b.scalars.substepsLast


def test_async_error_and_destroy():
    fs = FluidSolver(nx=24, ny=24, nz=24, dx=1.0, coreR=8.0, targetParticles=1000, capacity=4096)
    assert fs.step_async(1 / 60)                          # no terrain: the frame fails on the worker
    with pytest.raises(WsError) as e:
        fs.step_wait()
    assert e.value.code == WS_ERR_STATE
    o = planet("planet32")
    b = to_device(o)
    assert b.step_async(1 / 30)
    b.close()                                             # waits for the frame, then frees

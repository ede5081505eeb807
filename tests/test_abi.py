"""The C-ABI library loads without a GPU and exports every entry point that
include/watersim.h declares (no compute calls are made here)."""
import os
import re

import fluid_solver
from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "watersim.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:ws_status|const char\*)\s+(ws_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_header():
    L = fluid_solver.load_library()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(fluid_solver.SYMBOLS)


def test_version_and_defaults_without_gpu():
    L = fluid_solver.load_library()
    assert b"sm_100a" in L.ws_version()
    p = fluid_solver.WsParams()
    assert L.ws_default_params(p) == 0
    assert p.pic == 0.15 and p.omega == 1.55 and p.pressureIters == 20 and p.maxSpeed == 3.2
    assert p.sorRedBlack == 1 and p.viscJacobi == 1 and p.extrapJacobi == 1


def test_struct_layouts_match_oracle():
    from oracle.oracle import OrParams, OrScalars
    assert [f[0] for f in fluid_solver.WsParams._fields_] == [f[0] for f in OrParams._fields_]
    assert [f[0] for f in fluid_solver.WsScalars._fields_] == [f[0] for f in OrScalars._fields_]
    import ctypes
    assert ctypes.sizeof(fluid_solver.WsParams) == ctypes.sizeof(OrParams)
    assert ctypes.sizeof(fluid_solver.WsScalars) == ctypes.sizeof(OrScalars)


def test_create_fails_cleanly_without_device(monkeypatch):
    import torch
    if torch.cuda.is_available():
        return
    try:
        fluid_solver.FluidSolver(nx=8, ny=8, nz=8, dx=1.0)
    except fluid_solver.WsError as e:
        assert e.code < 0
    else:
        raise AssertionError("ws_create must fail without a device")

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


def _zero_args(fn):
    import ctypes as C
    args = []
    for t in fn.argtypes or []:
        if t in (C.c_double, C.c_float):
            args.append(0.0)
        elif t in (C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_int, C.c_uint8):
            args.append(0)
        else:
            args.append(None)
    return args


def test_null_handle_rejected_everywhere():
    """Every entry point that takes a handle (or an output pointer) answers a
    NULL one with WS_ERR_INVALID before any device call; ws_last_error names it."""
    L = fluid_solver.load_library()
    for name in fluid_solver.SYMBOLS:
        if name in ("ws_version", "ws_last_error"):
            continue
        fn = getattr(L, name)
        assert fn(*_zero_args(fn)) == -1, name
    assert L.ws_last_error(None) == b"null handle"


def test_create_and_noalloc_validate_sizes_before_any_device_call():
    import ctypes as C
    L = fluid_solver.load_library()
    h = C.c_void_p()

    def create(nx, ny, nz, dx=1.0, cap=16):
        cfg = fluid_solver.WsConfig(nx=nx, ny=ny, nz=nz, capacity=cap, dx=dx, coreR=1.0, bumpiness=0.3,
                                    targetParticles=16.0, terrainSeed=1, device=0)
        return L.ws_create(C.byref(cfg), C.byref(h))

    assert create(3, 8, 8) == -1                     # below the 4-cell minimum
    assert create(8, 8, 8, dx=0.0) == -1
    assert create(8, 8, 8, cap=0) == -1
    assert create(1024, 1024, 1024) == -7            # beyond 2^29 cells
    buf = (C.c_float * 4)()
    rel = C.c_double()
    p = C.cast(buf, C.c_void_p)
    assert L.ws_residual_noalloc(2, 8, 8, p, p, p, C.byref(rel), None) == -1
    assert L.ws_residual_noalloc(8, 8, 8, None, p, p, C.byref(rel), None) == -1
    assert L.ws_residual_noalloc(512, 512, 512, p, p, p, C.byref(rel), None) == -7

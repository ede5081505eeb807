"""ws_residual_noalloc — the allocation-free FP64 residual entry point.

Some callers own every device buffer and cannot let a library allocate (a
host with its own device allocator, a frame loop where cudaMalloc would
synchronise the device). This entry point takes their buffers and uses a
fixed device array as scratch. The test calls it through the C ABI on
buffers torch owns and checks it against the handle-based ws_residual on
two calls in a row (the shared scratch keeps the first call's contents), at
the FP64 reduction tolerance of the other tests. Collected last so a failure
here never hides another test's result.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

WS_ERR_RANGE = -7


def test_noalloc_residual_matches_handle():
    import torch
    import fluid_solver
    from helpers import planet, to_device, PLAIN32
    o = planet("planet32", **PLAIN32)
    o.set_scalars(gRamp=1.5)
    fs = to_device(o)
    fs._substep(0.01)                          # q, rhs and cell types of a solved substep
    ref = fs.residual()                        # the existing entry point (ws_residual)
    assert ref > 0
    q = torch.from_numpy(fs.q).cuda()
    rhs = torch.from_numpy(fs.rhs).cuda()
    ct = torch.from_numpy(fs.cellType).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = fluid_solver.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(-1.0)
        rc = L.ws_residual_noalloc(o.nx, o.ny, o.nz, q.data_ptr(), rhs.data_ptr(), ct.data_ptr(),
                                   out.data_ptr(), C.c_void_p(stream))
        torch.cuda.synchronize()
        assert rc == 0
        assert abs(out.item() - ref) <= 1e-9 * ref, (out.item(), ref)
    # a grid beyond the fixed scratch is rejected before anything runs
    rc = L.ws_residual_noalloc(256, 256, 256, q.data_ptr(), rhs.data_ptr(), ct.data_ptr(),
                               out.data_ptr(), C.c_void_p(stream))
    assert rc == WS_ERR_RANGE
    fs.close()


def test_noalloc_leaves_pending_error_alone():
    """An earlier, unrelated CUDA error pending on the calling thread (here a
    harmless cudaSetDevice(-1), which faults nothing) is neither reported as
    this call's nor cleared: the call succeeds and the error is still there
    for its owner to read."""
    import torch
    import fluid_solver
    cudart = C.CDLL("libcudart.so.12")
    q = torch.zeros(32 ** 3, dtype=torch.float32, device="cuda")
    rhs = torch.ones(32 ** 3, dtype=torch.float32, device="cuda")
    ct = torch.zeros(32 ** 3, dtype=torch.uint8, device="cuda")
    ct.view(32, 32, 32)[8:24, 8:24, 8:24] = 1              # a fluid block: the residual of q = 0 is 1
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = fluid_solver.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    assert cudart.cudaSetDevice(-1) != 0                   # leaves a pending, non-sticky error
    pending = cudart.cudaPeekAtLastError()
    assert pending != 0
    rc = L.ws_residual_noalloc(32, 32, 32, q.data_ptr(), rhs.data_ptr(), ct.data_ptr(), out.data_ptr(),
                               C.c_void_p(stream))
    assert rc == 0
    assert cudart.cudaPeekAtLastError() == pending         # still the caller's to read
    assert cudart.cudaGetLastError() == pending            # which clears it
    torch.cuda.synchronize()
    assert abs(out.item() - 1.0) <= 1e-12

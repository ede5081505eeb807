"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of liboracle_unet.so, the CPU
restatement of the warm-start U-Net (oracle/ws_unet_oracle.c). Only tests/
use it, as the checker of the network's output and gradients on the GPU."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_L = None


def lib():
    global _L
    if _L is None:
        path = os.path.join(_HERE, "liboracle_unet.so")
        if not os.path.exists(path):
            raise OSError("liboracle_unet.so not built; run make -C oracle")
        L = C.CDLL(path)
        vp, i32 = C.c_void_p, C.c_int32
        L.un_num_params.restype = C.c_int64
        L.un_num_params.argtypes = []
        L.un_forward.restype = None
        L.un_forward.argtypes = [i32, i32, i32, vp, vp, vp, i32, vp]
        L.un_loss_grad.restype = C.c_double
        L.un_loss_grad.argtypes = [i32, i32, i32, vp, vp, vp, vp, i32, vp]
        _L = L
    return _L


def num_params():
    return int(lib().un_num_params())


def forward(dims, params, r0n, types, rounding=True):
    nx, ny, nz = dims
    params = np.ascontiguousarray(params, np.float32)
    r0n = np.ascontiguousarray(r0n, np.float32)
    types = np.ascontiguousarray(types, np.uint8)
    out = np.zeros(nx * ny * nz, np.float32)
    lib().un_forward(nx, ny, nz, params.ctypes.data, r0n.ctypes.data, types.ctypes.data, 1 if rounding else 0,
                     out.ctypes.data)
    return out


def loss_grad(dims, params, r0n, types, target, rounding=True):
    """(loss, grads) of one sample; target already divided by the gain."""
    nx, ny, nz = dims
    params = np.ascontiguousarray(params, np.float32)
    r0n = np.ascontiguousarray(r0n, np.float32)
    types = np.ascontiguousarray(types, np.uint8)
    target = np.ascontiguousarray(target, np.float32)
    g = np.zeros(num_params(), np.float64)
    loss = lib().un_loss_grad(nx, ny, nz, params.ctypes.data, r0n.ctypes.data, types.ctypes.data,
                              target.ctypes.data, 1 if rounding else 0, g.ctypes.data)
    return loss, g


# layer table of the network: name, level, upsampled input channels, skip/plain input channels, outputs
LAYERS = [("e0a", 0, 0, 16, 16), ("e0b", 0, 0, 16, 16), ("e1a", 1, 0, 16, 32), ("e1b", 1, 0, 32, 32),
          ("ba", 2, 0, 32, 64), ("bb", 2, 0, 64, 64), ("d1a", 1, 64, 32, 32), ("d1b", 1, 0, 32, 32),
          ("d0a", 0, 32, 16, 16), ("d0b", 0, 0, 16, 16)]


def slices():
    """name -> (weight slice, bias slice) in the flat parameter vector, plus 'head'."""
    out, n = {}, 0
    for name, _lv, c0, c1, cout in LAYERS:
        nw = 27 * (c0 + c1) * cout
        out[name] = (slice(n, n + nw), slice(n + nw, n + nw + cout))
        n += nw + cout
    out["head"] = (slice(n, n + 16), slice(n + 16, n + 17))
    return out

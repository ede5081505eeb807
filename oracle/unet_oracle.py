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
        L.un_num_params_levels.restype = C.c_int64
        L.un_num_params_levels.argtypes = [i32]
        L.un_forward_levels.restype = None
        L.un_forward_levels.argtypes = [i32, i32, i32, i32, vp, vp, vp, i32, vp]
        L.un_loss_grad_levels.restype = C.c_double
        L.un_loss_grad_levels.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, i32, vp]
        _L = L
    return _L


def num_params(levels=3):
    return int(lib().un_num_params_levels(levels))


def forward(dims, params, r0n, types, rounding=True, levels=3):
    nx, ny, nz = dims
    params = np.ascontiguousarray(params, np.float32)
    r0n = np.ascontiguousarray(r0n, np.float32)
    types = np.ascontiguousarray(types, np.uint8)
    out = np.zeros(nx * ny * nz, np.float32)
    lib().un_forward_levels(nx, ny, nz, levels, params.ctypes.data, r0n.ctypes.data, types.ctypes.data,
                            1 if rounding else 0, out.ctypes.data)
    return out


def loss_grad(dims, params, r0n, types, target, rounding=True, levels=3):
    """(loss, grads) of one sample; target already divided by the gain."""
    nx, ny, nz = dims
    params = np.ascontiguousarray(params, np.float32)
    r0n = np.ascontiguousarray(r0n, np.float32)
    types = np.ascontiguousarray(types, np.uint8)
    target = np.ascontiguousarray(target, np.float32)
    g = np.zeros(num_params(levels), np.float64)
    loss = lib().un_loss_grad_levels(nx, ny, nz, levels, params.ctypes.data, r0n.ctypes.data, types.ctypes.data,
                                     target.ctypes.data, 1 if rounding else 0, g.ctypes.data)
    return loss, g


def layers(levels=3):
    """Layer table (forward order): name, level, upsampled input channels,
    skip/plain input channels, outputs."""
    out = []
    for l in range(levels - 1):
        c = 16 << l
        out += [("e%da" % l, l, 0, 16 if l == 0 else c // 2, c), ("e%db" % l, l, 0, c, c)]
    cb = 16 << (levels - 1)
    out += [("ba", levels - 1, 0, cb // 2, cb), ("bb", levels - 1, 0, cb, cb)]
    for l in range(levels - 2, -1, -1):
        c = 16 << l
        out += [("d%da" % l, l, 2 * c, c, c), ("d%db" % l, l, 0, c, c)]
    return out


LAYERS = layers(3)


def slices(levels=3):
    """name -> (weight slice, bias slice) in the flat parameter vector, plus 'head'."""
    out, n = {}, 0
    for name, _lv, c0, c1, cout in layers(levels):
        nw = 27 * (c0 + c1) * cout
        out[name] = (slice(n, n + nw), slice(n + nw, n + nw + cout))
        n += nw + cout
    out["head"] = (slice(n, n + 16), slice(n + 16, n + 17))
    return out

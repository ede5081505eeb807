"""The CPU restatement of the warm-start network (oracle/ws_unet_oracle.c)
pinned by finite differences: its analytic loss gradient (FP64, no BF16
rounding) must match central differences of its own loss, within the 2%
that ReLU kinks crossed by the step leave. The GPU kernels
are then checked against this oracle (tests/test_gpu_unet.py)."""
import numpy as np
import pytest

from oracle import unet_oracle as U


def _case(n=16, seed=3):
    rng = np.random.default_rng(seed)
    N = n ** 3
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((x - n / 2 + 0.5) ** 2 + (y - n / 2 + 0.5) ** 2 + (z - n / 2 + 0.5) ** 2).ravel()
    types = np.zeros(N, np.uint8)                  # air
    types[r < n * 0.28] = 2                        # solid core
    types[(r >= n * 0.28) & (r < n * 0.40)] = 1    # fluid shell
    r0n = np.where(types == 1, rng.standard_normal(N), 0).astype(np.float32)
    target = np.where(types == 1, rng.standard_normal(N), 0).astype(np.float32)
    params = np.zeros(U.num_params(), np.float32)
    sl = U.slices()
    for name, _lv, c0, c1, cout in U.LAYERS:
        w, b = sl[name]
        params[w] = rng.standard_normal(w.stop - w.start) * np.sqrt(2.0 / (27 * (c0 + c1)))
        params[b] = 0.05 * rng.standard_normal(cout)
    params[sl["head"][0]] = 0.25 * rng.standard_normal(16)
    return (n, n, n), params, r0n, types, target


def test_output_zero_outside_active_tiles():
    dims, params, r0n, types, target = _case()
    out = U.forward(dims, params, r0n, types, rounding=False)
    n = dims[0]
    t = types.reshape(n, n, n)
    act = np.zeros_like(t, bool)
    for tz in range(0, n, 8):
        for ty in range(0, n, 16):
            for tx in range(0, n, 8):
                blk = (slice(tz, tz + 8), slice(ty, ty + 16), slice(tx, tx + 8))
                act[blk] = (t[blk] == 1).any()
    assert np.all(out.reshape(n, n, n)[~act] == 0)
    assert np.abs(out.reshape(n, n, n)[act]).max() > 0


def test_bf16_rounding_is_small():
    dims, params, r0n, types, target = _case()
    a = U.forward(dims, params, r0n, types, rounding=False)
    b = U.forward(dims, params, r0n, types, rounding=True)
    fl = types == 1
    rel = np.linalg.norm(a[fl] - b[fl]) / np.linalg.norm(a[fl])
    assert 0 < rel < 3e-2


@pytest.mark.parametrize("seed", [3, 11])
def test_gradient_matches_finite_differences(seed):
    dims, params, r0n, types, target = _case(seed=seed)
    loss, g = U.loss_grad(dims, params, r0n, types, target, rounding=False)
    assert loss > 0
    rng = np.random.default_rng(seed + 100)
    sl = U.slices()
    picks = []
    for name in ["e0a", "e1b", "bb", "d1a", "d0a", "d0b"]:       # weights of every level and both concats
        w, b = sl[name]
        idx = np.arange(w.start, w.stop)
        picks.append(int(idx[np.argmax(np.abs(g[idx]) * rng.uniform(0.5, 1.0, idx.size))]))
        picks.append(int(b.start + np.argmax(np.abs(g[b]))))
    picks += [sl["head"][0].start + 3, sl["head"][1].start]
    for i in picks:
        p = params.copy()
        h = np.float32(1e-4 * max(1.0, abs(float(params[i]))))
        p[i] = params[i] + h
        lp = U.loss_grad(dims, p, r0n, types, target, rounding=False)[0]
        hp = float(p[i]) - float(params[i])
        p[i] = params[i] - h
        lm = U.loss_grad(dims, p, r0n, types, target, rounding=False)[0]
        hm = float(params[i]) - float(p[i])
        fd = (lp - lm) / (hp + hm)
        # ReLU kinks crossed inside +-h leave a small mismatch; structural
        # errors (a missing term, a wrong tap or channel) are O(1)
        assert abs(fd - g[i]) <= 2e-2 * max(abs(g[i]), 1e-2 * np.abs(g).max()), (i, fd, g[i])

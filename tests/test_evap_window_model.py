"""The parallel evaporation walk (k_evap_wsum/band/table/chain/emit in
watersim-v1_b200/csrc/ws_frame.cu), restated in Python with small windows,
against the serial _evS walk of _evapChunk (js/solver.js:3028-3125).

The GPU parity tests run the device passes on real planets, where band
misses and u1 retries almost never happen. Here the same pass structure runs
with bands only 2 or 4 inputs wide (forcing the direct resolve of a window in
the chain) and with a retry threshold raised from 5 to 5% of 2^32 (forcing
irregular kicks and host restarts), and must reproduce the serial walk's
ejection flags and final stream state exactly.
"""
import math
import random

M = 2 ** 32
A1, C1 = 1664525, 1013904223


def nxt(u):
    return (u * A1 + C1) % M


def affine(k):
    """T^k(x) = A x + C for the generator T."""
    A, C, a, c = 1, 0, A1, C1
    while k:
        if k & 1:
            A, C = A * a % M, (C * a + c) % M
        c, a = c * (a + 1) % M, a * a % M
        k >>= 1
    return A, C


def jump(u, k):
    A, C = affine(k % M)
    return (A * u + C) % M


A6, C6 = affine(6)


def kick_end(s, th):
    for _ in range(3):
        while True:
            s = nxt(s)
            if s >= th:
                break
        s = nxt(s)
    return s


def serial(s, thr, th):
    """The reference's order: one decision draw per candidate, six or more per kick."""
    flags = []
    for t in thr:
        s = nxt(s)
        if s > t:
            flags.append(0)
            continue
        s = kick_end(s, th)
        flags.append(1)
    return s, flags


def resolve(b, thr, e_in, emit=None):
    A, C = affine(6 * e_in)
    e = e_in
    for j in range(len(b)):
        u = (A * b[j] + C) % M
        if u <= thr[j]:
            if emit:
                emit(j, e, u)
            e += 1
            C, A = (A6 * C + C6) % M, A6 * A % M
    return e


def windowed(s, thr, W, K, th, stats):
    n = len(thr)
    t0, eoff, s_start = 0, 0, s
    flags, ej = [0] * n, {}
    while True:
        nw = (n - t0 + W - 1) // W if n > t0 else 0
        wins = [thr[t0 + w * W: t0 + (w + 1) * W] for w in range(nw)]
        wsum = [sum(0 if v < 0 else 1 if v >= M else v / M for v in win) for win in wins]
        L, acc = [], 0.0
        for w in range(nw):
            L.append(max(0, math.floor(acc) - K // 2))
            acc += wsum[w]
        b = [jump(s_start, t - t0 + 1) for t in range(t0, n)]
        bw = [b[w * W:(w + 1) * W] for w in range(nw)]
        tables = [[resolve(bw[w], wins[w], L[w] + k) - (L[w] + k) for k in range(K)] for w in range(nw)]
        e, e_w = 0, []
        for w in range(nw):                        # the chain, with the direct resolve on a band miss
            e_w.append(e)
            rel = e - L[w]
            if 0 <= rel < K:
                e += tables[w][rel]
            else:
                stats['misses'] += 1
                e = resolve(bw[w], wins[w], e)
        n_ej, s_end = e, jump(s_start, (n - t0) + 6 * e)
        irr, rec = None, {}
        for w in range(nw):                        # the emit pass
            def em(j, e, u, w=w):
                nonlocal irr
                rec[e] = (t0 + w * W + j, u)
                s1 = nxt(u)
                s3 = nxt(nxt(s1))
                s5 = nxt(nxt(s3))
                if min(s1, s3, s5) < th and (irr is None or (e, w * W + j) < irr):
                    irr = (e, w * W + j)
            resolve(bw[w], wins[w], e_w[w], em)
        if irr is None:
            for e, (t, _) in rec.items():
                ej[eoff + e] = t
            total, s_fin = eoff + n_ej, s_end
            break
        stats['restarts'] += 1
        e_irr, t_irr = irr                         # the host restart after an irregular kick
        for e, (t, _) in rec.items():
            if e <= e_irr:
                ej[eoff + e] = t
        q = kick_end(rec[e_irr][1], th)
        eoff += e_irr + 1
        t0 += t_irr + 1
        if t0 >= n:
            total, s_fin = eoff, q
            break
        s_start = q
    for k in range(total):
        flags[ej[k]] = 1
    return s_fin, flags


def test_windowed_walk_equals_serial_walk():
    rnd = random.Random(3)
    stats = {'misses': 0, 'restarts': 0}
    for case in range(120):
        n = rnd.randint(0, 260)
        thr = []
        for _ in range(n):
            r = rnd.random()
            if r < 0.05:
                thr.append(-1)                     # never ejects
            elif r < 0.10 and case % 2:
                thr.append(M)                      # always ejects (prob >= 1)
            else:
                thr.append(int(rnd.choice([0.001, 0.01, 0.05, 0.3]) * M))
        s0 = rnd.randrange(M)
        th = rnd.choice([5, 5, int(0.05 * M)])
        W = rnd.choice([8, 32, 64])
        K = rnd.choice([2, 4, 64])
        ref = serial(s0, thr, th)
        assert windowed(s0, thr, W, K, th, stats) == ref, (case, n, W, K, th)
    assert stats['restarts'] > 10 and stats['misses'] > 10   # both fallback paths ran

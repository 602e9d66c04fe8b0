"""A second, deliberately naive restatement of the reference's local move and
modularity in pure Python (test-only; for graphs of a few hundred vertices).

It cross-checks the C oracle: two independent restatements of
src/louvain/louvain.cu:404-589 (gain, tie-break, clamp) and :105-238 (Q).
"""
from __future__ import annotations

import numpy as np


def local_move(n, offsets, cols, weights, C, sigma, k, mass, version=2, up=True):
    m = mass / 2.0
    out = np.zeros(n, np.uint32)
    for i in range(n):
        src = int(C[i])
        ki = float(k[i])
        a = float(sigma[src]) - ki
        kic = {}
        e = 0.0
        for p in range(int(offsets[i]), int(offsets[i + 1])):
            j = int(cols[p])
            c = int(C[j])
            w = 1.0 if weights is None else float(weights[p])
            if version == 1:
                cand = c < src if up else c > src
            else:
                cand = c != src
            if cand:
                kic[c] = kic.get(c, 0.0) + w
            elif c == src and j != i:
                e += w
        best, dst = 0.0, src
        for c, val in kic.items():
            t = ki * (a - float(sigma[c]))
            t = t / (2.0 * m)
            t = e - t
            g = (val - t) / m
            if g > best or (g == best and (c < dst if up else c > dst)):
                best, dst = g, c
        if version == 1:
            out[i] = dst
        else:
            out[i] = min(dst, src) if up else max(dst, src)
    return out


def modularity(n, offsets, cols, weights, C):
    w = np.ones(len(cols)) if weights is None else np.asarray(weights, dtype=np.float64)
    k = np.zeros(n)
    sin = 0.0
    for i in range(n):
        for p in range(int(offsets[i]), int(offsets[i + 1])):
            k[i] += w[p]
            if C[int(cols[p])] == C[i]:
                sin += w[p]
    sig = np.zeros(n)
    for i in range(n):
        sig[C[i]] += k[i]
    mass = w.sum()
    return sin / mass - (sig * sig).sum() / (mass * mass)

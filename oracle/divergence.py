"""Explaining streamline differences against the oracle -- TEST INFRASTRUCTURE ONLY.

The oracle emulates the stop map's hardware texture filter with 8-bit
weights; the hardware's filter arithmetic is not documented and differs from
the emulation by up to ~4e-3 (measured, tests/golden/tex.npz).  A stop
decision can therefore flip when the filtered value lands within that band of
the threshold.  After such a flip the two runs consume different numbers of
Philox draws, so every later streamline of the same seed is unrelated.
`explain` accepts a difference only if, in tracking order, the first differing
track of the seed is a strict prefix of the other one and the point where
they part has a stop-map value within `band` of the threshold.
"""

from __future__ import annotations

import numpy as np


def split(L, P):
    off = np.concatenate([[0], np.cumsum(L)])
    return [P[off[i]:off[i + 1]] for i in range(len(L))]


def _seed_index(sl, seed):
    hit = np.nonzero(np.all(sl == seed, axis=1))[0]
    return int(hit[0]) if len(hit) else None


def _prefix_split(a, b):
    """If one array is a strict prefix of the other return the parting index."""
    n = min(len(a), len(b))
    if len(a) == len(b) or not np.array_equal(a[:n], b[:n]):
        return None
    return n


def explain(La, Pa, Lb, Pb, S, seeds, stop_value, thr, band=5e-3):
    """Return (n_identical_seeds, n_explained_seeds, n_unexplained_seeds)."""
    A, B = split(La, Pa), split(Lb, Pb)
    ident = expl = bad = 0
    for s in np.unique(S):
        idx = np.nonzero(S == s)[0]
        pairs = [(A[j], B[j]) for j in idx]
        if all(a.shape == b.shape and np.array_equal(a, b) for a, b in pairs):
            ident += 1
            continue
        ok = False
        for a, b in pairs:
            if a.shape == b.shape and np.array_equal(a, b):
                continue
            ia, ib = _seed_index(a, seeds[s]), _seed_index(b, seeds[s])
            if ia is None or ib is None:
                break
            for pa, pb in ((a[ia::-1], b[ib::-1]), (a[ia:], b[ib:])):
                if np.array_equal(pa, pb):
                    continue
                m = _prefix_split(pa, pb)
                if m is not None:
                    longer = pa if len(pa) > len(pb) else pb
                    v = stop_value(longer[m:m + 1])[0]
                    ok = abs(float(v) - thr) < band
                break
            break
        expl += ok
        bad += not ok
    return ident, expl, bad

"""The cooperative kNN list (scan 8 of the single-pass flock kernel),
restated in Python over 32-candidate rounds, against the reference's
sequential replacement (Proximity3D_resources.cu:71-104, restated in the
oracle): the first M accepted fill the list with one ballot, then only
candidates below max(bound, previous bound) are tried one at a time, each
replacing the first entry holding the largest distance when it is below the
(stale) bound.  Random candidate streams with ties, repeated distances and
NaN, CPU only."""
import math
import random

import numpy as np


def reference(dists, M):
    lst, dl = [], []
    mx = 0.0
    for j, d in enumerate(dists):
        if d > 4.0:                      # the radius test (NaN passes it)
            continue
        if len(lst) < M:
            lst.append(j)
            dl.append(d)
            mx = mx if not (mx < d) else d   # std::max(maxDistValue, dist)
        elif d < mx:
            mx = dl[0]
            idx = 0
            for k in range(1, len(dl)):
                if mx < dl[k]:
                    mx = dl[k]
                    idx = k
            lst[idx] = j
            dl[idx] = d
    return lst


def cooperative(dists, M):
    ks = [0] * 32
    kd = [0.0] * 32
    an = 0
    amx = amx_prev = 0.0
    for base in range(0, len(dists), 32):
        rnd = dists[base:base + 32]
        acc = [not (d > 4.0) for d in rnd]
        bal = [i for i, a in enumerate(acc) if a]
        if an < M:
            take = bal[:M - an]
            for k, src in enumerate(take):
                ks[an + k] = base + src
                kd[an + k] = rnd[src]
            vals = [rnd[s] for s in take if not math.isnan(rnd[s])]
            if take:
                amx = max(amx, max(vals) if vals else 0.0)
            an += len(take)
            bal = bal[len(take):]
            amx_prev = amx
        ceil_b = amx if math.isnan(amx_prev) else (amx_prev if math.isnan(amx) else max(amx, amx_prev))
        bal = [s for s in bal if rnd[s] < ceil_b]
        for src in bal:
            cd = rnd[src]
            if cd < amx:
                d0 = kd[0]
                if math.isnan(d0):
                    idx, mv = 0, d0
                else:
                    ok = [k for k in range(an) if not math.isnan(kd[k])]
                    mv = max(kd[k] for k in ok)
                    idx = min(k for k in ok if kd[k] == mv)
                amx_prev, amx = amx, mv
                ks[idx] = base + src
                kd[idx] = cd
    return ks[:an]


def _stream(rng, n, pool):
    out = []
    for _ in range(n):
        u = rng.random()
        if u < 0.02:
            out.append(float("nan"))
        elif u < 0.25:
            out.append(rng.uniform(4.0, 6.0))       # beyond the radius
        elif u < 0.45:
            out.append(rng.choice(pool))              # repeated distances (ties)
        else:
            out.append(float(np.float32(rng.uniform(0.0, 4.0))))
    return out


def test_cooperative_knn_matches_sequential_replacement():
    rng = random.Random(11)
    for trial in range(4000):
        M = rng.choice([1, 2, 5, 16, 31, 32])
        n = rng.randrange(0, 400)
        pool = [float(np.float32(rng.uniform(0.0, 4.0))) for _ in range(rng.randrange(1, 6))]
        d = _stream(rng, n, pool)
        assert cooperative(d, M) == reference(d, M), (trial, M)


def test_the_bound_can_rise():
    # the stale bound rises after a replacement whose candidate lies above
    # the list's new maximum: the ceiling keeps such later candidates in play
    d = [3.0, 1.0, 2.5, 0.5, 2.0]
    assert reference(d, 2) == cooperative(d, 2)
    rng = random.Random(3)
    rose = 0
    for _ in range(800):
        M = rng.choice([2, 3, 4])
        dd = [float(np.float32(rng.uniform(0.0, 4.0))) for _ in range(rng.randrange(5, 40))]
        lst, dl, mx, seq = [], [], 0.0, []
        for j, x in enumerate(dd):
            if len(lst) < M:
                lst.append(j); dl.append(x); mx = max(mx, x)
            elif x < mx:
                mx = max(dl); idx = dl.index(mx); lst[idx] = j; dl[idx] = x; seq.append(mx)
        rose += any(b > a for a, b in zip(seq, seq[1:]))
        assert cooperative(dd, M) == reference(dd, M)
    assert rose > 0

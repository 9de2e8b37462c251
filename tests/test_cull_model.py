"""The bounding-box cull of the cooperative scan (scan variant 7), restated
in numpy float32: the squared distance from a candidate to the box of a home
cell's agents, built like an agent's own d2, is never above any of those
agents' d2, so a candidate it drops fails every agent's radius test.  Checked
on random runs, on candidates placed on and next to the box faces, and on
positions near float32 spacing limits (CPU only).  Also the whole-cell cull
of the per-agent scans (exact for positions inside their cells, not for NaN
candidates, hence its gate) and the power-of-two cell units (product with the
reciprocal equal to the quotient)."""
import numpy as np

F = np.float32


def _d2(dx, dy, dz):
    # (dx * dx + dy * dy) + dz * dz, one rounding per operation
    return F(F(F(dx * dx) + F(dy * dy)) + F(dz * dz))


def _box_d2(q, lo, hi):
    e = [np.maximum(np.maximum(F(lo[k] - q[k]), F(q[k] - hi[k])), F(0)) for k in range(3)]
    return _d2(*e)


def _pair_d2(cands, agents):
    d = (cands[:, None, :] - agents[None, :, :]).astype(F)   # one rounding per subtraction
    return _d2(d[..., 0], d[..., 1], d[..., 2])


def _check(agents, cands):
    lo, hi = agents.min(axis=0), agents.max(axis=0)
    b = _box_d2(cands.T, lo, hi)
    d = _pair_d2(cands, agents)
    assert (b[:, None] <= d).all()


def test_box_distance_bounds_every_agent_random_runs():
    rng = np.random.default_rng(7)
    for _ in range(300):
        k = int(rng.integers(1, 12))
        base = rng.uniform(0, 252, 3)
        agents = (base + rng.uniform(0, 4, (k, 3))).astype(F)
        cands = (base + rng.uniform(-4, 8, (40, 3))).astype(F)
        _check(agents, cands)


def test_box_distance_bounds_on_faces_and_spacing_limits():
    rng = np.random.default_rng(8)
    for scale in (1.0, 255.99, 1e-3, 1e6):
        agents = (rng.uniform(0, 1, (5, 3)) * scale).astype(F)
        lo, hi = agents.min(axis=0), agents.max(axis=0)
        cands = [lo.copy(), hi.copy()]
        for k in range(3):
            for v in (np.nextafter(lo[k], F(-np.inf)), np.nextafter(hi[k], F(np.inf))):
                q = agents[0].copy()
                q[k] = v
                cands.append(q)
        cands += list((lo + (hi - lo) * rng.uniform(-2, 3, (30, 3))).astype(F))
        _check(agents, np.array(cands, F))


def test_dropped_candidates_fail_the_radius_test():
    # with the library's threshold (largest d2 whose sqrt does not exceed r)
    r = F(4.0)
    thr = F(r * r)
    while np.sqrt(np.nextafter(thr, F(np.inf))) <= r:
        thr = np.nextafter(thr, F(np.inf))
    rng = np.random.default_rng(9)
    dropped = 0
    for _ in range(200):
        agents = (F(100) + rng.uniform(0, 4, (3, 3))).astype(F)
        lo, hi = agents.min(axis=0), agents.max(axis=0)
        cands = (F(100) + rng.uniform(-4, 8, (50, 3))).astype(F)
        drop = _box_d2(cands.T, lo, hi) > thr
        dropped += int(drop.sum())
        assert (_pair_d2(cands[drop], agents) > thr).all()
    assert dropped > 1000


# ---------------------------------------------------------------------------
# The whole-cell cull of scan variants 0 and 1, restated: a neighbour cell is
# skipped when the squared distance from the agent to the shared faces
# exceeds the radius threshold plus a margin.  Exact while every position
# lies in its hashed cell; a NaN position (hashed to cell 0, accepted by
# every agent that reads it) breaks it, which is why the kernels skip the cull
# for a step whose sorted state holds one.

def _grid(x, cell, G):
    q = np.floor(x / cell)
    return 0 if np.isnan(q) else int(min(max(q, 0), G - 1))


def _culled_lists(pos, L, cell, M, thr, cull):
    """First-M lists in the reference's visit order from the sorted state,
    with the face-distance cell cull on or off."""
    G = int(round(L / cell))
    g = np.array([[_grid(v, cell, G) for v in p] for p in pos])
    key = (g[:, 2] * G + g[:, 1]) * G + g[:, 0]
    order = np.argsort(key, kind="stable")
    sp, sk, sg = pos[order], key[order], g[order]
    cs = np.searchsorted(sk, np.arange(G ** 3))
    ce = np.searchsorted(sk, np.arange(G ** 3), side="right")
    margin = F(F(thr + F(0.01)) + F(F(F(1e-6) * F(cell)) * F(L)))
    lists = []
    for i in range(len(sp)):
        p, h = sp[i], sg[i]
        lo2 = [F(F(p[a] - F(F(h[a]) * F(cell))) ** 2) for a in range(3)]
        hi2 = [F(F(F(F(h[a] + 1) * F(cell)) - p[a]) ** 2) for a in range(3)]
        out = []
        for ox in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for oz in (-1, 0, 1):
                    o = (ox, oy, oz)
                    b = F(0)
                    for a in range(3):
                        b = F(b + (lo2[a] if o[a] < 0 else (hi2[a] if o[a] > 0 else F(0))))
                    if cull and b > margin:
                        continue
                    c = [h[a] + o[a] for a in range(3)]
                    s = [F(-L) if c[a] < 0 else (F(L) if c[a] >= G else F(0)) for a in range(3)]
                    cw = [c[a] % G for a in range(3)]
                    hh = (cw[2] * G + cw[1]) * G + cw[0]
                    for j in range(cs[hh], ce[hh]):
                        if j == i or len(out) == M:
                            continue
                        d = [F(F(sp[j, a] + s[a]) - p[a]) for a in range(3)]
                        if not (_d2(*d) > thr):
                            out.append(j)
        lists.append(out)
    return lists


def _thr(r):
    thr = F(F(r) * F(r))
    while np.sqrt(np.nextafter(thr, F(np.inf))) <= r:
        thr = np.nextafter(thr, F(np.inf))
    while np.sqrt(thr) > r:
        thr = np.nextafter(thr, F(0))
    return thr


def test_cell_cull_exact_for_positions_in_their_cells():
    rng = np.random.default_rng(21)
    L, cell, thr = 16.0, 4.0, _thr(F(4.0))
    pos = rng.uniform(0, L, (300, 3)).astype(F)
    pos[:20, 0] = F(4.0) * rng.integers(0, 4, 20).astype(F)          # on cell faces
    pos[20:30] = np.nextafter(F(L), F(0))                              # against the far faces
    assert _culled_lists(pos, L, cell, 40, thr, True) == _culled_lists(pos, L, cell, 40, thr, False)


def test_cell_cull_drops_nan_candidates_sharing_cell_zero():
    rng = np.random.default_rng(22)
    L, cell, thr = 16.0, 4.0, _thr(F(4.0))
    pos = rng.uniform(0, L, (300, 3)).astype(F)
    pos[:3] = np.nan
    with np.errstate(invalid="ignore"):
        full = _culled_lists(pos, L, cell, 40, thr, False)
        culled = _culled_lists(pos, L, cell, 40, thr, True)
    assert full != culled


# x / cell for a power-of-two cell is computed as x * (1 / cell) on the
# device: the two are the correctly rounded values of the same real number.

def test_power_of_two_cell_units_equal_the_quotient():
    rng = np.random.default_rng(23)
    xs = np.concatenate([
        rng.uniform(-300, 300, 20000).astype(F),
        (rng.standard_normal(2000) * F(1e-38)).astype(F),              # subnormal results
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 3.0e38, -3.0e38, 1e-45], F),
        np.nextafter(F(4.0) * np.arange(-64, 65, dtype=F), F(np.inf)),
        np.nextafter(F(4.0) * np.arange(-64, 65, dtype=F), F(-np.inf)),
    ])
    for cell in (F(0.25), F(1.0), F(2.0), F(4.0), F(8.0), F(1024.0)):
        with np.errstate(invalid="ignore", over="ignore", under="ignore"):
            q = xs / cell
            m = xs * (F(1.0) / cell)
        nq, nm = np.isnan(q), np.isnan(m)
        assert np.array_equal(nq, nm)
        assert np.array_equal(q[~nq].view(np.uint32), m[~nm].view(np.uint32)), cell
    # and the host's test for a power of two keeps other cells on the quotient
    for cell, pow2 in ((4.0, True), (0.5, True), (3.0, False), (2.5, False), (6.0, False)):
        m, e = np.frexp(np.float32(cell))
        assert (m == 0.5) == pow2

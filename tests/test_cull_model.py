"""The bounding-box cull of the cooperative scan (scan variant 7), restated
in numpy float32: the squared distance from a candidate to the box of a home
cell's agents, built like an agent's own d2, is never above any of those
agents' d2, so a candidate it drops fails every agent's radius test.  Checked
on random runs, on candidates placed on and next to the box faces, and on
positions near float32 spacing limits (CPU only)."""
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

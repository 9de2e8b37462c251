"""The incremental re-sort's algorithm (csrc/brt_resort.cu), restated in
numpy and checked against a stable sort on (cell, id): the order it builds
from the previous step's order must be exactly the full sort's, for any
movement.  CPU only; the GPU kernels are checked against the full sort and
the oracle in tests/test_gpu_resort.py."""
import numpy as np
import pytest

MAX_MOVERS_PER_CELL = 32


def _previous_order(rng, n, cells):
    """Canonical slots as a fused step leaves them: sorted by (cell, id)."""
    ids = rng.permutation(n)
    key = rng.integers(0, cells, n)
    order = np.lexsort((ids, key))
    return key[order], ids[order]


def _ranges(key, cells):
    start = np.full(cells, -1)
    end = np.full(cells, -1)
    for j, c in enumerate(key):
        if j == 0 or key[j - 1] != c:
            start[c] = j
        if j == len(key) - 1 or key[j + 1] != c:
            end[c] = j + 1
    return start, end


def resort(old_key, ids, new_key, cells, chunk):
    """Sorted slots of the new step, or None where the device would take the
    full sort (a cell receiving more than MAX_MOVERS_PER_CELL movers)."""
    n = len(ids)
    stay = new_key == old_key
    start, end = _ranges(old_key, cells)
    # mark: stayer prefix inside each chunk and the chunk totals
    prefix = np.zeros(n, np.int64)
    chunk_total = []
    for b in range(0, n, chunk):
        s = stay[b:b + chunk].astype(np.int64)
        prefix[b:b + chunk] = np.cumsum(s) - s
        chunk_total.append(int(s.sum()))
    chunk_base = np.concatenate([[0], np.cumsum(chunk_total)])
    movers = {}
    for j in np.nonzero(~stay)[0]:
        movers.setdefault(int(new_key[j]), []).append(int(j))
    if any(len(m) > MAX_MOVERS_PER_CELL for m in movers.values()):
        return None

    def before(x):  # stayers among slots [0, x)
        return chunk_base[x // chunk] + prefix[x] if x < n else chunk_base[-1]

    # cell scan: totals, starts, and each cell's base for its stayers
    total = np.zeros(cells, np.int64)
    ahead = np.zeros(cells, np.int64)
    for c in range(cells):
        stayers = 0
        if start[c] >= 0:
            ahead[c] = before(start[c])
            stayers = before(end[c]) - ahead[c]
        total[c] = stayers + len(movers.get(c, []))
    new_start = np.concatenate([[0], np.cumsum(total)])[:cells]
    stay_base = new_start - ahead
    # place
    out = np.full(n, -1)
    for j in range(n):
        c = int(new_key[j])
        if stay[j]:
            pos = stay_base[c] + before(j)
        else:
            pos = new_start[c]
            if start[c] >= 0:
                lo, hi = start[c], end[c]
                while lo < hi:
                    mid = (lo + hi) // 2
                    if ids[mid] < ids[j]:
                        lo = mid + 1
                    else:
                        hi = mid
                pos += before(lo) - before(start[c])
        pos += sum(1 for m in movers.get(c, []) if ids[m] < ids[j])
        assert out[pos] == -1, "two slots placed at one position"
        out[pos] = j
    return out


@pytest.mark.parametrize("seed", range(12))
def test_resort_equals_full_sort(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 2500))
    cells = int(rng.integers(1, 600))
    old_key, ids = _previous_order(rng, n, cells)
    for frac in (0.0, 0.03, 0.3, 1.0):
        new_key = old_key.copy()
        moved = rng.random(n) < frac
        # movers go to a nearby cell, like agents crossing a face
        new_key[moved] = np.clip(old_key[moved] + rng.integers(-3, 4, moved.sum()), 0, cells - 1)
        got = resort(old_key, ids, new_key, cells, chunk=int(rng.choice([32, 64, 1024])))
        if got is None:
            continue  # the full sort runs
        assert np.array_equal(got, np.lexsort((ids, new_key)))


def test_crowded_cell_takes_the_full_sort():
    rng = np.random.default_rng(3)
    old_key, ids = _previous_order(rng, 400, 50)
    new_key = old_key.copy()
    new_key[old_key != 7] = np.where(rng.random((old_key != 7).sum()) < 0.2, 7, old_key[old_key != 7])
    assert (new_key != old_key).sum() > MAX_MOVERS_PER_CELL
    assert resort(old_key, ids, new_key, 50, chunk=64) is None


def test_empty_and_single_agent():
    assert resort(np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64), 4, 32).size == 0
    got = resort(np.array([2]), np.array([0]), np.array([3]), 5, 32)
    assert np.array_equal(got, [0])

"""Independent numpy restatement of the neighbour-list contract, used to
cross-check the C++ oracle on small inputs (test helper)."""
import numpy as np


def grid_coord(x, cell, G):
    g = np.floor(x.astype(np.float32) / np.float32(cell)).astype(np.int64)
    return np.clip(g, 0, G - 1)


def lists_bruteforce(pos_sorted, L, cell, radius, M, self_slots=None):
    """pos_sorted: (n,4) float32 in sorted order.  Returns list of lists of
    sorted slots in the reference visit order (x outer, y, z inner, then slot),
    truncated at M, using float32 arithmetic q+s, (q+s)-p, ((dx*dx+dy*dy)+dz*dz),
    accept iff not sqrt(d2) > radius."""
    G = int(round(L / cell))
    n = pos_sorted.shape[0]
    p = pos_sorted[:, :3].astype(np.float32)
    g = grid_coord(p, cell, G)
    out = []
    f32 = np.float32
    for i in range(n):
        cands = []
        for j in range(n):
            if j == i:
                continue
            o = []
            s = []
            ok = True
            for a in range(3):
                d = (g[j, a] - g[i, a]) % G
                if d == 0:
                    o.append(0); s.append(f32(0))
                elif d == 1:
                    o.append(1); s.append(f32(L) if g[i, a] == G - 1 else f32(0))
                elif d == G - 1:
                    o.append(-1); s.append(f32(-L) if g[i, a] == 0 else f32(0))
                else:
                    ok = False
                    break
            if not ok:
                continue
            dx = f32(f32(p[j, 0] + s[0]) - p[i, 0])
            dy = f32(f32(p[j, 1] + s[1]) - p[i, 1])
            dz = f32(f32(p[j, 2] + s[2]) - p[i, 2])
            d2 = f32(f32(f32(dx * dx) + f32(dy * dy)) + f32(dz * dz))
            if np.sqrt(d2, dtype=np.float32) > f32(radius):
                continue
            visit = (o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)
            cands.append((visit, j))
        cands.sort()
        out.append([j for _, j in cands[:M]])
    return out

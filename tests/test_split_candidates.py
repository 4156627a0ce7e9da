"""The half-warp split of small BVH nodes (k_split_tiny in scene_build.cu) evaluates
the SAH only at the last triangle of each occupied bin, in bin order, instead of
sweeping every bin boundary (bvh.ts:110-144). This checks on the host, with the
same float bounds and double costs, that both give the same choice: the same cost,
split bin and left count, and no split where the sweep has none."""
import math

import numpy as np


def _area(b):
    dx, dy, dz = b[3] - b[0], b[4] - b[1], b[5] - b[2]
    return dx * dy + dy * dz + dz * dx


def _union(boxes):
    return [min(b[0] for b in boxes), min(b[1] for b in boxes), min(b[2] for b in boxes),
            max(b[3] for b in boxes), max(b[4] for b in boxes), max(b[5] for b in boxes)]


def _sweep(bins_of, boxes, bins):
    """Every boundary after bin s, first minimum wins (the binned sweep)."""
    cnt, bb = [0] * bins, [None] * bins
    for b, x in zip(bins_of, boxes):
        cnt[b] += 1
        bb[b] = x if bb[b] is None else _union([bb[b], x])
    best = (math.inf, -1, 0)
    for s in range(bins - 1):
        lc, rc = sum(cnt[:s + 1]), sum(cnt[s + 1:])
        if lc == 0 or rc == 0:
            continue
        cost = lc * _area(_union([bb[i] for i in range(s + 1) if cnt[i]])) + \
            rc * _area(_union([bb[i] for i in range(s + 1, bins) if cnt[i]]))
        if cost < best[0]:
            best = (cost, s, lc)
    return best


def _sorted_candidates(bins_of, boxes):
    """The last triangle of each occupied bin in (bin, index) order, ties to the lower bin."""
    n = len(boxes)
    order = sorted(range(n), key=lambda i: (bins_of[i], i))
    best = (math.inf, -1, 0)
    for p in range(n - 1):
        if bins_of[order[p]] == bins_of[order[p + 1]]:
            continue
        cost = (p + 1) * _area(_union([boxes[order[q]] for q in range(p + 1)])) + \
            (n - p - 1) * _area(_union([boxes[order[q]] for q in range(p + 1, n)]))
        s = bins_of[order[p]]
        if cost < best[0] or (cost == best[0] and s < best[1]):
            best = (cost, s, p + 1)
    return best


def test_sorted_candidates_choose_what_the_binned_sweep_chooses():
    rng = np.random.default_rng(1)
    checked = 0
    for trial in range(4000):
        n = int(rng.integers(2, 17))
        bins = int(rng.choice([16, 32]))
        lo = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
        hi = lo + rng.uniform(0, 0.5, (n, 3)).astype(np.float32)
        if trial % 3 == 0:
            hi = lo.copy()  # flat boxes: zero areas, equal costs
        boxes = [[float(v) for v in lo[i]] + [float(v) for v in hi[i]] for i in range(n)]
        c = ((lo + hi) / 2).astype(np.float32)
        if trial % 5 == 0:
            c[:, 0] = np.round(c[:, 0], 1)  # shared centroids: several triangles per bin
        for a in range(3):
            cmin, cmax = float(c[:, a].min()), float(c[:, a].max())
            if not cmax - cmin > 0:
                continue
            scale = bins / (cmax - cmin)
            b = [int(min(bins - 1, math.floor((float(x) - cmin) * scale))) for x in c[:, a]]
            want, got = _sweep(b, boxes, bins), _sorted_candidates(b, boxes)
            assert got[0] == want[0]
            if want[0] < math.inf:
                assert got[1:] == want[1:]
            checked += 1
    assert checked > 8000

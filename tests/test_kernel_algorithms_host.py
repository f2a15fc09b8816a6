"""The algorithms of the descriptor and archetype kernels, restated step for step in Python and
checked against the oracles on many random and ragged inputs (CPU; the kernels themselves are
checked on the GPU by the -m gpu suite):

* k_chords_seg: lines cut into segments of at most 32 cells, runs between a segment's solid cells
  emitted by its thread, segment summaries (leading pore, trailing pore, all pore) joined in order
  by the line's first lane, the wrap-around chord closed at the end;
* k_label_tiles + k_label_merge + k_label_roots: 26-connected clusters labelled inside tiles of
  8 x 8 x 16 cells (z-runs linked first, then the other 12 forward neighbours), tile-local roots as
  global indices, unions across tile faces, local sizes and box faces passed to the final roots;
* k_stamp_first + k_first_hist: fibers or holes in batches, each cell keeping the first one that
  covers it; the one-at-a-time loop's stopping point from the per-shape new cells.
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy.ndimage import label

from oracle import morphology as om
from porerad_b200 import geometry as g

# ---------------------------------------------------------------------------- segmented chords


def seg_lanes(N: int) -> tuple[int, int]:
    lpl = 1
    while lpl < 32 and -(-N // lpl) > 16:
        lpl *= 2
    return lpl, -(-N // lpl)


def chords_segmented(line: np.ndarray) -> np.ndarray:
    N = len(line)
    lpl, seg = seg_lanes(N)
    hist = np.zeros(N + 1, np.int64)
    summaries = []
    for part in range(lpl):
        s0 = part * seg
        cnt = 0 if s0 >= N else min(seg, N - s0)
        pre = suf = cnt
        if cnt:
            solid = [q for q in range(cnt) if not line[s0 + q]]
            if solid:
                pre, suf = solid[0], cnt - 1 - solid[-1]
                for p1, p2 in zip(solid, solid[1:]):
                    if p2 - p1 - 1 > 0:
                        hist[p2 - p1 - 1] += 1
        summaries.append((cnt, pre, suf, pre == cnt))
    run, head = 0, -1
    for cnt, pre, suf, full in summaries:
        if full:
            run += cnt
        else:
            run += pre
            if head < 0:
                head = run
            elif run:
                hist[run] += 1
            run = suf
    if head < 0:
        hist[N] += 1
    elif run + head:
        hist[run + head] += 1
    return hist


@pytest.mark.parametrize("N", [1, 2, 15, 16, 17, 31, 32, 33, 64, 100, 128, 129, 255, 500, 1024])
def test_segmented_chords_equal_the_oracle(N):
    rng = np.random.default_rng(N)
    for trial in range(40):
        p = [0.0, 1.0, 0.05, 0.5, 0.95][trial % 5] if trial < 5 else rng.random()
        line = rng.random(N) < p
        want, _, _, _ = om.periodic_chord_histogram(line.reshape(1, 1, N), 2)
        assert chords_segmented(line).tolist() == want.tolist()


# ---------------------------------------------------------------------------- tile labelling

TX, TY, TZ = 8, 8, 16


def _find(parent, x):
    while parent[x] != x:
        parent[x] = parent[parent[x]]
        x = parent[x]
    return x


def _union(parent, x, y):
    x, y = _find(parent, x), _find(parent, y)
    if x == y:
        return
    if x < y:
        x, y = y, x
    parent[x] = y  # the larger root under the smaller


FORWARD = [(q // 9 - 1, (q // 3) % 3 - 1, q % 3 - 1) for q in range(14, 27)]


def label_tiles(pore: np.ndarray):
    """(clusters, largest, percolation bits) by the kernels' three phases."""

    nx, ny, nz = pore.shape
    n = pore.size
    gidx = lambda i, j, k: (i * ny + j) * nz + k  # noqa: E731
    parent = np.full(n, -1, np.int64)
    size = np.zeros(n, np.int64)
    faces = np.zeros(n, np.int64)
    for ti in range(0, nx, TX):
        for tj in range(0, ny, TY):
            for tk in range(0, nz, TZ):
                loc = {}
                for li in range(TX):
                    for lj in range(TY):
                        for lk in range(TZ):
                            i, j, k = ti + li, tj + lj, tk + lk
                            if i < nx and j < ny and k < nz and pore[i, j, k]:
                                loc[(li, lj, lk)] = (li * TY + lj) * TZ + lk
                lp = {v: v for v in loc.values()}
                # z-runs first: a pore cell points at the first cell of its run
                for (li, lj, lk), v in loc.items():
                    s = lk
                    while s > 0 and (li, lj, s - 1) in loc:
                        s -= 1
                    lp[v] = (li * TY + lj) * TZ + s
                for (li, lj, lk), v in loc.items():
                    for di, dj, dk in FORWARD[1:]:
                        u = (li + di, lj + dj, lk + dk)
                        if u in loc:
                            _union(lp, v, loc[u])
                cnt, fc = {}, {}
                for (li, lj, lk), v in loc.items():
                    r = _find(lp, v)
                    ri, rj, rk = r // (TY * TZ), (r // TZ) % TY, r % TZ
                    i, j, k = ti + li, tj + lj, tk + lk
                    parent[gidx(i, j, k)] = gidx(ti + ri, tj + rj, tk + rk)
                    cnt[r] = cnt.get(r, 0) + 1
                    f = (i == 0) | (i == nx - 1) << 1 | (j == 0) << 2 | (j == ny - 1) << 3 | (k == 0) << 4 | \
                        (k == nz - 1) << 5
                    fc[r] = fc.get(r, 0) | f
                for r in cnt:
                    c = gidx(ti + r // (TY * TZ), tj + (r // TZ) % TY, tk + r % TZ)
                    size[c], faces[c] = cnt[r], fc[r]
    gp = {c: int(parent[c]) for c in range(n) if parent[c] >= 0}
    for c in list(gp):  # unions across tile faces
        i, j, k = c // (ny * nz), (c // nz) % ny, c % nz
        for di, dj, dk in FORWARD:
            a, b, cc = i + di, j + dj, k + dk
            same = (i % TX + di < TX) and 0 <= j % TY + dj < TY and 0 <= k % TZ + dk < TZ
            if same or not (a < nx and 0 <= b < ny and 0 <= cc < nz) or not pore[a, b, cc]:
                continue
            _union(gp, gp[c], gp[gidx(a, b, cc)])
    for c in np.flatnonzero(size):
        r = _find(gp, int(c))
        if r != c:
            size[r] += size[c]
            faces[r] |= faces[c]
    roots = [c for c in gp if _find(gp, c) == c]
    largest = max((int(size[r]) for r in roots), default=0)
    perc = 0
    for r in roots:
        for a in range(3):
            if (faces[r] >> (2 * a)) & 3 == 3:
                perc |= 1 << a
    return len(roots), largest, perc


@pytest.mark.parametrize("shape,p", [((1, 1, 1), 0.5), ((3, 5, 7), 0.6), ((9, 9, 17), 0.45), ((8, 8, 16), 0.35),
                                     ((17, 10, 33), 0.3), ((12, 20, 18), 0.7), ((16, 16, 16), 0.2)])
def test_tile_labelling_equals_scipy(shape, p):
    rng = np.random.default_rng(sum(shape))
    for _ in range(3):
        pore = rng.random(shape) < p
        lbl, n = label(pore, structure=np.ones((3, 3, 3), bool))
        sizes = np.bincount(lbl.ravel(), minlength=n + 1)[1:]
        perc = 0
        for a in range(3):
            lo = set(np.unique(np.take(lbl, 0, axis=a)).tolist()) - {0}
            hi = set(np.unique(np.take(lbl, lbl.shape[a] - 1, axis=a)).tolist()) - {0}
            perc |= int(bool(lo & hi)) << a
        assert label_tiles(pore) == (n, int(sizes.max()) if n else 0, perc)


# ---------------------------------------------------------------------------- first-cover batches


def fibers_batched(n, phi, seed, aligned, batch):
    rng = np.random.default_rng(seed)
    ball = g._ball(2.0)
    target = phi * n ** 3
    if not 0 < target:
        return np.zeros((n,) * 3, np.uint8)
    first = np.full(n ** 3, np.iinfo(np.int32).max, np.int64)
    base, count, last = 0, 0, -1
    while last < 0:
        nodes = [g._segment_points(*g._fiber_draws(n, rng, aligned)) % n for _ in range(batch)]
        for f, nd in enumerate(nodes):
            p = ((nd[:, None, :] + ball[None, :, :]) % n).reshape(-1, 3)
            np.minimum.at(first, (p[:, 0] * n + p[:, 1]) * n + p[:, 2], base + f)
        new = np.bincount(first[(first >= base) & (first < base + batch)] - base, minlength=batch)
        for f in range(batch):
            count += int(new[f])
            if not count < target:
                last = base + f
                break
        base += batch
    return (first <= last).astype(np.uint8).reshape((n,) * 3)


@pytest.mark.parametrize("arch,n,phi,seed,batch", [("FI", 32, 0.10, 0, 64), ("FA", 40, 0.15, 3, 5),
                                                   ("FI", 24, 0.30, 7, 1), ("FA", 16, 0.0, 1, 64)])
def test_batched_fibers_equal_the_one_at_a_time_loop(arch, n, phi, seed, batch):
    assert np.array_equal(fibers_batched(n, phi, seed, arch == "FA", batch), g.make(arch, n, phi, seed))

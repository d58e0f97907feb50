"""The ray binning walks the tiles a ray's support can reach (k3dom_b200/csrc/evidence.cu:
for_each_tile): the segment is clipped to the grid grown by R, then walked slab by slab along its
dominant axis, and each candidate tile's cell-centre box grown by R is tested against the
segment in FP32. The placed ray lists give each ray two threads, one per alternate slab
(first = 0, 1; step = 2). This restates the walk and checks, against brute force, that every
tile holding a cell centre within R of the segment is visited, and that the two threads'
walks split the full walk with nothing missed or repeated, and that no walk exceeds the per-ray
bound the lists are sized by. CPU only."""
import math

import numpy as np

f32 = np.float32


def clip(a, d, lo, hi, t0, t1):
    """Intersect [t0, t1] with the slab lo <= a + t d <= hi (FP32, the kernel's operation order)."""
    if d == 0:
        return (t0, t1) if lo <= a <= hi else (f32(np.inf), f32(-np.inf))
    inv = f32(1) / d
    e0, e1 = (lo - a) * inv, (hi - a) * inv
    return max(t0, min(e0, e1)), min(t1, max(e0, e1))


def walk(a, b, R, G, Gz, ts, first=0, step=1):
    """Tiles (ix, iy, iz) visited for the segment a -> b (cell-index space), in visit order."""
    d = [f32(b[k] - a[k]) for k in range(3)]
    nt = [G // ts[0], G // ts[1], Gz // ts[2]]
    glo = [f32(-R)] * 3
    ghi = [f32(G - 1) + R, f32(G - 1) + R, f32(Gz - 1) + R]
    t0, t1 = f32(0), f32(1)
    for k in range(3):
        t0, t1 = clip(a[k], d[k], glo[k], ghi[k], t0, t1)
    if t0 > t1:
        return []
    A = 0
    if abs(d[1]) > abs(d[A]):
        A = 1
    if abs(d[2]) > abs(d[A]):
        A = 2
    B, C = (A + 1) % 3, (A + 2) % 3
    pa0, pa1 = a[A] + d[A] * t0, a[A] + d[A] * t1
    ta0 = max(int(np.floor((min(pa0, pa1) - R) / f32(ts[A]))), 0)
    ta1 = min(int(np.floor((max(pa0, pa1) + R) / f32(ts[A]))), nt[A] - 1)
    out = []
    for ta in range(ta0 + first, ta1 + 1, step):
        slo, shi = f32(ta * ts[A]) - R, f32(ta * ts[A] + ts[A] - 1) + R
        s0, s1 = clip(a[A], d[A], slo, shi, t0, t1)
        if s0 > s1:
            continue
        b0, b1 = a[B] + d[B] * s0, a[B] + d[B] * s1
        c0, c1 = a[C] + d[C] * s0, a[C] + d[C] * s1
        tb0 = max(int(np.floor((min(b0, b1) - R) / f32(ts[B]))), 0)
        tb1 = min(int(np.floor((max(b0, b1) + R) / f32(ts[B]))), nt[B] - 1)
        tc0 = max(int(np.floor((min(c0, c1) - R) / f32(ts[C]))), 0)
        tc1 = min(int(np.floor((max(c0, c1) + R) / f32(ts[C]))), nt[C] - 1)
        for tb in range(tb0, tb1 + 1):
            for tc in range(tc0, tc1 + 1):
                t = [0, 0, 0]
                t[A], t[B], t[C] = ta, tb, tc
                lo = [f32(t[k] * ts[k]) - R for k in range(3)]
                hi = [f32(t[k] * ts[k] + ts[k] - 1) + R for k in range(3)]
                u0, u1 = t0, t1
                for k in range(3):
                    u0, u1 = clip(a[k], d[k], lo[k], hi[k], u0, u1)
                if u0 <= u1:
                    out.append(tuple(t))
    return out


def seg_dist(p, a, d):
    dd = float(d @ d)
    t = np.clip(((p - a) @ d) / dd, 0.0, 1.0) if dd > 0 else np.zeros(len(p))
    return np.linalg.norm(p - (a + t[:, None] * d), axis=1)


def test_walk_covers_support_and_halves_split_it():
    rng = np.random.default_rng(7)
    G, Gz, ts = 64, 16, (16, 16, 4)
    R = f32(0.3 / 0.1 * (1 + 1e-4) + 1e-3)  # ls 0.3 m at 0.1 m cells, the binning radius
    ix, iy, iz = np.meshgrid(np.arange(G), np.arange(G), np.arange(Gz), indexing="ij")
    cells = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1).astype(np.float64)
    tile_of = np.stack([cells[:, 0] // ts[0], cells[:, 1] // ts[1], cells[:, 2] // ts[2]], 1).astype(int)
    sensor = np.array([G / 2 - 0.5, G / 2 - 0.5, Gz / 2 - 0.5], dtype=np.float32)
    checked = 0
    for r in range(120):
        if r % 4 == 0:  # axis-aligned and degenerate rays among them
            end = sensor.copy()
            end[r % 3] += f32(rng.uniform(-40, 40))
        else:
            end = (sensor + rng.uniform(-45, 45, 3).astype(np.float32) * np.array([1, 1, 0.3], np.float32))
        a = [f32(v) for v in sensor]
        b = [f32(v) for v in end]
        full = walk(a, b, R, G, Gz, ts)
        halves = [walk(a, b, R, G, Gz, ts, h, 2) for h in (0, 1)]
        assert len(set(full)) == len(full), "a tile visited twice"
        assert sorted(halves[0] + halves[1]) == sorted(full), "the two threads' walks differ from the full walk"
        assert not set(halves[0]) & set(halves[1])
        # brute force, a hair inside R so that FP32 rounding at the boundary does not decide
        near = seg_dist(cells, np.array(a, np.float64), np.array(b, np.float64) - np.array(a, np.float64))
        need = {tuple(t) for t in tile_of[near < float(R) - 1e-3]}
        assert need <= set(full), f"ray {r}: tiles within R not visited: {sorted(need - set(full))[:5]}"
        checked += len(need)
    assert checked > 500


def entries_bound(R, G, Gz, ts):
    """Tiles one ray can reach at most: the per-ray factor of the list capacity
    (evidence.cu: ray_entries_bound, restated)."""
    Rb = float(R) + 0.01
    nt = [G // ts[0], G // ts[1], Gz // ts[2]]
    worst = 0
    for A in range(3):
        per_slab = 1
        for k in (1, 2):
            o = (A + k) % 3
            per_slab *= min(math.ceil((ts[A] + 4.0 * Rb) / ts[o]) + 1, nt[o])
        worst = max(worst, per_slab * nt[A])
    return min(worst, nt[0] * nt[1] * nt[2])


def test_walk_stays_within_the_list_capacity():
    """The ray lists are sized by a per-ray bound on the tiles a walk visits (times the point
    slots); no ray's walk may exceed it, whatever its direction and length, for each tile shape."""
    rng = np.random.default_rng(11)
    G, Gz = 64, 32
    R = f32(0.3 / 0.1 * (1 + 1e-4) + 1e-3)
    for ts in ((16, 16, 4), (16, 16, 8), (8, 8, 4)):
        bound = entries_bound(R, G, Gz, ts)
        worst = 0
        for r in range(150):
            a = rng.uniform([0, 0, 0], [G, G, Gz]).astype(np.float32)
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            if r % 5 == 0:  # along an axis or a diagonal of the grid
                u = np.eye(3)[r % 3] if r % 2 else np.array([1.0, 1.0, 0.5]) / 1.5
            b = (a + u * rng.uniform(1, 2 * G)).astype(np.float32)
            n = len(walk([f32(v) for v in a], [f32(v) for v in b], R, G, Gz, ts))
            worst = max(worst, n)
            assert n <= bound, (ts, r, n, bound)
        assert worst > 0

"""The evidence kernels list each ray of a 16x16 tile's chunk under the 8x8-cell columns its binned
segment meets (k3dom_b200/csrc/evidence.cu: region_mask, stage_item_rays), and a sub-block then
culls only its column's rays. That is exact only if no ray that can reach a cell of a column is
left off the column's list. This restates the column test (FP32 slab intersection of the segment
with the column's cell-centre box grown by R) and checks it against brute force: every column
holding a cell centre within R of the segment is in the ray's mask. CPU only."""
import numpy as np

f32 = np.float32


def slab(a, d, lo, hi):
    if d == 0:
        inside = lo <= a <= hi
        return (f32(-np.inf), f32(np.inf)) if inside else (f32(np.inf), f32(-np.inf))
    inv = f32(1) / d
    e0, e1 = (lo - a) * inv, (hi - a) * inv
    return min(e0, e1), max(e0, e1)


def region_mask(a, d, x0, y0, z0, tz, R):
    zl, zh = slab(a[2], d[2], z0 - R, z0 + f32(tz - 1) + R)
    zl, zh = max(zl, f32(0)), min(zh, f32(1))
    xs = [slab(a[0], d[0], x0 + f32(8 * h) - R, x0 + f32(8 * h + 7) + R) for h in range(2)]
    ys = [slab(a[1], d[1], y0 + f32(8 * h) - R, y0 + f32(8 * h + 7) + R) for h in range(2)]
    q = 0
    for qy in range(2):
        for qx in range(2):
            if max(zl, xs[qx][0], ys[qy][0]) <= min(zh, xs[qx][1], ys[qy][1]):
                q |= 1 << (qx + 2 * qy)
    return q


def seg_dist(p, a, d):
    """Distance (FP64) from points p (n, 3) to the segment a + t d, t in [0, 1]."""
    dd = float(d @ d)
    t = np.clip(((p - a) @ d) / dd, 0.0, 1.0) if dd > 0 else np.zeros(len(p))
    return np.linalg.norm(p - (a + t[:, None] * d), axis=1)


def test_column_mask_keeps_every_reaching_ray():
    rng = np.random.default_rng(7)
    R_bin = 0.3 / 0.1 * (1 + 1e-4) + 1e-3  # binning radius in cells (ls 0.3 m at 0.1 m cells)
    R = f32(R_bin + 0.25)
    checked = hits = 0
    for _ in range(4000):
        tz = int(rng.choice([4, 8]))
        tile = np.array([rng.integers(0, 16) * 16, rng.integers(0, 16) * 16, rng.integers(0, 8) * tz], np.float64)
        a = (tile + rng.uniform(-40, 56, 3)).astype(f32)
        # segments ending in or near the tile, some axis-aligned (zero direction components)
        end = tile + rng.uniform(-6, 22, 3)
        d = (end.astype(f32) - a).astype(f32)
        if rng.random() < 0.15:
            d[rng.integers(0, 3)] = f32(0)
        m = region_mask(a, d, f32(tile[0]), f32(tile[1]), f32(tile[2]), tz, R)
        for qy in range(2):
            for qx in range(2):
                gx, gy, gz = np.meshgrid(np.arange(8) + tile[0] + 8 * qx, np.arange(8) + tile[1] + 8 * qy,
                                         np.arange(tz) + tile[2], indexing="ij")
                cells = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)
                reach = seg_dist(cells, a.astype(np.float64), d.astype(np.float64)).min() <= R_bin
                checked += 1
                if reach:
                    hits += 1
                    assert m >> (qx + 2 * qy) & 1, (a, d, tile, tz, qx, qy)
    assert checked == 16000 and hits > 1000

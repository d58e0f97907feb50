"""Resampling brackets (k3dom_b200/csrc/particles.cu: k_res_brackets) are found by a warp-wide
33-way search: 32 probes per step, then one last window of at most 32 entries. The cumulative
weights are an exactly rounded prefix of non-negative weights, hence non-decreasing, and every
draw is at most the replaced last entry (resampling.cu:58-63), so "acc[j] >= u" is false then true
along the whole array even where the replaced last entry drops below its neighbour. This restates
the search and checks it against a linear scan (the reference's lower_bound, resampling.cu:66-67),
with probes kept inside the current window. CPU only."""
import numpy as np


def warp_lower(acc, u):
    lo, hi = 0, len(acc)
    while hi - lo > 32:
        span = hi - lo
        pos = [lo + ((l + 1) * span) // 33 for l in range(32)]
        assert all(lo <= p < hi for p in pos) and all(p < q for p, q in zip(pos, pos[1:]))
        m = [acc[p] >= u for p in pos]
        f = m.index(True) if any(m) else 32
        if f < 32:
            hi = pos[f]
        if f > 0:
            lo = pos[f - 1] + 1
    for l in range(32):
        if lo + l < hi and acc[lo + l] >= u:
            return lo + l
    return hi


def test_warp_search_equals_lower_bound():
    rng = np.random.default_rng(11)
    for t in range(1500):
        n = int(rng.integers(1, 5000)) if t % 3 else int(rng.integers(1, 70))
        w = rng.random(n) * (rng.random(n) < 0.7)  # runs of zero weights make equal entries
        acc = np.cumsum(w).astype(np.float32)
        jmax = acc[-1]
        draws = (rng.random(6) * jmax).astype(np.float32)
        umax = draws.max()
        if umax != acc[-1]:
            acc[-1] = umax  # the reference's replacement of the last entry
        acc = list(acc)
        for u in list(draws) + [umax]:
            ref = next((j for j in range(n) if acc[j] >= u), n)
            assert warp_lower(acc, u) == ref, (t, n)

"""The particle sort (onesweep radix sort with decoupled look-back, csrc/onesweep.cu) through the
C ABI: stable permutations against the oracle's stable argsort, and its bounded waits.

A look-back wait that runs out must end the frame with K3DOM_ERR_TIMEOUT and leave the handle
usable. The test makes a wait run out without any fault: k3dom_set_sort_wait keeps one tile of
the first pass from publishing its counts (a flag that nothing sets), so every later tile's
wait ends at its poll limit.
"""
import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import _native as N
from k3dom_b200 import scene
from oracle import binding as O

pytestmark = pytest.mark.gpu


def make_dom(P, G=32, Gz=8):
    cfg = scene.small(seed=19, G=G, Gz=Gz, res=0.2, P=P, B=max(P // 4, 1), n_points=1500)
    cfg.params["seed"] = 77
    p = K.make_params("k3dom", **cfg.params)
    return cfg, K.DOM(p, "k3dom")


def frame(cfg, dom, f):
    t = 0.1 + 0.1 * f
    s, pts = cfg.scene.scan(f, t, cfg.n_points)
    dom.updatePose(*s)
    dom.updateGrid(t, pts)


def test_sort_wait_timeout_is_reported_and_the_handle_recovers():
    cfg, dom = make_dom(65536)  # 16 tiles of 4,096 keys
    try:
        frame(cfg, dom, 0)
        frame(cfg, dom, 1)
        dom.set_sort_wait(max_polls=256, skip_tile=3)
        with pytest.raises(N.K3domError) as ei:
            frame(cfg, dom, 2)
        assert ei.value.status == 6, ei.value  # K3DOM_ERR_TIMEOUT
        dom.set_sort_wait()  # normal waits again
        frame(cfg, dom, 3)
        # the next sort is whole again: a stage-by-stage frame sorts exactly like the oracle
        t = 0.1 + 0.1 * 4
        s, pts = cfg.scene.scan(4, t, cfg.n_points)
        dom.updatePose(*s)
        dt = float(np.float32(t) - np.float32(0.1 + 0.1 * 3))
        dom.particlePrediction(dt)
        cells = dom.get_particles("persistent")["cell"]
        dom.particleAssignment()
        perm, sk, st, en = O.assign(cells, dom.grid_cell_count)
        np.testing.assert_array_equal(dom.sort_permutation(), perm)
        np.testing.assert_array_equal(dom.get_particles("sorted")["cell"], sk)
        rs, re = dom.get_cell_ranges()
        np.testing.assert_array_equal(rs, st)
        np.testing.assert_array_equal(re, en)
    finally:
        dom.close()


@pytest.mark.parametrize("P,G,Gz", [(1000, 32, 8), (4095, 32, 8), (4096, 32, 8), (4097, 32, 8),
                                    (262144 + 123, 32, 8), (262144 + 123, 64, 16)])
def test_sort_sizes_and_ragged_tiles(P, G, Gz):
    """Particle counts around the 4,096-key tile (one key, a partial tile, exact tiles, one more)
    and a large ragged count: permutation, sorted keys and cell ranges equal the oracle's. The
    32x32x8 grid's 13-bit keys take passes of 7 and 6 bits, the 64x64x16 grid's 16-bit keys two of
    8 bits (the widest digit)."""
    cfg, dom = make_dom(P, G, Gz)
    try:
        frame(cfg, dom, 0)
        rng = np.random.default_rng(P)
        a = dom.get_particles("persistent")
        C_ = dom.grid_cell_count
        # crowded and sparse cells, many equal keys (stability), keys up to the last cell
        cells = np.where(rng.uniform(size=P) < 0.5, rng.integers(0, 8, P), rng.integers(0, C_, P)).astype(np.int32)
        cells[-1] = C_ - 1
        G = dom.grid_size
        pos = np.stack([cells % G, (cells // G) % G, cells // (G * G)], 1).astype(np.float32) + 0.5
        dom.set_particles("persistent", pos=pos, vel=np.zeros_like(pos), cell=cells,
                          weight=np.full(P, 1.0 / P, np.float32))
        dom.particlePrediction(0.0)  # zero noise at dt = 0 keeps the cells (noise 0.01 m < half a cell)
        keys = dom.get_particles("persistent")["cell"]
        dom.particleAssignment()
        perm, sk, st, en = O.assign(keys, C_)
        np.testing.assert_array_equal(dom.sort_permutation(), perm)
        np.testing.assert_array_equal(dom.get_particles("sorted")["cell"], sk)
        rs, re = dom.get_cell_ranges()
        np.testing.assert_array_equal(rs, st)
        np.testing.assert_array_equal(re, en)
    finally:
        dom.close()

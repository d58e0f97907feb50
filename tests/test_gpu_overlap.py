"""Stage overlap of the steady frame: with stage timing off, a K3DOM frame accumulates the
evidence beside prediction and assignment and updates the cells in a pass of its own; with
timing on, every stage runs in order and the evidence kernel updates each tile's cells itself.
Both must give the same bits (the evidence sums are exact, and the cell update is one function
of the same inputs), frame after frame, including frames with a map shift, and for the DS
variant (whose evidence pass follows assignment either way).
"""
import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import scene

pytestmark = pytest.mark.gpu

FIELDS = ["free_mass", "static_mass", "dynamic_mass", "occ_mass", "pers_mass", "pred_mass", "born_mass",
          "mean_x_vel", "mean_y_vel", "mean_z_vel", "mu_UA", "w_UA", "meas_occ", "meas_free", "del_occ",
          "del_free"]


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
@pytest.mark.parametrize("G,Gz,P,B,n,ego", [(32, 8, 8192, 2048, 1500, 2.5), (64, 16, 65536, 16384, 6000, 1.2)])
def test_overlapped_frame_equals_ordered_frame(variant, G, Gz, P, B, n, ego):
    cfg = scene.small(seed=11, variant=variant, G=G, Gz=Gz, res=0.2, P=P, B=B, n_points=n, ego=ego)
    cfg.params["seed"] = 77
    p = K.make_params(variant, **cfg.params)
    ordered, overlapped = K.DOM(p, variant), K.DOM(p, variant)
    try:
        ordered.set_timing(True)
        for f in range(8):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, n)
            for d in (ordered, overlapped):
                d.updatePose(*s)
                d.updateGrid(t, pts)
            for k in FIELDS:
                a, b = ordered.get_cell_field(k), overlapped.get_cell_field(k)
                assert np.array_equal(a, b, equal_nan=True), f"frame {f}: {k} differs"
            ra, rb = ordered.get_particles("persistent"), overlapped.get_particles("persistent")
            for k in ra:
                assert np.array_equal(ra[k], rb[k], equal_nan=True), f"frame {f}: particles {k} differ"
            assert ordered.info().center_x == overlapped.info().center_x
    finally:
        ordered.close()
        overlapped.close()


def test_placed_and_sorted_ray_lists_agree():
    """K3DOM ray lists are placed per tile (order within a tile arbitrary) up to 12,288 tiles and
    sorted by tile beyond; the evidence sums are exact, so a tiling on each side of that line
    gives the same frames bit for bit. 256 x 256 x 64 voxels: 16x16x4 tiles (4,096, placed)
    against 8x8x4 tiles (16,384, sorted)."""
    cfg = scene.small(seed=3, variant="k3dom", G=256, Gz=64, res=0.1, P=65536, B=16384, n_points=20000, ego=1.2)
    cfg.params["seed"] = 21
    p = K.make_params("k3dom", **cfg.params)
    placed, sorted_ = K.DOM(p, "k3dom"), K.DOM(p, "k3dom")
    try:
        for f in range(4):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            for d in (placed, sorted_):
                d.updatePose(*s)
                d.updateGrid(t, pts)
            if f == 0:
                placed.set_tuning(2, 512)
                sorted_.set_tuning(1, 256)
        assert placed.tuning()["tile_rule"] == 2 and sorted_.tuning()["tile_rule"] == 1
        for k in FIELDS:
            a, b = placed.get_cell_field(k), sorted_.get_cell_field(k)
            assert np.array_equal(a, b, equal_nan=True), k
        assert (placed.get_cell_field("del_free") > 0).sum() > 10000
    finally:
        placed.close()
        sorted_.close()

"""Batched update (k3dom_batch_*): every scene of a batch must produce exactly the bits the same
scene produces in a handle of its own.

Scenes differ in grid size, particle and birth counts, point counts, seeds and ego motion (so
map shifts happen in some scenes and not in others). After every frame all cell fields, the
persistent particle set, the sort permutation, the cell ranges and the resampling ancestors of
each scene are compared with np.array_equal. The evidence tiling is changed by the autotuner
in the middle of one run: results must not depend on it.
"""
import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import scene

pytestmark = pytest.mark.gpu

FIELDS = ["free_mass", "static_mass", "dynamic_mass", "occ_mass", "pers_mass", "pred_mass", "born_mass",
          "mean_x_vel", "mean_y_vel", "mean_z_vel", "mu_UA", "w_UA", "meas_occ", "meas_free", "del_occ",
          "del_free"]


def scenes(variant):
    specs = [
        dict(seed=3, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500, ego=0.0),
        dict(seed=4, G=24, Gz=6, res=0.2, P=4096, B=1024, n_points=900, ego=2.5),
        dict(seed=5, G=40, Gz=10, res=0.2, P=16384, B=4096, n_points=2600, ego=1.2),
    ]
    out = []
    for k, s in enumerate(specs):
        cfg = scene.small(seed=s["seed"], variant=variant, G=s["G"], Gz=s["Gz"], res=s["res"], P=s["P"], B=s["B"],
                          n_points=s["n_points"], ego=s["ego"])
        cfg.params["seed"] = 100 + k
        out.append(cfg)
    return out


def frame_inputs(cfgs, f):
    t = 0.1 + 0.1 * f
    poses, pts = [], []
    for cfg in cfgs:
        s, p = cfg.scene.scan(f, t, cfg.n_points - 7 * f)  # point counts change per frame
        poses.append(s)
        pts.append(p)
    return t, poses, pts


def snapshot(d):
    snap = {k: d.get_cell_field(k) for k in FIELDS}
    snap["ranges"] = d.get_cell_ranges()
    snap["particles"] = d.get_particles("persistent")
    snap["info"] = (d.info().center_x, d.info().center_y, d.info().frame_index)
    return snap


def assert_same(a, b, where):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k], equal_nan=True), f"{where}: {k} differs"
    for i in range(2):
        assert np.array_equal(a["ranges"][i], b["ranges"][i]), f"{where}: cell ranges differ"
    for k in ("pos", "vel", "weight", "cell", "associated"):
        assert np.array_equal(a["particles"][k], b["particles"][k]), f"{where}: particles.{k} differs"
    assert a["info"] == b["info"], where


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
def test_batch_equals_separate_scenes(variant):
    cfgs = scenes(variant)
    params = [K.make_params(variant, **c.params) for c in cfgs]
    plain = [K.DOM(p, variant) for p in params]
    batch = K.BatchDOM(params, variant)
    try:
        for f in range(5):
            t, poses, pts = frame_inputs(cfgs, f)
            for s, d in enumerate(plain):
                d.updatePose(*poses[s])
                d.updateGrid(t, pts[s])
                batch.updatePose(s, *poses[s])
            batch.update([t] * len(cfgs), pts)
            for s, d in enumerate(plain):
                assert_same(snapshot(batch.scene(s)), snapshot(d), f"{variant} frame {f} scene {s}")
                if f > 0:
                    assert np.array_equal(batch.scene(s).ancestors(), d.ancestors()), f"ancestors f{f} s{s}"
                    assert np.array_equal(batch.scene(s).sort_permutation(), d.sort_permutation())
                    jb, bb, mb = batch.scene(s).resampling_state()
                    jp, bp, mp = d.resampling_state()
                    assert np.array_equal(jb, jp) and np.array_equal(bb, bp) and mb == mp
    finally:
        batch.close()
        for d in plain:
            d.close()


@pytest.mark.parametrize("device_points", [False, True])
def test_batch_autotune_keeps_results(device_points):
    """The autotuner measures every (tile rule, chunk) candidate on live frames; the results
    must equal the untuned single-scene handles frame by frame. With scans in device memory the
    candidates that re-lay out the evidence buffers re-stage the frame's points device to device,
    which must be ordered after the new buffers' zero-fill."""
    import torch
    variant = "k3dom"
    cfgs = scenes(variant)
    params = [K.make_params(variant, **c.params) for c in cfgs]
    plain = [K.DOM(p, variant) for p in params]
    batch = K.BatchDOM(params, variant)
    try:
        n_frames = 2 + batch.tuning()["candidates"] + 2
        for f in range(n_frames):
            if f == 1:
                batch.autotune(True)
            t, poses, pts = frame_inputs(cfgs, f)
            for s, d in enumerate(plain):
                d.updatePose(*poses[s])
                d.updateGrid(t, pts[s])
                batch.updatePose(s, *poses[s])
            if device_points:
                batch.update([t] * len(cfgs), [torch.from_numpy(x).cuda() for x in pts])
            else:
                batch.update([t] * len(cfgs), pts)
            for s, d in enumerate(plain):
                assert_same(snapshot(batch.scene(s)), snapshot(d), f"tuned frame {f} scene {s}")
        tu = batch.tuning()
        assert tu["tuned"] == 1 and tu["tuning"] == 0
        assert all(ms > 0 for ms in tu["candidate_ms"])
        # candidate k is (rule k % 4, chunk (512, 1024)[k // 4])
        assert tu["candidate_ms"][tu["tile_rule"] + 4 * [512, 1024].index(tu["chunk"])] == pytest.approx(
            tu["best_ms"])
    finally:
        batch.close()
        for d in plain:
            d.close()


def test_plain_tiling_does_not_change_results():
    """Every tile rule and chunk gives bit-identical frames on one scene (fixed-point evidence)."""
    cfg = scenes("k3dom")[2]
    p = K.make_params("k3dom", **cfg.params)
    runs = []
    for rule, chunk in [(0, 1024), (1, 512), (2, 1024), (3, 64)]:
        d = K.DOM(p, "k3dom")
        d.set_tuning(rule, chunk)
        for f in range(3):
            t, poses, pts = frame_inputs([cfg], f)
            d.updatePose(*poses[0])
            d.updateGrid(t, pts[0])
        runs.append(snapshot(d))
        d.close()
    for r in runs[1:]:
        assert_same(r, runs[0], "tiling")


def test_batch_rejects_bad_arguments():
    cfgs = scenes("k3dom")[:2]
    params = [K.make_params("k3dom", **c.params) for c in cfgs]
    batch = K.BatchDOM(params, "k3dom")
    try:
        with pytest.raises(K.dom.N.K3domError):
            batch.updatePose(5, 0.0, 0.0, 0.0)
        with pytest.raises(ValueError):
            batch.update([0.1], [np.zeros((3, 3), np.float32)])
        # the plain single-scene update is refused on a batch of two
        with pytest.raises(K.dom.N.K3domError):
            batch.scene(0).updateGrid(0.1, np.zeros((3, 3), np.float32))
    finally:
        batch.close()


def test_config3_batch_equals_separate_scenes():
    """The batched benchmark workload at its own size: the 16 uneven config3 scenes (grids of
    64-256 cells, 2^18-2^22 particles, 10k-200k points) stepped together by one BatchDOM give,
    scene by scene, the bits that each scene gives alone."""
    cfgs = scene.config3(seed=0)
    assert len(cfgs) == 16
    params = [K.make_params("k3dom", **c.params) for c in cfgs]
    plain = [K.DOM(p, "k3dom") for p in params]
    batch = K.BatchDOM(params, "k3dom")
    try:
        for f in range(3):
            ts, pts = [], []
            for s, (c, d) in enumerate(zip(cfgs, plain)):
                t = 0.1 + f * c.dt
                pose, p = c.scene.scan(f, t, c.n_points)
                d.updatePose(*pose)
                d.updateGrid(t, p)
                batch.updatePose(s, *pose)
                ts.append(t)
                pts.append(p)
            batch.update(ts, pts)
        for s, d in enumerate(plain):
            assert_same(snapshot(batch.scene(s)), snapshot(d), f"config3 scene {s}")
            assert np.array_equal(batch.scene(s).ancestors(), d.ancestors()), f"ancestors scene {s}"
    finally:
        batch.close()
        for d in plain:
            d.close()

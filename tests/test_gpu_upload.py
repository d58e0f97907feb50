"""Point upload routes of k3dom_update_grid: an interleaved (N, 3) scan in pageable host memory
(staged through pinned memory), in pinned host memory (read in place by the synchronous call,
staged by the asynchronous one), in device memory (de-interleaved on the device), and three
separate coordinate arrays. Every route must give bit-identical frames."""
import numpy as np
import pytest
import torch

import k3dom_b200 as K
from k3dom_b200 import scene

pytestmark = pytest.mark.gpu

FIELDS = ["free_mass", "static_mass", "dynamic_mass", "pers_mass", "born_mass", "mean_x_vel", "del_occ", "del_free"]


def test_upload_routes_agree():
    cfg = scene.small(seed=21, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    p = K.make_params("k3dom", **cfg.params)
    routes = ["pageable", "pinned", "pinned_async", "device", "planes"]
    doms = {r: K.DOM(p) for r in routes}
    try:
        for f in range(4):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            pts = np.ascontiguousarray(pts, np.float32)
            pinned = torch.from_numpy(pts.copy()).pin_memory()
            for r, d in doms.items():
                d.updatePose(*s)
                if r == "pageable":
                    d.updateGrid(t, pts)
                elif r == "pinned":
                    d.updateGrid(t, pinned.numpy())
                elif r == "pinned_async":
                    d.updateGridAsync(t, pinned.numpy())
                    d.synchronize()
                elif r == "device":
                    d.updateGrid(t, pinned.to("cuda:0"))
                else:
                    d.updateGrid(t, pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy())
            ref = doms["pageable"]
            for r in routes[1:]:
                for fld in FIELDS:
                    np.testing.assert_array_equal(doms[r].get_cell_field(fld), ref.get_cell_field(fld),
                                                  err_msg=f"frame {f} route {r} field {fld}")
    finally:
        for d in doms.values():
            d.close()


@pytest.mark.parametrize("graph", [True, False])
def test_registered_output_equals_readback(graph):
    """k3dom_set_output: every frame writes the field into pinned host or device memory as part of
    the frame; after k3dom_update_grid returns it equals what k3dom_get_cell_field reads back.
    Mass fields are exported after the cell update, w_UA after the births' scan."""
    cfg = scene.small(seed=23, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    p = K.make_params("k3dom", **cfg.params)
    d = K.DOM(p)
    try:
        d.set_graph_mode(graph)
        n = d.grid_cell_count
        with pytest.raises(K.dom.N.K3domError):
            d.set_output("occ_mean", np.zeros(n, np.float32))  # pageable host memory is refused
        for f, field in enumerate(["occ_mean", "occ_mean", "w_UA", "w_UA", "dynamic_mass", "occ_mean"]):
            host = torch.full((n,), -7.0, dtype=torch.float32).pin_memory()
            dev = torch.full((n,), -7.0, dtype=torch.float32, device="cuda:0")
            out = host if f % 2 == 0 else dev
            d.set_output(field, out)
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            d.updatePose(*s)
            d.updateGrid(t, pts)
            got = out.cpu().numpy() if out.is_cuda else out.numpy()
            np.testing.assert_array_equal(got, d.get_cell_field(field), err_msg=f"frame {f} {field}")
        d.set_output(None)
        s, pts = cfg.scene.scan(9, 1.0, cfg.n_points)
        d.updatePose(*s)
        d.updateGrid(1.0, pts)  # no output registered: the frame runs without the export
    finally:
        d.close()


@pytest.mark.parametrize("pinned", [False, True])
def test_nonfinite_host_scan_is_refused_without_side_effects(pinned):
    """A host scan with a non-finite coordinate is refused (K3DOM_ERR_INVALID_INPUT) before the
    frame runs; the handle then continues exactly as one that never saw the refused call."""
    cfg = scene.small(seed=29, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    p = K.make_params("k3dom", **cfg.params)
    a, b = K.DOM(p), K.DOM(p)
    try:
        for f in range(4):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            pts = np.ascontiguousarray(pts, np.float32)
            if f == 2:
                bad = pts.copy()
                bad[777, 1] = np.nan
                if pinned:
                    bad = torch.from_numpy(bad).pin_memory().numpy()
                a.updatePose(*s)
                with pytest.raises(K.dom.N.K3domError) as e:
                    a.updateGrid(t, bad)
                assert e.value.status == 8  # K3DOM_ERR_INVALID_INPUT
            for d in (a, b):
                d.updatePose(*s)
                d.updateGrid(t, pts)
        for fld in FIELDS:
            np.testing.assert_array_equal(a.get_cell_field(fld), b.get_cell_field(fld), err_msg=fld)
    finally:
        a.close()
        b.close()


def test_nonfinite_device_points_are_skipped_per_frame():
    """Device scans may hold non-finite coordinates: those points are skipped (they take no
    evidence, as in the reference, whose comparisons with NaN fail) and counted for the frame.
    The frame equals the same scan without them."""
    cfg = scene.small(seed=31, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    p = K.make_params("k3dom", **cfg.params)
    a, b = K.DOM(p), K.DOM(p)
    try:
        for f in range(3):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            pts = np.ascontiguousarray(pts, np.float32)
            bad = pts.copy()
            bad[[5, 500, 1000], [0, 1, 2]] = [np.nan, np.inf, -np.inf]
            keep = np.ones(len(pts), bool)
            keep[[5, 500, 1000]] = False
            a.updatePose(*s)
            a.updateGrid(t, torch.from_numpy(bad if f == 1 else pts).to("cuda:0"))
            b.updatePose(*s)
            b.updateGrid(t, torch.from_numpy(pts[keep] if f == 1 else pts).to("cuda:0"))
            assert a.diagnostics()["nonfinite_points"] == (3 if f == 1 else 0)
            for fld in FIELDS:
                np.testing.assert_array_equal(a.get_cell_field(fld), b.get_cell_field(fld), err_msg=f"{f} {fld}")
    finally:
        a.close()
        b.close()

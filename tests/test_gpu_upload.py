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

"""Point-cloud transform on the device (k3dom_set_point_transform): the node rotates each scan from
the lidar frame into the map-aligned frame on the host (k3dom_node.cpp:73-83); here the rotation
(and an optional translation) is applied on the GPU where the points are read. A scan given in the
lidar frame with the transform set must give exactly the frames that the same scan, transformed
on the host in the same FP32 order, gives without it."""
import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import scene

pytestmark = pytest.mark.gpu

FIELDS = ["free_mass", "static_mass", "dynamic_mass", "pers_mass", "born_mass", "mean_x_vel", "del_occ", "del_free"]


def host_transform(R, t, q):
    """((R0 x + R1 y) + R2 z) + t per row, each operation rounded to float32 (no fused multiply-add)."""
    R = R.astype(np.float32)
    t = t.astype(np.float32)
    x, y, z = (q[:, k].astype(np.float32) for k in range(3))
    rows = [((R[i, 0] * x + R[i, 1] * y) + R[i, 2] * z) + t[i] for i in range(3)]
    return np.stack(rows, axis=1).astype(np.float32)


@pytest.mark.parametrize("variant", ["k3dom", "dsphdmib"])
def test_device_transform_equals_host_transform(variant):
    cfg = scene.small(seed=11, variant=variant, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    p = K.make_params(variant, **cfg.params)
    R = K.rotation_from_quaternion(0.05, -0.02, 0.38, 0.92)
    t = np.array([0.01, -0.02, 0.005], np.float32)
    a, b = K.DOM(p, variant), K.DOM(p, variant)
    try:
        for f in range(4):
            tt = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, tt, cfg.n_points)
            # the scan in the lidar frame: q = R^T (p - t)
            q = ((pts.astype(np.float64) - t) @ R.astype(np.float64)).astype(np.float32)
            a.set_point_transform(R, t)
            a.updatePose(*s)
            a.updateGrid(tt, q)
            b.updatePose(*s)
            b.updateGrid(tt, host_transform(R, t, q))
            for k in FIELDS:
                assert np.array_equal(a.get_cell_field(k), b.get_cell_field(k)), (f, k)
            pa, pb = a.get_particles(), b.get_particles()
            for k in ("pos", "vel", "weight", "cell"):
                assert np.array_equal(pa[k], pb[k]), (f, k)
        # switched off: points are used as given again
        a.set_point_transform(None)
        s, pts = cfg.scene.scan(9, 0.5, cfg.n_points)
        for d in (a, b):
            d.updatePose(*s)
            d.updateGrid(0.5, pts)
        assert np.array_equal(a.get_cell_field("free_mass"), b.get_cell_field("free_mass"))
    finally:
        a.close()
        b.close()


def test_transform_rejects_non_finite():
    cfg = scene.small(seed=1)
    d = K.DOM(K.make_params("k3dom", **cfg.params), "k3dom")
    try:
        R = np.eye(3, dtype=np.float32)
        R[1, 1] = np.nan
        with pytest.raises(K.dom.N.K3domError):
            d.set_point_transform(R)
    finally:
        d.close()

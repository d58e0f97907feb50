"""The FP64 reference of the differentiable update (oracle/k3dom_calib_oracle.c): 3-D DDA labels on
hand-worked rays, and the dual-number gradient against FP64 central finite differences.

These pin the oracle that the GPU adjoint is checked against (tests/test_gpu_calib.py)."""
import numpy as np
import pytest

from k3dom_b200 import scene
from oracle import binding as O


def labels(G, Gz, res, sensor, pts):
    n0 = np.zeros(G * G * Gz, np.uint32)
    n1 = np.zeros(G * G * Gz, np.uint32)
    p = np.ascontiguousarray(pts, np.float32).reshape(-1)
    O.oracle().orc_dda_labels(G, Gz, res, *[float(v) for v in sensor], p.size // 3, p, n0, n1)
    return n0, n1


def idx(G, x, y, z):
    return x + G * y + G * G * z


def test_dda_axis_ray():
    # cell i spans [i, i + 1) in X = x / res + G / 2: sensor at X = 0.5, hit at X = 3.5
    G, Gz = 4, 2
    n0, n1 = labels(G, Gz, 1.0, (-1.5, -1.5, -0.5), [[3.0, 0.0, 0.0]])
    assert [idx(G, i, 0, 0) for i in range(3)] == list(np.nonzero(n0)[0])
    assert list(np.nonzero(n1)[0]) == [idx(G, 3, 0, 0)]


def test_dda_diagonal_and_clipping():
    G, Gz = 8, 4
    # 45 degrees in x-y from the centre of cell (0, 0): equal tMax -> x steps first
    n0, n1 = labels(G, Gz, 1.0, (-3.5, -3.5, -1.5), [[2.0, 2.0, 0.0]])
    got = [int(i) for i in np.nonzero(n0)[0]]
    want = sorted([idx(G, 0, 0, 0), idx(G, 1, 0, 0), idx(G, 1, 1, 0), idx(G, 2, 1, 0)])
    assert got == want
    assert [int(i) for i in np.nonzero(n1)[0]] == [idx(G, 2, 2, 0)]
    # a hit outside the grid: free labels up to the border, no hit label
    n0, n1 = labels(G, Gz, 1.0, (-3.5, -3.5, -1.5), [[20.0, 0.0, 0.0]])
    assert n1.sum() == 0
    assert [int(i) for i in np.nonzero(n0)[0]] == [idx(G, i, 0, 0) for i in range(8)]
    # a sensor outside the grid looking in
    n0, n1 = labels(G, Gz, 1.0, (-6.5, -3.5, -1.5), [[4.0, 0.0, 0.0]])
    assert [int(i) for i in np.nonzero(n0)[0]] == [idx(G, i, 0, 0) for i in range(1)]
    assert [int(i) for i in np.nonzero(n1)[0]] == [idx(G, 1, 0, 0)]


def small_problem(seed=7, G=20, Gz=6):
    cfg = scene.small(seed=seed, G=G, Gz=Gz, res=0.2, n_points=600, n_moving=2)
    res = np.float32(0.2)
    oc = O.OracleCalib(G, Gz, float(res), 2.5)
    rng = np.random.default_rng(seed)
    for k in range(2):
        t = 0.1 + 0.1 * k
        s, pts = cfg.scene.scan(k, t, cfg.n_points)
        dyn = None
        if k > 0:
            dyn = np.where(rng.random(G * G * Gz) < 0.05, rng.uniform(0.0, 0.02, G * G * Gz), 0.0).astype(np.float32)
        oc.add_frame(0.0 if k == 0 else 0.1, np.zeros(3, np.float32), pts, dyn)
    for k in range(3):
        s, pts = cfg.scene.scan(50 + k, 0.2, 500, sensor_offset=rng.uniform(-0.3, 0.3, 3) * [1, 1, 0.2],
                                az_offset=float(rng.uniform(0, 6.28)))
        oc.add_heldout(s.astype(np.float32), pts)
    return oc


# The calibration's initial theta with the prescribed step 1e-4; a second theta with a free prior
# of 0.002, where a 1e-4 step (5 % of the parameter) straddles min/max kinks, with step 1e-6.
@pytest.mark.parametrize("theta,h", [((0.3, 1.0, 0.1, 0.01, 0.01), 1e-4), ((0.45, 0.4, 0.6, 0.05, 0.002), 1e-6)])
def test_dual_gradient_matches_central_differences(theta, h):
    oc = small_problem()
    assert oc.n0.sum() > 0 and oc.n1.sum() > 0
    loss, g = oc.loss_grad(theta)
    fd = oc.fd_grad(theta, h=h)
    assert np.isfinite(loss) and loss > 0
    scale = np.abs(g).max()
    # central differences carry O(h^2) truncation and a few cells crossing a kink of min/max
    np.testing.assert_allclose(g, fd, rtol=2e-3, atol=2e-4 * scale)


def test_loss_is_mean_bce_of_occupancy():
    oc = small_problem(seed=3)
    theta = (0.3, 1.0, 0.1, 0.01, 0.01)
    p = np.clip(oc.occupancy(theta), 1e-7, 1 - 1e-7)
    n0, n1 = oc.n0.astype(np.float64), oc.n1.astype(np.float64)
    want = (-(n1 * np.log(p)) - n0 * np.log(1 - p)).sum() / (n0.sum() + n1.sum())
    loss, _ = oc.loss_grad(theta, want_grad=False)
    assert loss == pytest.approx(want, rel=1e-12)

"""The differentiable kernel-inference update on the GPU (k3dom_bgki_forward / k3dom_bgki_backward)
against the FP64 oracle (oracle/k3dom_calib_oracle.c, pinned by tests/test_calib_oracle.py).

Bars
  * held-out labels (3-D DDA counts per cell): bit-exact;
  * per-cell kernel sums sum f(d/ls): 1e-5 relative (floor 1e-3 of the largest sum);
    derivative sums sum -x f'(x): 2e-5 of the largest |sum| (FP32 pair distances and tables);
  * occupancy and loss: 1e-5 relative;
  * gradient: within 1e-4 relative (plus 1e-4 of the largest component) of the FP64 dual-number
    gradient, and within 2e-3 (plus 2e-4 of the largest component) of FP64 central finite
    differences with step 1e-4.
"""
import numpy as np
import pytest

from k3dom_b200 import calib, scene
from oracle import binding as O

pytestmark = pytest.mark.gpu


def make(scale="config0", seed=0):
    cfg = scene.config4(seed=seed, scale=scale)
    pr = calib.build_problem(cfg)
    G, Gz, res, ms = pr.grid
    oc = O.OracleCalib(G, Gz, res, ms)
    for dt, rel, pts, dyn in pr.frames:
        oc.add_frame(dt, rel, pts, dyn)
    for rel, pts in pr.heldout:
        oc.add_heldout(rel, pts)
    return pr, oc


@pytest.fixture(scope="module")
def config4():
    pr, oc = make()
    yield pr, oc
    pr.close()


def test_labels_bit_exact(config4):
    pr, oc = config4
    n0, n1 = pr.calib.label_counts()
    assert n1.sum() > 1000 and n0.sum() > 10000
    assert np.array_equal(n0, oc.n0)
    assert np.array_equal(n1, oc.n1)


def test_kernel_sums(config4):
    pr, oc = config4
    ls = pr.theta0[0]
    want = oc.sums(ls)
    for k in range(len(pr.frames)):
        got = pr.calib.sums(ls, k)
        for q in (0, 1):
            w, g = want[k, q], got[q]
            floor = 1e-3 * np.abs(w).max()
            assert np.all(np.abs(g - w) <= 1e-5 * np.maximum(np.abs(w), floor)), (k, q)
        for q in (2, 3):
            w, g = want[k, q], got[q]
            assert np.abs(g - w).max() <= 2e-5 * np.abs(w).max(), (k, q)


def test_occupancy_and_loss(config4):
    pr, oc = config4
    th = pr.theta0
    p_gpu = pr.calib.occupancy(th).astype(np.float64)
    p_ref = oc.occupancy(th)
    assert np.abs(p_gpu - p_ref).max() <= 1e-5 * max(1.0, np.abs(p_ref).max())
    loss_ref, _ = oc.loss_grad(th, want_grad=False)
    assert pr.calib.loss(th) == pytest.approx(loss_ref, rel=1e-5)


@pytest.mark.parametrize("theta", [None, (0.36, 0.7, 0.3, 0.02, 0.015)])
def test_gradient_vs_fp64_reference_and_finite_differences(config4, theta):
    pr, oc = config4
    th = pr.theta0 if theta is None else theta
    loss, g = pr.calib.loss_and_grad(th)
    loss_ref, g_ref = oc.loss_grad(th)
    assert loss == pytest.approx(loss_ref, rel=1e-5)
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(g, g_ref, rtol=1e-4, atol=1e-4 * scale)
    fd = oc.fd_grad(th, h=1e-4)
    np.testing.assert_allclose(g, fd, rtol=2e-3, atol=2e-4 * scale)


def test_autograd_function(config4):
    import torch
    pr, _ = config4
    theta = torch.tensor(pr.theta0, dtype=torch.float32, requires_grad=True)
    loss = calib.calibration_loss(theta, pr.calib)
    loss.backward()
    _, g = pr.calib.loss_and_grad(pr.theta0)
    np.testing.assert_allclose(theta.grad.numpy(), g, rtol=1e-6, atol=0)
    # a small step against the gradient lowers the loss
    with torch.no_grad():
        step = theta - 1e-3 * theta.grad / theta.grad.norm() * theta.abs().min()
    assert pr.calib.loss(step.numpy()) < float(loss)


def test_gradient_at_config1_scale():
    """The same checks on config1's grid (256 x 256 x 32) and 120,000-point scans against the
    FP64 dual-number gradient."""
    pr, oc = make("config1")
    try:
        th = pr.theta0
        loss, g = pr.calib.loss_and_grad(th)
        loss_ref, g_ref = oc.loss_grad(th)
        assert loss == pytest.approx(loss_ref, rel=1e-5)
        np.testing.assert_allclose(g, g_ref, rtol=1e-4, atol=1e-4 * np.abs(g_ref).max())
    finally:
        pr.close()

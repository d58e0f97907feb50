"""The differentiable kernel-inference update (k3dom_calib_* / k3dom_bgki_forward / k3dom_bgki_backward
in include/k3dom_b200.h) and its torch.autograd.Function.

    problem = build_problem(scene.config4())          # training frames + held-out labels
    theta = torch.tensor(problem.theta0, requires_grad=True)
    loss = calibration_loss(theta, problem.calib)     # BCE of held-out rays vs occupancy
    loss.backward()                                   # hand-written adjoint on the GPU

theta = (kernel length-scale ls [m], kernel amplitude sigma, free-space decay gamma, occupied prior
mass, free prior mass). The loss is the mean binary cross-entropy between the occupancy after the
training frames and the held-out labels (3-D DDA: 1 for the voxel holding a hit, 0 for the voxels
traversed before it). The particle weight sums of the steady frames come from the library's own
update and are data: sort and resampling are not differentiated.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _native as N
from .dom import DOM, _ptr, make_params

THETA_NAMES = ("ls", "sigma", "gamma", "prior_occ", "prior_free")


class Calibration:
    """One calibration problem on one GPU (k3dom_calib)."""

    def __init__(self, params: N.Params, device: int = 0):
        self._lib = N.load()
        self.params = params
        h = C.c_void_p()
        N.check(self._lib.k3dom_calib_create(C.byref(params), int(device), C.byref(h)), "k3dom_calib_create")
        self._h = h
        cells = C.c_int32()
        N.check(self._lib.k3dom_calib_info(self._h, C.byref(cells), None, None), "k3dom_calib_info")
        self.cells = cells.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.k3dom_calib_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_frame(self, dt: float, sensor_rel, pts, dyn_pred=None) -> None:
        a = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        d = None if dyn_pred is None else np.ascontiguousarray(dyn_pred, np.float32).reshape(self.cells)
        s = [float(v) for v in sensor_rel]
        N.check(self._lib.k3dom_calib_add_frame(self._h, float(dt), s[0], s[1], s[2], _ptr(a), a.shape[0], _ptr(d),
                                                N.MEM_HOST), "k3dom_calib_add_frame")

    def add_heldout(self, sensor_rel, pts) -> None:
        a = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        s = [float(v) for v in sensor_rel]
        N.check(self._lib.k3dom_calib_add_heldout_scan(self._h, s[0], s[1], s[2], _ptr(a), a.shape[0], N.MEM_HOST),
                "k3dom_calib_add_heldout_scan")

    def label_counts(self):
        n0 = np.empty(self.cells, np.uint32)
        n1 = np.empty(self.cells, np.uint32)
        N.check(self._lib.k3dom_calib_label_counts(self._h, _ptr(n0), _ptr(n1), N.MEM_HOST), "label_counts")
        return n0, n1

    def sums(self, ls: float, frame: int) -> np.ndarray:
        out = np.empty((4, self.cells), np.float64)
        N.check(self._lib.k3dom_calib_get_sums(self._h, float(ls), int(frame), _ptr(out), N.MEM_HOST), "get_sums")
        return out

    @staticmethod
    def _theta(theta) -> C.Array:
        t = [float(v) for v in np.asarray(theta, np.float64).reshape(5)]
        return (C.c_float * 5)(*t)

    def loss(self, theta) -> float:
        out = C.c_float()
        N.check(self._lib.k3dom_bgki_forward(self._h, self._theta(theta), C.byref(out), None, N.MEM_HOST),
                "k3dom_bgki_forward", self._h)
        return out.value

    def occupancy(self, theta) -> np.ndarray:
        out = np.empty(self.cells, np.float32)
        loss = C.c_float()
        N.check(self._lib.k3dom_bgki_forward(self._h, self._theta(theta), C.byref(loss), _ptr(out), N.MEM_HOST),
                "k3dom_bgki_forward")
        return out

    def loss_and_grad(self, theta, grad_loss: float = 1.0):
        g = (C.c_float * 5)()
        loss = C.c_float()
        N.check(self._lib.k3dom_bgki_backward(self._h, self._theta(theta), float(grad_loss), g, C.byref(loss)),
                "k3dom_bgki_backward")
        return loss.value, np.array(list(g), np.float64)

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(self._lib.k3dom_calib_get_stream(self._h, C.byref(s)), "k3dom_calib_get_stream")
        return s.value or 0


def _autograd_function():
    import torch

    class BGKICalibrationLoss(torch.autograd.Function):
        """loss = BCE(held-out labels, occupancy(theta)); backward by k3dom_bgki_backward."""

        @staticmethod
        def forward(ctx, theta, calib):
            th = theta.detach().to("cpu", torch.float64).numpy().copy()
            ctx.calib = calib
            ctx.theta = th
            loss = calib.loss(th)
            return torch.tensor(loss, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            _, g = ctx.calib.loss_and_grad(ctx.theta, float(grad_out))
            return torch.tensor(g, dtype=grad_out.dtype, device=grad_out.device), None

    return BGKICalibrationLoss


_FN = None


def calibration_loss(theta, calib: Calibration):
    """Differentiable loss of the calibration problem (a torch.autograd.Function)."""
    global _FN
    if _FN is None:
        _FN = _autograd_function()
    return _FN.apply(theta, calib)


@dataclasses.dataclass
class Problem:
    calib: Calibration
    theta0: tuple
    frames: list      # (dt, sensor_rel, pts, dyn or None) as given to the calibration
    heldout: list     # (sensor_rel, pts)
    grid: tuple       # (G, Gz, res, mass_scale)

    def close(self):
        self.calib.close()


def build_problem(cfg, device: int = 0) -> Problem:
    """Runs the library's update over the training frames (for the particle weight sums of the
    steady frames), then builds the calibration problem of `cfg` (k3dom_b200.scene.config4)."""
    p = make_params("k3dom", **cfg.params)
    dom = DOM(p, "k3dom", device)
    calib = Calibration(p, device)
    frames = []
    t_prev = None
    centre = None
    for k, (t, s, pts) in enumerate(cfg.train):
        dom.updatePose(*s)
        info = dom.info()
        centre = np.array([info.center_x, info.center_y, info.center_z], np.float64)
        dom.updateGrid(t, pts)
        dyn = dom.get_cell_field("pred_mass") if k > 0 else None
        dt = 0.0 if t_prev is None else float(np.float32(t) - np.float32(t_prev))
        rel = (np.asarray(s, np.float64) - centre).astype(np.float32)
        calib.add_frame(dt, rel, pts, dyn)
        frames.append((dt, rel, np.ascontiguousarray(pts, np.float32), dyn))
        t_prev = t
    info = dom.info()
    heldout = []
    for s, pts in cfg.heldout:
        rel = (np.asarray(s, np.float64) - centre).astype(np.float32)
        calib.add_heldout(rel, pts)
        heldout.append((rel, np.ascontiguousarray(pts, np.float32)))
    grid = (info.grid_size, info.grid_size_z, float(p.resolution), float(p.mass_scale))
    dom.close()
    return Problem(calib, tuple(cfg.theta0), frames, heldout, grid)

"""Python mirror of the reference's update API (dom::DOM_c / dom::DOM).

Method names follow include/common/dom.h:54-94, include/k3dom/dom.h:19-29 and
include/dsphdmib/dom.h:19-32 so code written against the reference reads the same; every
call goes through the C ABI of libk3dom_b200.so (include/k3dom_b200.h).

    p = params_from_yaml("k3dom", "config/k3dom.yaml", "config/complex.yaml")
    dom = DOM(p, "k3dom")
    dom.updatePose(x, y, z)
    dom.updateGrid(t, xs, ys, zs)
    occ = dom.get_cell_field("occ_mean")
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _native as N

GRIDCELL_DTYPE = np.dtype([
    ("start_idx", "<i4"), ("end_idx", "<i4"), ("mu_A", "<f4"), ("mu_UA", "<f4"), ("w_A", "<f4"),
    ("w_UA", "<f4"), ("mean_x_vel", "<f4"), ("mean_y_vel", "<f4"), ("mean_z_vel", "<f4"),
    ("likelihood", "<f4"), ("p_A", "<f4"), ("free_mass", "<f4"), ("static_mass", "<f4"),
    ("dynamic_mass", "<f4"), ("occ_mass", "<f4"), ("pers_mass", "<f4"), ("pred_mass", "<f4"),
])
assert GRIDCELL_DTYPE.itemsize == 68

MAPPOINT_DTYPE = np.dtype([(n, "<f4") for n in (
    "x", "y", "z", "v_x", "v_y", "v_z", "occ_val", "dyn_val", "eval_aug", "dyn_aug")])

_VARIANTS = {"k3dom": N.VARIANT_K3DOM, "dsphdmib": N.VARIANT_DSPHDMIB,
             N.VARIANT_K3DOM: N.VARIANT_K3DOM, N.VARIANT_DSPHDMIB: N.VARIANT_DSPHDMIB}
_SETS = {"persistent": N.PARTICLES_PERSISTENT, "sorted": N.PARTICLES_SORTED, "birth": N.PARTICLES_BIRTH}


def _variant(v) -> int:
    try:
        return _VARIANTS[v]
    except KeyError:
        raise ValueError(f"unknown variant {v!r} (k3dom | dsphdmib)") from None


def params_default(variant="k3dom") -> N.Params:
    lib = N.load()
    p = N.Params()
    N.check(lib.k3dom_params_default(_variant(variant), C.byref(p)), "k3dom_params_default")
    return p


def params_from_yaml(variant, method_yaml: Optional[str], dataset_yaml: Optional[str] = None) -> N.Params:
    lib = N.load()
    p = N.Params()
    enc = lambda s: s.encode() if s else None  # noqa: E731
    N.check(lib.k3dom_params_from_yaml(_variant(variant), enc(method_yaml), enc(dataset_yaml), C.byref(p)),
            "k3dom_params_from_yaml")
    return p


def node_config_from_yaml(variant, method_yaml, dataset_yaml=None) -> N.NodeConfig:
    lib = N.load()
    c = N.NodeConfig()
    enc = lambda s: s.encode() if s else None  # noqa: E731
    N.check(lib.k3dom_node_config_from_yaml(_variant(variant), enc(method_yaml), enc(dataset_yaml), C.byref(c)),
            "k3dom_node_config_from_yaml")
    return c


def make_params(variant="k3dom", **kw) -> N.Params:
    p = params_default(variant)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"k3dom_params has no field {k!r}")
        setattr(p, k, v)
    return p


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _ptr(a) -> int:
    return a.ctypes.data if a is not None else None


def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and getattr(x, "is_cuda") and hasattr(x, "data_ptr")


class DOM:
    """The K3DOM / DS-PHD/MIB grid (dom::DOM), on one GPU.

    A DOM either owns a single-scene handle or is a view of one scene of a BatchDOM
    (BatchDOM.scene(s)); per-scene calls select that scene first."""

    def __init__(self, params: N.Params, variant="k3dom", device: int = 0, _handle=None, _scene: int = 0):
        self._lib = N.load()
        self.variant = _variant(variant)
        self.params = params
        self._scene = int(_scene)
        self._owner = _handle is None
        if _handle is None:
            h = C.c_void_p()
            N.check(self._lib.k3dom_create(C.byref(params), self.variant, int(device), C.byref(h)), "k3dom_create")
            self._h = h
        else:
            self._h = _handle
        info = self.info()
        self.grid_size = info.grid_size
        self.grid_size_z = info.grid_size_z
        self.grid_cell_count = info.grid_cell_count
        self.particle_count = info.particle_count
        self.new_born_particle_count = info.new_born_particle_count

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            if self._owner:
                self._lib.k3dom_destroy(self._h)
            self._h = None

    def _sel(self):
        N.check(self._lib.k3dom_select_scene(self._h, self._scene), "k3dom_select_scene")
        return self._h

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- points
    def _points(self, xs, ys=None, zs=None):
        """Returns (px, py, pz, n, mem, keepalive)."""
        if _is_cuda_tensor(xs):
            import torch
            if ys is None:
                t = xs.to(torch.float32).contiguous()
                assert t.dim() == 2 and t.shape[1] == 3
                return t.data_ptr(), None, None, int(t.shape[0]), N.MEM_DEVICE, (t,)
            tx, ty, tz = (v.to(torch.float32).contiguous() for v in (xs, ys, zs))
            if not (tx.numel() == ty.numel() == tz.numel()):
                raise ValueError("xs, ys, zs differ in length")
            return tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), int(tx.numel()), N.MEM_DEVICE, (tx, ty, tz)
        if ys is None:
            a = _f32(xs).reshape(-1, 3)
            return _ptr(a), None, None, int(a.shape[0]), N.MEM_HOST, (a,)
        x, y, z = _f32(xs), _f32(ys), _f32(zs)
        if not (x.size == y.size == z.size):  # src/k3dom/dom.cu:83 asserts equal lengths
            raise ValueError("xs, ys, zs differ in length")
        return _ptr(x), _ptr(y), _ptr(z), int(x.size), N.MEM_HOST, (x, y, z)

    # -- DOM_c interface (include/common/dom.h:57-94)
    def updatePose(self, x: float, y: float, z: float) -> None:
        N.check(self._lib.k3dom_update_pose(self._sel(), float(x), float(y), float(z)), "k3dom_update_pose")

    def set_point_transform(self, rotation=None, translation=None) -> None:
        """Points of the next updates are used as R p + t (the node's lidar-to-map rotation, done
        on the GPU); rotation=None switches it off."""
        r = None if rotation is None else np.ascontiguousarray(rotation, np.float32).reshape(9)
        t = None if translation is None else np.ascontiguousarray(translation, np.float32).reshape(3)
        N.check(self._lib.k3dom_set_point_transform(self._h, self._scene, _ptr(r), _ptr(t)),
                "k3dom_set_point_transform")

    def updateGrid(self, t: float, xs, ys=None, zs=None) -> None:
        px, py, pz, n, mem, _keep = self._points(xs, ys, zs)
        N.check(self._lib.k3dom_update_grid(self._h, float(t), px, py, pz, n, mem), "k3dom_update_grid", self._h)

    def updateGridAsync(self, t: float, xs, ys=None, zs=None) -> None:
        px, py, pz, n, mem, keep = self._points(xs, ys, zs)
        self._keep = keep
        N.check(self._lib.k3dom_update_grid_async(self._h, float(t), px, py, pz, n, mem), "k3dom_update_grid_async",
                self._h)

    def synchronize(self) -> None:
        N.check(self._lib.k3dom_synchronize(self._h), "k3dom_synchronize", self._h)

    update_pose = updatePose
    update_grid = updateGrid

    def particlePrediction(self, dt: float) -> None:
        N.check(self._lib.k3dom_particle_prediction(self._h, float(dt)), "particlePrediction")

    def particleAssignment(self) -> None:
        N.check(self._lib.k3dom_particle_assignment(self._h), "particleAssignment")

    def gridCellOccupancyUpdate(self, dt: float, xs, ys=None, zs=None) -> None:
        px, py, pz, n, mem, _keep = self._points(xs, ys, zs)
        N.check(self._lib.k3dom_grid_cell_occupancy_update(self._h, float(dt), px, py, pz, n, mem),
                "gridCellOccupancyUpdate")

    def updatePersistentParticles(self) -> None:
        N.check(self._lib.k3dom_update_persistent_particles(self._h), "updatePersistentParticles")

    def initializeNewParticles(self) -> None:
        N.check(self._lib.k3dom_initialize_new_particles(self._h), "initializeNewParticles")

    def statisticalMoments(self) -> None:
        N.check(self._lib.k3dom_statistical_moments(self._h), "statisticalMoments")

    def resampling(self) -> None:
        N.check(self._lib.k3dom_resampling(self._h), "resampling")

    def initializeParticles(self, xs, ys=None, zs=None) -> None:
        px, py, pz, n, mem, _keep = self._points(xs, ys, zs)
        N.check(self._lib.k3dom_initialize_particles(self._h, px, py, pz, n, mem), "initializeParticles")

    def finishFrame(self, t: float) -> None:
        N.check(self._lib.k3dom_finish_frame(self._h, float(t)), "finishFrame")

    def setFrameIndex(self, frame: int) -> None:
        N.check(self._lib.k3dom_set_frame_index(self._h, int(frame)), "setFrameIndex")

    def set_sort_wait(self, max_polls: int = 1 << 20, skip_tile: int = -1) -> None:
        """Test hook of the particle sort's bounded look-back waits (k3dom_set_sort_wait)."""
        N.check(self._lib.k3dom_set_sort_wait(self._h, int(max_polls), int(skip_tile)), "k3dom_set_sort_wait")

    # -- getters (include/common/dom.h:59-83)
    def info(self) -> N.Info:
        i = N.Info()
        N.check(self._lib.k3dom_get_info(self._sel(), C.byref(i)), "k3dom_get_info")
        return i

    def getGridSize(self) -> int:
        return self.grid_size

    def getResolution(self) -> float:
        return float(self.params.resolution)

    def getCenterPositionX(self) -> float: return self.info().center_x
    def getCenterPositionY(self) -> float: return self.info().center_y
    def getCenterPositionZ(self) -> float: return self.info().center_z
    def getSensorPositionX(self) -> float: return self.info().sensor_x
    def getSensorPositionY(self) -> float: return self.info().sensor_y
    def getSensorPositionZ(self) -> float: return self.info().sensor_z
    def getIteration(self) -> int: return self.info().iteration

    def indexToCoord(self, i: int):
        x, y, z = C.c_float(), C.c_float(), C.c_float()
        N.check(self._lib.k3dom_index_to_coord(self._sel(), int(i), C.byref(x), C.byref(y), C.byref(z)), "indexToCoord")
        return x.value, y.value, z.value

    def indexToCoordX(self, i: int) -> float: return self.indexToCoord(i)[0]
    def indexToCoordY(self, i: int) -> float: return self.indexToCoord(i)[1]
    def indexToCoordZ(self, i: int) -> float: return self.indexToCoord(i)[2]

    # -- readback
    def set_output(self, name: Optional[str], out=None) -> None:
        """Registered output: every following frame writes cell field `name` of this scene into
        `out` (a float32 array of grid_cell_count cells in pinned host memory, e.g.
        torch.empty(n).pin_memory(), or a CUDA tensor) as part of the frame; None stops it."""
        if name is None or out is None:
            N.check(self._lib.k3dom_set_output(self._sel(), 0, None, N.MEM_HOST), "set_output")
            self._output = None
            return
        dev = _is_cuda_tensor(out)
        n = out.numel() if dev or hasattr(out, "numel") else np.asarray(out).size
        if n != self.grid_cell_count:
            raise ValueError(f"output needs {self.grid_cell_count} floats, got {n}")
        if dev:
            ptr, mem = out.data_ptr(), N.MEM_DEVICE
        elif hasattr(out, "data_ptr"):
            ptr, mem = out.data_ptr(), N.MEM_HOST
        else:
            arr = np.asarray(out)
            if arr.dtype != np.float32 or not arr.flags.c_contiguous:
                raise ValueError("output must be a contiguous float32 array")
            ptr, mem = arr.ctypes.data, N.MEM_HOST
        N.check(self._lib.k3dom_set_output(self._sel(), N.CELL_FIELDS[name], ptr, mem), "set_output")
        self._output = out

    def get_cell_field(self, name: str) -> np.ndarray:
        out = np.empty(self.grid_cell_count, np.float32)
        N.check(self._lib.k3dom_get_cell_field(self._sel(), N.CELL_FIELDS[name], _ptr(out), N.MEM_HOST), name)
        return out

    def get_cell_ranges(self):
        s = np.empty(self.grid_cell_count, np.int32)
        e = np.empty(self.grid_cell_count, np.int32)
        N.check(self._lib.k3dom_get_cell_ranges(self._sel(), _ptr(s), _ptr(e), N.MEM_HOST), "cell_ranges")
        return s, e

    def get_gridcells(self) -> np.ndarray:
        """The 68-byte dom::GridCell array the ROS node copies back (k3dom_node.cpp:131-132)."""
        out = np.empty(self.grid_cell_count, GRIDCELL_DTYPE)
        N.check(self._lib.k3dom_get_gridcell_aos(self._sel(), _ptr(out), N.MEM_HOST), "gridcell_aos")
        return out

    def get_mappoints(self) -> np.ndarray:
        out = np.empty(self.grid_cell_count, MAPPOINT_DTYPE)
        N.check(self._lib.k3dom_get_mappoints(self._sel(), _ptr(out), N.MEM_HOST), "mappoints")
        return out

    def set_cell_masses(self, free=None, static=None, dynamic=None, occ=None) -> None:
        arrs = [None if a is None else _f32(a) for a in (free, static, dynamic, occ)]
        for a in arrs:
            if a is not None and a.size != self.grid_cell_count:
                raise ValueError("cell array size mismatch")
        N.check(self._lib.k3dom_set_cell_masses(self._sel(), *[_ptr(a) for a in arrs], N.MEM_HOST), "set_cell_masses")

    def get_particles(self, which: str = "persistent") -> dict:
        n = self.new_born_particle_count if which == "birth" else self.particle_count
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        w = np.empty(n, np.float32)
        cell = np.empty(n, np.int32)
        assoc = np.empty(n, np.uint8)
        N.check(self._lib.k3dom_get_particles(self._sel(), _SETS[which], _ptr(pos), _ptr(vel), _ptr(w), _ptr(cell),
                                              _ptr(assoc), N.MEM_HOST), "get_particles")
        return {"pos": pos, "vel": vel, "weight": w, "cell": cell, "associated": assoc}

    def set_particles(self, which: str, pos=None, vel=None, weight=None, cell=None, associated=None) -> None:
        n = self.new_born_particle_count if which == "birth" else self.particle_count
        pos = None if pos is None else _f32(pos).reshape(n, 3)
        vel = None if vel is None else _f32(vel).reshape(n, 3)
        weight = None if weight is None else _f32(weight).reshape(n)
        cell = None if cell is None else np.ascontiguousarray(cell, np.int32).reshape(n)
        associated = None if associated is None else np.ascontiguousarray(associated, np.uint8).reshape(n)
        N.check(self._lib.k3dom_set_particles(self._sel(), _SETS[which], _ptr(pos), _ptr(vel), _ptr(weight), _ptr(cell),
                                              _ptr(associated), N.MEM_HOST), "set_particles")

    def sort_permutation(self) -> np.ndarray:
        out = np.empty(self.particle_count, np.int32)
        N.check(self._lib.k3dom_get_sort_permutation(self._sel(), _ptr(out), N.MEM_HOST), "sort_permutation")
        return out

    def ancestors(self) -> np.ndarray:
        out = np.empty(self.particle_count, np.int32)
        N.check(self._lib.k3dom_get_ancestors(self._sel(), _ptr(out), N.MEM_HOST), "ancestors")
        return out

    def resampling_state(self):
        jc = np.empty(self.particle_count + self.new_born_particle_count, np.float32)
        bc = np.empty(self.grid_cell_count, np.float32)
        jm = np.empty(1, np.float32)
        N.check(self._lib.k3dom_get_resampling_state(self._sel(), _ptr(jc), _ptr(bc), _ptr(jm), N.MEM_HOST),
                "resampling_state")
        return jc, bc, float(jm[0])

    def stage_times(self) -> dict:
        t = N.StageTimes()
        N.check(self._lib.k3dom_get_stage_times(self._h, C.byref(t)), "stage_times")
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_timing(self, on: bool) -> None:
        N.check(self._lib.k3dom_set_timing(self._h, 1 if on else 0), "set_timing")

    def set_graph_mode(self, on: bool) -> None:
        N.check(self._lib.k3dom_set_graph_mode(self._h, 1 if on else 0), "set_graph_mode")

    def diagnostics(self) -> dict:
        d = N.Diagnostics()
        N.check(self._lib.k3dom_get_diagnostics(self._h, C.byref(d)), "diagnostics")
        return {k: getattr(d, k) for k, _ in d._fields_}

    def autotune(self, on: bool = True) -> None:
        N.check(self._lib.k3dom_autotune(self._h, 1 if on else 0), "k3dom_autotune")

    def tuning(self) -> dict:
        t = N.Tuning()
        N.check(self._lib.k3dom_get_tuning(self._h, C.byref(t)), "k3dom_get_tuning")
        d = {k: getattr(t, k) for k, _ in t._fields_ if k != "candidate_ms"}
        d["candidate_ms"] = list(t.candidate_ms)[: t.candidates]
        return d

    def set_tuning(self, tile_rule: int, chunk: int) -> None:
        N.check(self._lib.k3dom_set_tuning(self._h, int(tile_rule), int(chunk)), "k3dom_set_tuning")

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(self._lib.k3dom_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0


def rotation_from_quaternion(x: float, y: float, z: float, w: float) -> np.ndarray:
    """Row-major 3x3 rotation of the unit quaternion (x, y, z, w), as float32 for
    k3dom_set_point_transform (the node's tf rotation of a pose's orientation)."""
    n = math.sqrt(x * x + y * y + z * z + w * w)
    x, y, z, w = x / n, y / n, z / n, w / n
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], np.float32)


def _points_of(item):
    """(xs, ys, zs) of one scene's points: an (n, 3) array/tensor or an (xs, ys, zs) tuple."""
    if isinstance(item, (tuple, list)) and len(item) == 3:
        return item[0], item[1], item[2]
    return item, None, None


class BatchDOM:
    """S independent scenes updated together (k3dom_batch_*): one launch per stage for all
    scenes, each scene bit-identical to the same scene in a DOM of its own."""

    def __init__(self, params_list, variant="k3dom", device: int = 0):
        self._lib = N.load()
        self.variant = _variant(variant)
        self.params = list(params_list)
        arr = (N.Params * len(self.params))(*self.params)
        h = C.c_void_p()
        N.check(self._lib.k3dom_batch_create(arr, len(self.params), self.variant, int(device), C.byref(h)),
                "k3dom_batch_create")
        self._h = h
        self.scenes = [DOM(p, variant, _handle=h, _scene=s) for s, p in enumerate(self.params)]

    def __len__(self):
        return len(self.scenes)

    def scene(self, s: int) -> DOM:
        return self.scenes[s]

    def close(self) -> None:
        if getattr(self, "_h", None):
            for v in self.scenes:
                v._h = None
            self._lib.k3dom_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def updatePose(self, scene: int, x: float, y: float, z: float) -> None:
        N.check(self._lib.k3dom_batch_update_pose(self._h, int(scene), float(x), float(y), float(z)),
                "k3dom_batch_update_pose")

    def _pack(self, points):
        S = len(self.scenes)
        if len(points) != S:
            raise ValueError(f"expected points for {S} scenes, got {len(points)}")
        xs, ys, zs, ns, keep, mems = [], [], [], [], [], set()
        for s in range(S):
            px, py, pz, n, mem, k = self.scenes[s]._points(*_points_of(points[s]))
            xs.append(px)
            ys.append(py)
            zs.append(pz)
            ns.append(n)
            keep.append(k)
            mems.add(mem)
        if len(mems) != 1:
            raise ValueError("all scenes' points must be host arrays, or all CUDA tensors")
        PA = C.c_void_p * S
        return (PA(*xs), PA(*ys), PA(*zs), (C.c_int32 * S)(*ns), mems.pop(), keep)

    def update(self, t, points) -> None:
        """One frame of every scene: t[s] and points[s] ((n, 3) or (xs, ys, zs))."""
        xs, ys, zs, ns, mem, _keep = self._pack(points)
        tt = (C.c_float * len(self.scenes))(*[float(v) for v in t])
        N.check(self._lib.k3dom_batch_update(self._h, tt, xs, ys, zs, ns, mem), "k3dom_batch_update", self._h)

    def update_async(self, t, points) -> None:
        xs, ys, zs, ns, mem, keep = self._pack(points)
        self._keep = (keep, xs, ys, zs, ns)
        tt = (C.c_float * len(self.scenes))(*[float(v) for v in t])
        self._keep_t = tt
        N.check(self._lib.k3dom_batch_update_async(self._h, tt, xs, ys, zs, ns, mem), "k3dom_batch_update_async",
                self._h)

    def synchronize(self) -> None:
        N.check(self._lib.k3dom_synchronize(self._h), "k3dom_synchronize", self._h)

    def autotune(self, on: bool = True) -> None:
        N.check(self._lib.k3dom_autotune(self._h, 1 if on else 0), "k3dom_autotune")

    def tuning(self) -> dict:
        t = N.Tuning()
        N.check(self._lib.k3dom_get_tuning(self._h, C.byref(t)), "k3dom_get_tuning")
        d = {k: getattr(t, k) for k, _ in t._fields_ if k != "candidate_ms"}
        d["candidate_ms"] = list(t.candidate_ms)[: t.candidates]
        return d

    def set_tuning(self, tile_rule: int, chunk: int) -> None:
        N.check(self._lib.k3dom_set_tuning(self._h, int(tile_rule), int(chunk)), "k3dom_set_tuning")

    def set_timing(self, on: bool) -> None:
        N.check(self._lib.k3dom_set_timing(self._h, 1 if on else 0), "set_timing")

    def set_graph_mode(self, on: bool) -> None:
        N.check(self._lib.k3dom_set_graph_mode(self._h, 1 if on else 0), "set_graph_mode")

    def stage_times(self) -> dict:
        return self.scenes[0].stage_times()

    def diagnostics(self) -> dict:
        return self.scenes[0].diagnostics()

    def stream(self) -> int:
        return self.scenes[0].stream()


def debug_draws(seed: int, frame: int, stage: int, first: int, count: int) -> np.ndarray:
    """The library's random draws (stage 1: 6 normals per item, 2/3: 3 uniforms, 4: 1 uniform)."""
    lib = N.load()
    per = 6 if stage == 1 else (1 if stage == 4 else 3)
    out = np.empty(count * per, np.float32)
    N.check(lib.k3dom_debug_draws(int(seed), int(frame), int(stage), int(first), int(count), _ptr(out), N.MEM_HOST),
            "k3dom_debug_draws")
    return out.reshape(count, per) if per > 1 else out

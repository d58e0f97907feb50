"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU oracle (oracle/_build/libk3dom_oracle.so)
and of the reference harness (oracle/_ref/libref_*.so). Imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg -- never by the library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libk3dom_oracle.so"
REF_SO = {"k3dom": HERE / "_ref" / "libref_k3dom.so", "dsphdmib": HERE / "_ref" / "libref_dsphdmib.so"}

_F = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_U = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_B = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class OrcGrid(C.Structure):
    _fields_ = [("G", C.c_int), ("Gz", C.c_int), ("res", C.c_float), ("sx", C.c_float), ("sy", C.c_float),
                ("sz", C.c_float)]


def build_oracle() -> Path:
    srcs = [HERE / "k3dom_oracle.c", HERE / "k3dom_calib_oracle.c"]
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return ORACLE_SO


_orc = None


def oracle() -> C.CDLL:
    global _orc
    if _orc is not None:
        return _orc
    lib = C.CDLL(os.fspath(build_oracle()))
    sig = {
        "orc_uniforms": (None, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int64, C.c_int64, _F]),
        "orc_resample_keys": (None, [C.c_uint64, C.c_uint32, C.c_int64, _U]),
        "orc_normals_libm": (None, [C.c_uint64, C.c_uint32, C.c_int64, C.c_int64, _F]),
        "orc_philox_raw": (None, [_U, _U, _U]),
        "orc_predict": (None, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                               C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, _F, _F, _F, _F, _F, _I]),
        "orc_assign": (None, [C.c_int, C.c_int, _I, _I, _I, _I, _I]),
        "orc_cell_sums": (None, [C.c_int, C.c_int, _I, _F, _F, _F, _F, _D, _D, _D, _D]),
        "orc_bgki": (None, [C.POINTER(OrcGrid), C.c_float, C.c_float, C.c_int, _F, _F, _F, _D, _D, _D, _I]),
        "orc_k3dom_update": (None, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _D, _D, _F, _F, _F,
                                    _I, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]),
        "orc_ds_measgrid": (None, [C.POINTER(OrcGrid), C.c_float, C.c_float, C.c_int, _F, _F, _F, _F, _F, _I,
                                   _I]),
        "orc_ds_update": (None, [C.c_int, C.c_double, _F, _F, _F, _F, _I, _D, _D, _D, _D, _D, _D, _D, _D, _D,
                                 _D, _D, _D, _D, _D]),
        "orc_exact_scan": (None, [C.c_int64, _F, C.c_int64, _F, _F]),
        "orc_births": (None, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _F, _F, _F, _I, _B,
                              _F, _F, _F, _B]),
        "orc_init_particles": (None, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _F, _F, _I, _F, _F,
                                      _F]),
        "orc_resample": (C.c_float, [C.c_int, C.c_int, _F, _F, C.c_uint64, C.c_uint32, _I, _F]),
        "orc_lower_bound_rule": (None, [C.c_int64, _F, C.c_int64, _F, _I]),
        "orc_slot_bounds": (None, [C.c_int, _F, C.c_int, _I, _I]),
        "orc_num_threads": (C.c_int, []),
        "orc_bgki_ref32": (None, [C.POINTER(OrcGrid), C.c_float, C.c_float, C.c_int, _F, _F, _F, _F, _F, _I]),
        "orc_k3dom_update_ref32": (None, [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, _F, _F, _F, _F, _F,
                                          _F, _F, _F, _F, _F, _F]),
        "orc_bgki_sums": (None, [C.POINTER(OrcGrid), C.c_double, C.c_int, _F, _F, _F, _D, _D, _D, _D]),
        "orc_calib_loss_grad": (C.c_double, [C.c_int64, C.c_int, _D, _F, _F, _I, _U, _U, _D, C.c_double,
                                             C.c_void_p]),
        "orc_calib_occupancy": (None, [C.c_int64, C.c_int, _D, _F, _F, _I, _D, C.c_double, _D]),
        "orc_dda_labels": (None, [C.c_int, C.c_int, C.c_double, C.c_float, C.c_float, C.c_float, C.c_int, _F, _U,
                                  _U]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _orc = lib
    return lib


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- thin numpy wrappers
def uniforms(seed, frame, stage, first, count):
    per = 1 if stage == 4 else 3
    out = np.empty(count * per, np.float32)
    oracle().orc_uniforms(seed, frame, stage, first, count, out)
    return out.reshape(count, per) if per > 1 else out


def resample_keys(seed, frame, count):
    out = np.empty(count, np.uint32)
    oracle().orc_resample_keys(seed, frame, count, out)
    return out


def philox_raw(ctr, key):
    out = np.empty(4, np.uint32)
    oracle().orc_philox_raw(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def predict(state, normals, G, Gz, dt, p_S, noise_pos, noise_vel, imv, shift=None):
    """state: dict pos (n,3), vel (n,3), weight (n,). Returns a new dict with cell."""
    pos, vel = f32(state["pos"]), f32(state["vel"])
    px, py, pz = (f32(pos[:, k]) for k in range(3))
    vx, vy, vz = (f32(vel[:, k]) for k in range(3))
    w = f32(state["weight"]).copy()
    n = w.size
    cell = np.empty(n, np.int32)
    sp = 1 if shift is not None else 0
    sx, sy, sz = shift if shift is not None else (0, 0, 0)
    oracle().orc_predict(n, G, Gz, dt, p_S, noise_pos, noise_vel, imv, sp, sx, sy, sz, f32(normals).reshape(-1),
                         px, py, pz, vx, vy, vz, w, cell)
    return {"pos": np.stack([px, py, pz], 1), "vel": np.stack([vx, vy, vz], 1), "weight": w, "cell": cell}


def assign(keys, C_):
    keys = i32(keys)
    n = keys.size
    perm, sk, st, en = (np.empty(n, np.int32), np.empty(n, np.int32), np.empty(C_, np.int32), np.empty(C_, np.int32))
    oracle().orc_assign(n, C_, keys, perm, sk, st, en)
    return perm, sk, st, en


def cell_sums(sorted_keys, w, vel, C_):
    out = [np.empty(C_, np.float64) for _ in range(4)]
    vel = f32(vel)
    oracle().orc_cell_sums(int(w.size), C_, i32(sorted_keys), f32(w), f32(vel[:, 0]), f32(vel[:, 1]),
                           f32(vel[:, 2]), *out)
    return out


def grid(G, Gz, res, sensor_rel):
    return OrcGrid(G, Gz, res, *[float(np.float32(v)) for v in sensor_rel])


def bgki(G, Gz, res, sensor_rel, ls, sigma, pts):
    C_ = G * G * Gz
    out = [np.empty(C_, np.float64) for _ in range(3)] + [np.empty(C_, np.int32)]
    pts = f32(pts)
    g = grid(G, Gz, res, sensor_rel)
    oracle().orc_bgki(C.byref(g), ls, sigma, pts.shape[0], f32(pts[:, 0]), f32(pts[:, 1]), f32(pts[:, 2]), *out)
    return {"del_occ": out[0], "del_free": out[1], "tie_mass": out[2], "tie_count": out[3]}


def bgki_ref32(G, Gz, res, sensor_rel, ls, sigma, pts):
    """The reference's FP32 BGKI, brute force (small grids only)."""
    C_ = G * G * Gz
    o, fr, nd = np.empty(C_, np.float32), np.empty(C_, np.float32), np.empty(C_, np.int32)
    pts = f32(pts)
    g = grid(G, Gz, res, sensor_rel)
    oracle().orc_bgki_ref32(C.byref(g), ls, sigma, pts.shape[0], f32(pts[:, 0]), f32(pts[:, 1]), f32(pts[:, 2]), o,
                            fr, nd)
    return {"del_occ": o, "del_free": fr, "nan_drop": nd}


def k3dom_update_ref32(dt, gamma, p_B, mass_scale, ev, free, static, dyn, dyn_pred):
    C_ = free.size
    names = ["free", "static", "dyn", "born", "pers"]
    out = [np.empty(C_, np.float32) for _ in names]
    oracle().orc_k3dom_update_ref32(C_, dt, gamma, p_B, mass_scale, f32(ev["del_occ"]), f32(ev["del_free"]),
                                    f32(free), f32(static), f32(dyn), f32(dyn_pred), *out)
    return dict(zip(names, out))


def k3dom_update(dt, gamma, p_B, mass_scale, ev, free, static, dyn, has, sw, swx, swy, swz):
    C_ = free.size
    names = ["free", "static", "dyn", "born", "pers", "pred", "mu", "mvx", "mvy", "mvz"]
    out = [np.empty(C_, np.float64) for _ in names]
    oracle().orc_k3dom_update(C_, dt, gamma, p_B, mass_scale, f64(ev["del_occ"]), f64(ev["del_free"]), f32(free),
                              f32(static), f32(dyn), i32(has), f64(sw), f64(swx), f64(swy), f64(swz), *out)
    return dict(zip(names, out))


def ds_measgrid(G, Gz, res, sensor_rel, max_range, delta, pts):
    C_ = G * G * Gz
    mo, mf = np.empty(C_, np.float32), np.empty(C_, np.float32)
    nb, tie = np.empty(C_, np.int32), np.empty(C_, np.int32)
    pts = f32(pts)
    g = grid(G, Gz, res, sensor_rel)
    oracle().orc_ds_measgrid(C.byref(g), max_range, delta, pts.shape[0], f32(pts[:, 0]), f32(pts[:, 1]),
                             f32(pts[:, 2]), mo, mf, nb, tie)
    return {"meas_occ": mo, "meas_free": mf, "nbr": nb, "tie": tie}


def ds_update(p_B, meas_occ, meas_free, occ, free, has, sw, swx, swy, swz):
    C_ = occ.size
    names = ["occ", "free", "born", "pers", "pred", "mu", "div", "mvx", "mvy", "mvz"]
    out = [np.empty(C_, np.float64) for _ in names]
    oracle().orc_ds_update(C_, p_B, f32(meas_occ), f32(meas_free), f32(occ), f32(free), i32(has), f64(sw), f64(swx),
                           f64(swy), f64(swz), *out)
    return dict(zip(names, out))


def exact_scan(a, b=None):
    a = f32(a)
    b = f32(np.zeros(0) if b is None else b)
    out = np.empty(a.size + b.size, np.float32)
    oracle().orc_exact_scan(a.size, a, b.size, b if b.size else np.zeros(1, np.float32), out)
    return out


def births(born, cum, B, G, p_A, vmax, min_vel, uniforms3, prev_cell=None, prev_assoc=None):
    C_ = born.size
    cell = i32(np.zeros(B) if prev_cell is None else prev_cell).copy()
    assoc = np.ascontiguousarray(np.zeros(B) if prev_assoc is None else prev_assoc, np.uint8).copy()
    pos, vel, w, slow = np.empty(3 * B, np.float32), np.empty(3 * B, np.float32), np.empty(B, np.float32), \
        np.empty(B, np.uint8)
    oracle().orc_births(C_, B, G, p_A, vmax, min_vel, f32(born), f32(cum), f32(uniforms3).reshape(-1), cell, assoc,
                        pos, vel, w, slow)
    return {"cell": cell, "associated": assoc, "pos": pos.reshape(B, 3), "vel": vel.reshape(B, 3), "weight": w,
            "slow": slow}


def init_particles(cum, P, G, vmax, min_vel, uniforms3, prev_cell=None):
    C_ = cum.size
    cell = i32(np.zeros(P) if prev_cell is None else prev_cell).copy()
    pos, vel, w = np.empty(3 * P, np.float32), np.empty(3 * P, np.float32), np.empty(P, np.float32)
    oracle().orc_init_particles(C_, P, G, vmax, min_vel, f32(cum), f32(uniforms3).reshape(-1), cell, pos, vel, w)
    return {"cell": cell, "pos": pos.reshape(P, 3), "vel": vel.reshape(P, 3), "weight": w}


def resample(w_sorted, w_birth, seed, frame):
    P, B = w_sorted.size, w_birth.size
    anc = np.empty(P, np.int32)
    cum = np.empty(P + B, np.float32)
    jmax = oracle().orc_resample(P, B, f32(w_sorted), f32(w_birth), seed, frame, anc, cum)
    return anc, cum, jmax


def lower_bound_rule(cum, sorted_u):
    cum, sorted_u = f32(cum), f32(sorted_u)
    anc = np.empty(sorted_u.size, np.int32)
    oracle().orc_lower_bound_rule(cum.size, cum, sorted_u.size, sorted_u, anc)
    return anc


def slot_bounds(cum, v):
    cum = f32(cum)
    st, en = np.empty(cum.size, np.int32), np.empty(cum.size, np.int32)
    oracle().orc_slot_bounds(cum.size, cum, v, st, en)
    return st, en


# ---------------------------------------------------------------- map shift and map export
def map_move(sensor, center, sensor_off, res):
    """DOM_c::updatePose's integer move (src/common/dom.cu:125-127): static_cast<int> of
    (sensor - centre - offset) / resolution, every operation in FP32."""
    s, c, o = f32(sensor), f32(center), f32(sensor_off)
    q = ((s - c) - o) / np.float32(res)
    return np.trunc(q).astype(np.int64)


def map_shift_fires(move, thresh):
    """The shift condition of src/common/dom.cu:129."""
    return bool(np.any(np.abs(move) >= int(thresh)))


def shift_gridcells(cells, move, G, Gz, prior_free, prior_static, prior_dynamic, prior_occ):
    """initGridCellsKernel (src/common/kernel/init.cu:20-34) followed by moveMapKernel
    (src/common/kernel/ego_motion_compensation.cu:21-41) on a 68-byte GridCell array: a cell
    whose source x+move lies inside the grid takes the whole source record; every other cell
    keeps its own record with the priors, start/end = -1, likelihood 1 and p_A 0."""
    out = np.array(cells, copy=True)
    C_ = G * G * Gz
    idx = np.arange(C_, dtype=np.int64)
    x, y, z = idx % G, (idx % (G * G)) // G, idx // (G * G)
    nx, ny, nz = x + int(move[0]), y + int(move[1]), z + int(move[2])
    ok = (nx >= 0) & (nx < G) & (ny >= 0) & (ny < G) & (nz >= 0) & (nz < Gz)
    init = ~ok
    out["free_mass"][init] = np.float32(prior_free)
    out["static_mass"][init] = np.float32(prior_static)
    out["dynamic_mass"][init] = np.float32(prior_dynamic)
    out["occ_mass"][init] = np.float32(prior_occ)
    out["start_idx"][init] = -1
    out["end_idx"][init] = -1
    out["likelihood"][init] = np.float32(1.0)
    out["p_A"][init] = np.float32(0.0)
    src = (nx + G * ny + G * G * nz)[ok]
    out[ok] = cells[src]
    return out


def shift_positions(pos, move):
    """moveParticlesKernel (src/common/kernel/ego_motion_compensation.cu:12-18): pos -= move in
    FP32."""
    return (f32(pos) - np.asarray(move, np.float32)[None, :]).astype(np.float32)


def index_to_coord(idx, G, res, size, size_z, center):
    """DOM_c::indexToCoord{X,Y,Z} (include/common/dom.h:70-81), FP32 in the written order."""
    idx = np.asarray(idx, np.int64)
    r = np.float32(res)
    c = f32(center)
    hx = np.float32(size) / np.float32(2.0)
    hz = np.float32(size_z) / np.float32(2.0)
    ix = (idx % G).astype(np.float32)
    iy = ((idx % (G * G)) // G).astype(np.float32)
    iz = (idx // (G * G)).astype(np.float32)
    x = ((ix + np.float32(0.5)) * r - hx) + c[0]
    y = ((iy + np.float32(0.5)) * r - hx) + c[1]
    z = ((iz + np.float32(0.5)) * r - hz) + c[2]
    return np.stack([x, y, z], 1).astype(np.float32)


def mappoints(cells, G, res, size, size_z, center):
    """The node's /map_data point per cell (src/k3dom/k3dom_node.cpp:161-184): indexToCoord,
    velocity x resolution, occ_mean, dyn_mean and total_mass (include/common/dom_types.h:47-49),
    dyn_aug = 1.1. Returns (C, 10) float32 in MapPoint's field order."""
    C_ = cells.shape[0]
    out = np.empty((C_, 10), np.float32)
    out[:, 0:3] = index_to_coord(np.arange(C_), G, res, size, size_z, center)
    r = np.float32(res)
    out[:, 3] = cells["mean_x_vel"] * r
    out[:, 4] = cells["mean_y_vel"] * r
    out[:, 5] = cells["mean_z_vel"] * r
    f, s, d = cells["free_mass"], cells["static_mass"], cells["dynamic_mass"]
    with np.errstate(divide="ignore", invalid="ignore"):
        tm = ((f + s) + d).astype(np.float32)
        out[:, 6] = (s + d) / tm
        out[:, 7] = d / tm
    out[:, 8] = tm
    out[:, 9] = np.float32(1.1)
    return out


# ---------------------------------------------------------------- reference harness
GRIDCELL_DTYPE = np.dtype([
    ("start_idx", "<i4"), ("end_idx", "<i4"), ("mu_A", "<f4"), ("mu_UA", "<f4"), ("w_A", "<f4"),
    ("w_UA", "<f4"), ("mean_x_vel", "<f4"), ("mean_y_vel", "<f4"), ("mean_z_vel", "<f4"),
    ("likelihood", "<f4"), ("p_A", "<f4"), ("free_mass", "<f4"), ("static_mass", "<f4"),
    ("dynamic_mass", "<f4"), ("occ_mass", "<f4"), ("pers_mass", "<f4"), ("pred_mass", "<f4"),
])


def reference_available(variant="k3dom") -> bool:
    return REF_SO[variant].exists()


class Reference:
    """The reference's own dom::DOM behind oracle/ref_harness.cu (GPU)."""

    def __init__(self, params, variant="k3dom"):
        if not REF_SO[variant].exists():
            raise FileNotFoundError(f"{REF_SO[variant]} not built (oracle/build_ref.sh)")
        lib = C.CDLL(os.fspath(REF_SO[variant]))
        V = C.c_void_p
        P = C.c_void_p
        sig = {
            "ref_create": (V, [P, C.c_uint64]), "ref_destroy": (None, [V]), "ref_sizes": (None, [V, _I]),
            "ref_update_pose": (None, [V, C.c_float, C.c_float, C.c_float]), "ref_sensor_rel": (None, [V, _F]),
            "ref_center": (None, [V, _F]), "ref_index_to_coord": (None, [V, _I, C.c_longlong, _F]),
            "ref_set_draws": (None, [V, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]),
            "ref_particle_prediction": (None, [V, C.c_float]), "ref_particle_assignment": (None, [V]),
            "ref_occupancy": (None, [V, C.c_float, _F, _F, _F, C.c_int]), "ref_update_persistent": (None, [V]),
            "ref_initialize_new_particles": (None, [V]), "ref_statistical_moments": (None, [V]),
            "ref_resampling": (None, [V]), "ref_initialize_particles": (None, [V, _F, _F, _F, C.c_int]),
            "ref_finish": (None, [V, C.c_float, C.c_int]),
            "ref_update_grid": (None, [V, C.c_float, _F, _F, _F, C.c_int]),
            "ref_get_particles": (None, [V, C.c_int, P, P, P, P, P]),
            "ref_set_particles": (None, [V, C.c_int, P, P, P, P, P]),
            "ref_get_cells": (None, [V, P]), "ref_set_cells": (None, [V, P]),
            "ref_get_born": (None, [V, _F]), "ref_set_born": (None, [V, _F]),
            "ref_thrust_scan": (None, [_F, C.c_longlong, _F]),
            "ref_thrust_lower_bound": (None, [_F, C.c_longlong, _F, C.c_longlong, _I]),
            "ref_last_error": (C.c_int, []), "ref_updated_time": (C.c_float, [V]),
        }
        if variant == "dsphdmib":
            sig["ref_get_meas"] = (None, [V, _F, _F])
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib
        self.variant = variant
        self.params = params
        self.seed = int(params.seed)
        self.h = lib.ref_create(C.byref(params), self.seed)
        sz = np.empty(6, np.int32)
        lib.ref_sizes(self.h, sz)
        self.G, self.Gz, self.C, self.P, self.B, self.states = (int(v) for v in sz)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self):
        e = self.lib.ref_last_error()
        if e:
            raise RuntimeError(f"reference CUDA error {e}")

    def draws(self, frame, stage, dpi):
        self.lib.ref_set_draws(self.h, self.seed, frame, stage, dpi)

    def update_pose(self, x, y, z):
        self.lib.ref_update_pose(self.h, float(x), float(y), float(z))

    def sensor_rel(self):
        s = np.empty(3, np.float32)
        self.lib.ref_sensor_rel(self.h, s)
        return s

    def center(self):
        c = np.empty(3, np.float32)
        self.lib.ref_center(self.h, c)
        return c

    def index_to_coord(self, idx):
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.empty((idx.size, 3), np.float32)
        self.lib.ref_index_to_coord(self.h, idx, idx.size, out)
        return out

    def predict(self, frame, dt):
        self.draws(frame, 1, 6)
        self.lib.ref_particle_prediction(self.h, float(dt))
        self.check()

    def assign(self):
        self.lib.ref_particle_assignment(self.h)
        self.check()

    def occupancy(self, dt, pts):
        pts = f32(pts)
        self.lib.ref_occupancy(self.h, float(dt), f32(pts[:, 0]), f32(pts[:, 1]), f32(pts[:, 2]), pts.shape[0])
        self.check()

    def persistent(self):
        self.lib.ref_update_persistent(self.h)
        self.check()

    def births(self, frame):
        self.draws(frame, 3, 3)
        self.lib.ref_initialize_new_particles(self.h)
        self.check()

    def moments(self):
        self.lib.ref_statistical_moments(self.h)
        self.check()

    def resampling(self, frame):
        self.draws(frame, 4, 1)
        self.lib.ref_resampling(self.h)
        self.check()

    def init_particles(self, frame, pts):
        self.draws(frame, 2, 3)
        pts = f32(pts)
        self.lib.ref_initialize_particles(self.h, f32(pts[:, 0]), f32(pts[:, 1]), f32(pts[:, 2]), pts.shape[0])
        self.check()

    def finish(self, t, steady):
        self.lib.ref_finish(self.h, float(t), 1 if steady else 0)

    def update_grid(self, t, pts):
        pts = f32(pts)
        self.lib.ref_update_grid(self.h, float(t), f32(pts[:, 0]), f32(pts[:, 1]), f32(pts[:, 2]), pts.shape[0])

    def particles(self, which):
        n = self.B if which == 2 else self.P
        pos, vel = np.empty((n, 3), np.float32), np.empty((n, 3), np.float32)
        w, cell, assoc = np.empty(n, np.float32), np.empty(n, np.int32), np.empty(n, np.uint8)
        self.lib.ref_get_particles(self.h, which, pos.ctypes.data, vel.ctypes.data, w.ctypes.data, cell.ctypes.data,
                                   assoc.ctypes.data)
        return {"pos": pos, "vel": vel, "weight": w, "cell": cell, "associated": assoc}

    def set_particles(self, which, pos=None, vel=None, weight=None, cell=None, associated=None):
        keep = []

        def p(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data
        self.lib.ref_set_particles(self.h, which, p(pos, np.float32), p(vel, np.float32), p(weight, np.float32),
                                   p(cell, np.int32), p(associated, np.uint8))

    def cells(self):
        out = np.empty(self.C, GRIDCELL_DTYPE)
        self.lib.ref_get_cells(self.h, out.ctypes.data)
        return out

    def set_cells(self, cells):
        cells = np.ascontiguousarray(cells, GRIDCELL_DTYPE)
        self.lib.ref_set_cells(self.h, cells.ctypes.data)

    def born(self):
        out = np.empty(self.C, np.float32)
        self.lib.ref_get_born(self.h, out)
        return out

    def set_born(self, b):
        self.lib.ref_set_born(self.h, f32(b))

    def meas(self):
        o, f = np.empty(self.C, np.float32), np.empty(self.C, np.float32)
        self.lib.ref_get_meas(self.h, o, f)
        return o, f

    def thrust_scan(self, a):
        a = f32(a)
        out = np.empty_like(a)
        self.lib.ref_thrust_scan(a, a.size, out)
        return out

    def thrust_lower_bound(self, cum, u):
        cum, u = f32(cum), f32(u)
        out = np.empty(u.size, np.int32)
        self.lib.ref_thrust_lower_bound(cum, cum.size, u, u.size, out)
        return out


# ------------------------------------------------------------------ calibration (differentiable update)
class OracleCalib:
    """FP64 reference of the calibration loss (k3dom_bgki_forward/backward): per-cell kernel and
    derivative sums (orc_bgki_sums), the mass recursion with forward-mode dual numbers
    (orc_calib_loss_grad) and DDA labels (orc_dda_labels)."""

    def __init__(self, G: int, Gz: int, res: float, mass_scale: float):
        self.G, self.Gz, self.res, self.mass_scale = int(G), int(Gz), float(res), float(mass_scale)
        self.C = self.G * self.G * self.Gz
        self.frames = []  # (dt, sensor_rel (3,), pts (n, 3) float32, dyn (C,) float32 | None)
        self.n0 = np.zeros(self.C, np.uint32)
        self.n1 = np.zeros(self.C, np.uint32)
        self._sums = {}

    def add_frame(self, dt, sensor, pts, dyn=None):
        self.frames.append((float(dt), np.asarray(sensor, np.float32), np.ascontiguousarray(pts, np.float32),
                            None if dyn is None else np.ascontiguousarray(dyn, np.float32)))
        self._sums.clear()

    def add_heldout(self, sensor, pts):
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1)
        oracle().orc_dda_labels(self.G, self.Gz, self.res, float(sensor[0]), float(sensor[1]), float(sensor[2]),
                                pts.size // 3, pts, self.n0, self.n1)

    def sums(self, ls: float) -> np.ndarray:
        """F x 4 x C: sum f occ, sum f free, sum -x f' occ, sum -x f' free."""
        key = float(ls)
        if key in self._sums:
            return self._sums[key]
        out = np.zeros((len(self.frames), 4, self.C), np.float64)
        for k, (dt, s, pts, dyn) in enumerate(self.frames):
            g = OrcGrid(self.G, self.Gz, self.res, float(s[0]), float(s[1]), float(s[2]))
            xs = np.ascontiguousarray(pts[:, 0])
            ys = np.ascontiguousarray(pts[:, 1])
            zs = np.ascontiguousarray(pts[:, 2])
            oracle().orc_bgki_sums(C.byref(g), key, xs.size, xs, ys, zs, out[k, 0], out[k, 1], out[k, 2], out[k, 3])
        self._sums[key] = out
        return out

    def _frame_arrays(self):
        F = len(self.frames)
        dt = np.array([f[0] for f in self.frames], np.float32)
        present = np.array([0 if f[3] is None else 1 for f in self.frames], np.int32)
        dyn = np.zeros((F, self.C), np.float32)
        for k, f in enumerate(self.frames):
            if f[3] is not None:
                dyn[k] = f[3]
        return F, dt, dyn, present

    def loss_grad(self, theta, want_grad=True):
        th = np.ascontiguousarray(theta, np.float64)
        s = np.ascontiguousarray(self.sums(th[0]))
        F, dt, dyn, present = self._frame_arrays()
        g = np.zeros(5, np.float64)
        loss = oracle().orc_calib_loss_grad(self.C, F, s, dt, dyn, present, self.n0, self.n1, th, self.mass_scale,
                                            g.ctypes.data if want_grad else None)
        return loss, g

    def occupancy(self, theta):
        th = np.ascontiguousarray(theta, np.float64)
        s = np.ascontiguousarray(self.sums(th[0]))
        F, dt, dyn, present = self._frame_arrays()
        p = np.zeros(self.C, np.float64)
        oracle().orc_calib_occupancy(self.C, F, s, dt, dyn, present, th, self.mass_scale, p)
        return p

    def fd_grad(self, theta, h=1e-4):
        """FP64 central finite differences of the loss, step h in every parameter."""
        th = np.asarray(theta, np.float64)
        g = np.zeros(5)
        for i in range(5):
            a, b = th.copy(), th.copy()
            a[i] += h
            b[i] -= h
            g[i] = (self.loss_grad(a, False)[0] - self.loss_grad(b, False)[0]) / (2 * h)
        return g

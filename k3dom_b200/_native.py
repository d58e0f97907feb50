"""ctypes binding of the C ABI declared in include/k3dom_b200.h.

The shared library is loaded from k3dom_b200/_lib/libk3dom_b200.so. There is no fallback:
if the library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libk3dom_b200.so"

K3DOM_OK = 0
STATUS_NAMES = {
    0: "K3DOM_OK",
    1: "K3DOM_ERR_INVALID_ARGUMENT",
    2: "K3DOM_ERR_CUDA",
    3: "K3DOM_ERR_OUT_OF_MEMORY",
    4: "K3DOM_ERR_CAPACITY",
    5: "K3DOM_ERR_NOT_READY",
    6: "K3DOM_ERR_TIMEOUT",
    7: "K3DOM_ERR_IO",
    8: "K3DOM_ERR_INVALID_INPUT",
    9: "K3DOM_ERR_NO_DEVICE",
}
VARIANT_K3DOM = 0
VARIANT_DSPHDMIB = 1
MEM_HOST = 0
MEM_DEVICE = 1
PARTICLES_PERSISTENT = 0
PARTICLES_SORTED = 1
PARTICLES_BIRTH = 2

CELL_FIELDS = {
    "free_mass": 0, "static_mass": 1, "dynamic_mass": 2, "occ_mass": 3, "pers_mass": 4,
    "pred_mass": 5, "born_mass": 6, "mean_x_vel": 7, "mean_y_vel": 8, "mean_z_vel": 9,
    "mu_A": 10, "mu_UA": 11, "w_A": 12, "w_UA": 13, "likelihood": 14, "p_A": 15,
    "occ_mean": 16, "dyn_mean": 17, "total_mass": 18, "occ_prob": 19, "var": 20,
    "meas_occ": 21, "meas_free": 22, "del_occ": 23, "del_free": 24,
}


class K3domError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


class Params(C.Structure):
    """k3dom_params: dom::DOM_c::Params (include/common/dom.h:19-52) plus seed/max_points."""

    _fields_ = [
        ("size", C.c_float), ("size_z", C.c_float), ("mass_scale", C.c_float),
        ("resolution", C.c_float), ("particle_count", C.c_int32),
        ("new_born_particle_count", C.c_int32), ("persistence_prob", C.c_float),
        ("stddev_process_noise_position", C.c_float), ("stddev_process_noise_velocity", C.c_float),
        ("birth_prob", C.c_float), ("stddev_velocity", C.c_float), ("init_max_velocity", C.c_float),
        ("particle_min_vel", C.c_float), ("sensor_off_x", C.c_float), ("sensor_off_y", C.c_float),
        ("sensor_off_z", C.c_float), ("map_shift_thresh", C.c_int32), ("prior_free", C.c_float),
        ("prior_static", C.c_float), ("prior_dynamic", C.c_float), ("prior_occ", C.c_float),
        ("sigma", C.c_float), ("ls", C.c_float), ("gamma", C.c_float), ("max_range", C.c_float),
        ("meas_occ_stddev", C.c_float), ("seed", C.c_uint64), ("max_points", C.c_int32),
        ("reserved", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class NodeConfig(C.Structure):
    _fields_ = [
        ("occupied_thresh", C.c_float), ("valid_thresh", C.c_float), ("free_thresh", C.c_float),
        ("min_z", C.c_float), ("max_z", C.c_float), ("min_var", C.c_float), ("max_var", C.c_float),
        ("ds_resolution", C.c_float), ("imu_pose_offset", C.c_float), ("map_pub_freq", C.c_int32),
        ("map_vis_mode", C.c_int32), ("do_eval", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("grid_size", C.c_int32), ("grid_size_z", C.c_int32), ("grid_cell_count", C.c_int32),
        ("particle_count", C.c_int32), ("new_born_particle_count", C.c_int32),
        ("iteration", C.c_int32), ("variant", C.c_int32), ("initialized", C.c_int32),
        ("resolution", C.c_float), ("center_x", C.c_float), ("center_y", C.c_float),
        ("center_z", C.c_float), ("sensor_x", C.c_float), ("sensor_y", C.c_float),
        ("sensor_z", C.c_float), ("updated_time", C.c_float), ("max_points", C.c_int32),
        ("frame_index", C.c_int32),
    ]


class StageTimes(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "predict_ms", "assign_ms", "occupancy_ms", "persistent_ms", "births_ms", "resample_ms",
        "total_ms", "binning_ms", "evidence_ms")]


class Diagnostics(C.Structure):
    _fields_ = [
        ("nonfinite_points", C.c_int64), ("ray_list_entries", C.c_int64),
        ("ray_list_capacity", C.c_int64), ("work_items", C.c_int64), ("overflow", C.c_int32),
        ("kernel_launches_per_frame", C.c_int32), ("kernel_evaluations", C.c_int64),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("tile_rule", C.c_int32), ("chunk", C.c_int32), ("tuned", C.c_int32), ("tuning", C.c_int32),
        ("candidates", C.c_int32), ("evidence_blocks", C.c_int32), ("best_ms", C.c_float),
        ("candidate_ms", C.c_float * 16), ("evidence_count_blocks", C.c_int32),
    ]


_P = C.c_void_p
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_ST = C.c_int

# name -> (restype, argtypes); this table is also the list of symbols the header declares.
SIGNATURES = {
    "k3dom_params_default": (_ST, [C.c_int, C.POINTER(Params)]),
    "k3dom_params_from_yaml": (_ST, [C.c_int, C.c_char_p, C.c_char_p, C.POINTER(Params)]),
    "k3dom_node_config_from_yaml": (_ST, [C.c_int, C.c_char_p, C.c_char_p, C.POINTER(NodeConfig)]),
    "k3dom_create": (_ST, [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(_P)]),
    "k3dom_destroy": (_ST, [_P]),
    "k3dom_update_pose": (_ST, [_P, C.c_float, C.c_float, C.c_float]),
    "k3dom_set_point_transform": (_ST, [_P, C.c_int32, _P, _P]),
    "k3dom_update_grid": (_ST, [_P, C.c_float, _P, _P, _P, C.c_int32, C.c_int]),
    "k3dom_update_grid_async": (_ST, [_P, C.c_float, _P, _P, _P, C.c_int32, C.c_int]),
    "k3dom_synchronize": (_ST, [_P]),
    "k3dom_get_stream": (_ST, [_P, C.POINTER(_P)]),
    "k3dom_set_graph_mode": (_ST, [_P, C.c_int]),
    "k3dom_particle_prediction": (_ST, [_P, C.c_float]),
    "k3dom_particle_assignment": (_ST, [_P]),
    "k3dom_grid_cell_occupancy_update": (_ST, [_P, C.c_float, _P, _P, _P, C.c_int32, C.c_int]),
    "k3dom_update_persistent_particles": (_ST, [_P]),
    "k3dom_initialize_new_particles": (_ST, [_P]),
    "k3dom_statistical_moments": (_ST, [_P]),
    "k3dom_resampling": (_ST, [_P]),
    "k3dom_initialize_particles": (_ST, [_P, _P, _P, _P, C.c_int32, C.c_int]),
    "k3dom_finish_frame": (_ST, [_P, C.c_float]),
    "k3dom_get_info": (_ST, [_P, C.POINTER(Info)]),
    "k3dom_index_to_coord": (_ST, [_P, C.c_int32, _F, _F, _F]),
    "k3dom_get_cell_field": (_ST, [_P, C.c_int, _P, C.c_int]),
    "k3dom_set_output": (_ST, [_P, C.c_int, _P, C.c_int]),
    "k3dom_get_cell_ranges": (_ST, [_P, _P, _P, C.c_int]),
    "k3dom_get_gridcell_aos": (_ST, [_P, _P, C.c_int]),
    "k3dom_get_mappoints": (_ST, [_P, _P, C.c_int]),
    "k3dom_set_cell_masses": (_ST, [_P, _P, _P, _P, _P, C.c_int]),
    "k3dom_get_particles": (_ST, [_P, C.c_int, _P, _P, _P, _P, _P, C.c_int]),
    "k3dom_set_particles": (_ST, [_P, C.c_int, _P, _P, _P, _P, _P, C.c_int]),
    "k3dom_get_sort_permutation": (_ST, [_P, _P, C.c_int]),
    "k3dom_get_ancestors": (_ST, [_P, _P, C.c_int]),
    "k3dom_get_resampling_state": (_ST, [_P, _P, _P, _P, C.c_int]),
    "k3dom_debug_draws": (_ST, [C.c_uint64, C.c_int32, C.c_int32, C.c_int64, C.c_int64, _P, C.c_int]),
    "k3dom_set_frame_index": (_ST, [_P, C.c_int32]),
    "k3dom_set_sort_wait": (_ST, [_P, C.c_uint32, C.c_int32]),
    "k3dom_get_stage_times": (_ST, [_P, C.POINTER(StageTimes)]),
    "k3dom_set_timing": (_ST, [_P, C.c_int]),
    "k3dom_get_diagnostics": (_ST, [_P, C.POINTER(Diagnostics)]),
    "k3dom_exact_prefix_sum_noalloc": (_ST, [_P, _P, C.c_int64, _P]),
    "k3dom_batch_create": (_ST, [C.POINTER(Params), C.c_int32, C.c_int, C.c_int, C.POINTER(_P)]),
    "k3dom_batch_size": (_ST, [_P, C.POINTER(C.c_int32)]),
    "k3dom_select_scene": (_ST, [_P, C.c_int32]),
    "k3dom_batch_update_pose": (_ST, [_P, C.c_int32, C.c_float, C.c_float, C.c_float]),
    "k3dom_batch_update": (_ST, [_P, _F, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), _I, C.c_int]),
    "k3dom_batch_update_async": (_ST, [_P, _F, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), _I, C.c_int]),
    "k3dom_autotune": (_ST, [_P, C.c_int]),
    "k3dom_get_tuning": (_ST, [_P, C.POINTER(Tuning)]),
    "k3dom_set_tuning": (_ST, [_P, C.c_int32, C.c_int32]),
    "k3dom_calib_create": (_ST, [C.POINTER(Params), C.c_int, C.POINTER(_P)]),
    "k3dom_calib_destroy": (_ST, [_P]),
    "k3dom_calib_add_frame": (_ST, [_P, C.c_float, C.c_float, C.c_float, C.c_float, _P, C.c_int32, _P, C.c_int]),
    "k3dom_calib_add_heldout_scan": (_ST, [_P, C.c_float, C.c_float, C.c_float, _P, C.c_int32, C.c_int]),
    "k3dom_calib_label_counts": (_ST, [_P, _P, _P, C.c_int]),
    "k3dom_calib_get_sums": (_ST, [_P, C.c_float, C.c_int32, _P, C.c_int]),
    "k3dom_calib_info": (_ST, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "k3dom_calib_get_stream": (_ST, [_P, C.POINTER(_P)]),
    "k3dom_bgki_forward": (_ST, [_P, _F, _F, _P, C.c_int]),
    "k3dom_bgki_backward": (_ST, [_P, _F, C.c_float, _F, _F]),
    "k3dom_status_string": (C.c_char_p, [C.c_int]),
    "k3dom_last_cuda_error": (C.c_char_p, [_P]),
    "k3dom_abi_version": (C.c_int32, []),
}

_lib = None


def load() -> C.CDLL:
    """Load libk3dom_b200.so (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m k3dom_b200.build` "
            "(the CUDA path has no fallback)")
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str, handle=None) -> None:
    if status != K3DOM_OK:
        if handle is not None and status == 2:
            where = f"{where} ({load().k3dom_last_cuda_error(handle).decode()})"
        raise K3domError(status, where)

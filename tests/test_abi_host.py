"""Host-side tests of the C ABI (no GPU): the library loads and exports every function
include/k3dom_b200.h declares; parameter loading follows the ROS nodes' defaults, YAML reads and
unit conversions (k3dom_node.cpp:219-368, dsphdmib_node.cpp:205-356); creation rejects invalid
parameters before touching a device."""
import ctypes as C
import os
import re
from pathlib import Path

import numpy as np
import pytest

import k3dom_b200 as K
from k3dom_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]
CONFIG = ROOT / "tests" / "golden" / "config"


def declared_functions():
    text = (ROOT / "include" / "k3dom_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(k3dom_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    names = declared_functions()
    assert len(names) >= 35
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    # the Python binding knows every declared function, and nothing undeclared
    assert sorted(N.SIGNATURES) == names


def test_abi_version_and_status_strings():
    lib = N.load()
    assert lib.k3dom_abi_version() == 2
    assert lib.k3dom_status_string(0) == b"ok"
    assert lib.k3dom_status_string(8) == b"non-finite input"


def test_struct_layouts_match_reference_params():
    # DOM_c::Params (include/common/dom.h:19-52): 26 four-byte fields, then our additions
    assert C.sizeof(N.Params) == 26 * 4 + 8 + 4 + 4
    assert N.Params.seed.offset == 26 * 4
    assert K.GRIDCELL_DTYPE.itemsize == 68


def test_defaults_k3dom_node():
    p = K.params_default("k3dom")
    # k3dom_node.cpp:219-258 then the index-unit conversions of :344-368 (resolution 0.1)
    assert p.resolution == pytest.approx(0.1)
    assert p.size == 10.0 and p.size_z == 5.0
    assert p.particle_count == 30_000_000 and p.new_born_particle_count == 3_000_000
    assert p.stddev_process_noise_position == pytest.approx(0.1 / 0.1)
    assert p.init_max_velocity == pytest.approx(5.0 / np.float32(0.1), rel=1e-6)
    assert p.particle_min_vel == pytest.approx(1.0 / np.float32(0.1), rel=1e-6)
    assert p.map_shift_thresh == 10
    assert (p.sigma, p.ls, p.gamma) == (1.0, 1.0, pytest.approx(0.9))
    assert (p.prior_free, p.prior_static, p.prior_dynamic, p.prior_occ) == (1.0, 1.0, 1.0, 0.0)


def test_defaults_ds_node():
    p = K.params_default("dsphdmib")
    assert p.max_range == 50.0
    assert p.meas_occ_stddev == pytest.approx(0.6)
    assert p.particle_min_vel == 0.0
    assert (p.prior_free, p.prior_occ) == (0.0, 0.0)


def test_yaml_k3dom_complex():
    p = K.params_from_yaml("k3dom", str(CONFIG / "k3dom.yaml"), str(CONFIG / "complex.yaml"))
    res = np.float32(0.2)
    assert p.resolution == pytest.approx(0.2)
    assert p.size == 40.0 and p.size_z == 5.0
    assert p.particle_count == 1_000_000 and p.new_born_particle_count == 100_000
    assert p.sigma == pytest.approx(0.1) and p.ls == pytest.approx(0.5)
    assert p.mass_scale == pytest.approx(2.5) and p.gamma == pytest.approx(0.99)
    assert p.stddev_process_noise_position == pytest.approx(np.float32(0.01) / res)
    assert p.stddev_velocity == pytest.approx(np.float32(4.0) / res)
    assert p.init_max_velocity == pytest.approx(np.float32(5.0) / res)
    assert p.particle_min_vel == pytest.approx(np.float32(0.1) / res)
    assert (p.sensor_off_x, p.sensor_off_y) == (5.0, pytest.approx(-4.7))
    assert p.map_shift_thresh == 5  # int(1 m / 0.2 m)
    assert (p.prior_free, p.prior_static, p.prior_dynamic) == (pytest.approx(0.001),) * 3


def test_yaml_ds_quirks():
    p = K.params_from_yaml("dsphdmib", str(CONFIG / "dsphdmib.yaml"), str(CONFIG / "kitti.yaml"))
    assert p.meas_occ_stddev == pytest.approx(0.1)
    assert p.max_range == 50.0  # dsphdmib_node.cpp:346 fixes it
    assert p.resolution == pytest.approx(0.4) and p.sensor_off_z == 1.0
    nc = K.node_config_from_yaml("dsphdmib", str(CONFIG / "dsphdmib.yaml"), str(CONFIG / "kitti.yaml"))
    # dsphdmib_node.cpp:255 reads occupied_thresh into valid_thresh
    assert nc.valid_thresh == pytest.approx(0.5)
    # `free_thresh: free_thresh` is not a number: the node default (0.3) stays
    assert nc.free_thresh == pytest.approx(0.3)
    # the dataset files spell the key pose_imu_offset; the node reads imu_pose_offset
    assert nc.imu_pose_offset == 0.0


def test_yaml_missing_file():
    with pytest.raises(N.K3domError) as e:
        K.params_from_yaml("k3dom", "/nonexistent/k3dom.yaml")
    assert e.value.status == 7


@pytest.mark.parametrize("field,value", [("resolution", 0.0), ("resolution", -1.0), ("size", 0.0),
                                         ("particle_count", 0), ("new_born_particle_count", 0), ("ls", 0.0)])
def test_create_rejects_invalid_params(field, value):
    lib = N.load()
    p = K.make_params("k3dom", size=3.2, size_z=1.6, resolution=0.2, particle_count=1024,
                      new_born_particle_count=256, ls=0.3)
    setattr(p, field, value)
    h = C.c_void_p()
    st = lib.k3dom_create(C.byref(p), 0, 0, C.byref(h))
    assert st == 1 and not h.value


def test_create_rejects_bad_variant_and_null():
    lib = N.load()
    p = K.params_default("k3dom")
    h = C.c_void_p()
    assert lib.k3dom_create(C.byref(p), 7, 0, C.byref(h)) == 1
    assert lib.k3dom_create(None, 0, 0, C.byref(h)) == 1
    assert lib.k3dom_destroy(None) == 1


def test_scene_generator_is_deterministic():
    from k3dom_b200 import scene
    c = scene.config0()
    s1, p1 = c.scene.scan(0, 0.0, c.n_points)
    s2, p2 = scene.config0().scene.scan(0, 0.0, c.n_points)
    assert p1.shape == (30000, 3) and np.array_equal(p1, p2) and np.array_equal(s1, s2)
    r = np.linalg.norm(p1, axis=1)
    assert r.max() < 12.8 * 1.2 and r.min() > 0.5


REF_CONFIG = Path(os.environ.get("K3DOM_REFERENCE", "/nonexistent")) / "config"


@pytest.mark.skipif(not REF_CONFIG.is_dir(), reason="set K3DOM_REFERENCE to a reference checkout")
@pytest.mark.parametrize("variant,method", [("k3dom", "k3dom.yaml"), ("dsphdmib", "dsphdmib.yaml")])
@pytest.mark.parametrize("dataset", ["complex.yaml", "kitti.yaml", "simple.yaml", "urban.yaml"])
def test_reference_config_files_load(variant, method, dataset):
    """The reference's own config files parse and agree with the local fixtures' semantics."""
    p = K.params_from_yaml(variant, str(REF_CONFIG / method), str(REF_CONFIG / dataset))
    G = int(np.float32(p.size) / np.float32(p.resolution))
    assert G > 0 and p.particle_count == 1_000_000


def _zero_args(argtypes):
    """Null for every pointer argument, zero for every number."""
    out = []
    for t in argtypes:
        if t in (C.c_float, C.c_double):
            out.append(0.0)
        elif t in (C.c_int, C.c_int32, C.c_int64, C.c_long, C.c_uint32, C.c_uint64, C.c_ulong, C.c_size_t):
            out.append(0)
        else:
            out.append(None)
    return out


def test_every_entry_point_refuses_a_null_handle():
    """The reference's DOM has no error path (device asserts trap); here every call that takes a
    handle returns K3DOM_ERR_INVALID_ARGUMENT for a null one, before touching a device, and the
    creators refuse a null output slot."""
    lib = N.load()
    handle_calls = [n for n, (_, a) in N.SIGNATURES.items()
                    if a and a[0] is N._P and n not in ("k3dom_exact_prefix_sum_noalloc", "k3dom_last_cuda_error")]
    assert len(handle_calls) >= 50
    for name in handle_calls:
        st = getattr(lib, name)(*_zero_args(N.SIGNATURES[name][1]))
        assert st == 1, f"{name} returned {st} for a null handle"
    for name in ("k3dom_create", "k3dom_batch_create", "k3dom_calib_create"):
        st = getattr(lib, name)(*_zero_args(N.SIGNATURES[name][1]))
        assert st == 1, f"{name} returned {st} for a null output"
    assert lib.k3dom_last_cuda_error(None) == b"no handle"
    # the allocation-free scan: bad sizes and missing buffers are refused, an empty scan is a no-op
    assert lib.k3dom_exact_prefix_sum_noalloc(None, None, -1, None) == 1
    assert lib.k3dom_exact_prefix_sum_noalloc(None, None, 5, None) == 1
    assert lib.k3dom_exact_prefix_sum_noalloc(None, None, 0, None) == 0

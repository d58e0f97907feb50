"""The C++ drop-in (include/k3dom_b200.hpp): dom::DOM over the C ABI, driven the way the
reference's node drives its own dom::DOM (tests/cpp/dom_frames.cpp).

CPU: the header and the driver compile with -Wall -Wextra -Werror and link against the library.
GPU: the driver runs three frames of a small scene; its 68-byte GridCell records (read back with
the node's cudaMemcpy of grid_cell_array), its /map_data points (built with the GridCell helpers
and indexToCoord*, k3dom_node.cpp:161-184) and the library's MapPoint export equal, bit for
bit, what the Python mirror of the same API gives on the same frames.
"""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "k3dom_b200" / "_lib"


def cuda_home() -> Path:
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parents[1]
    return Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def build_driver(out: Path) -> Path:
    cuda = cuda_home()
    exe = out / "dom_frames"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           "-I", str(cuda / "include"), str(ROOT / "tests" / "cpp" / "dom_frames.cpp"), "-o", str(exe),
           "-L", str(LIBDIR), "-lk3dom_b200", "-L", str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_header_compiles_and_links(tmp_path):
    if not (LIBDIR / "libk3dom_b200.so").exists():
        pytest.skip("library not built")
    exe = build_driver(tmp_path)
    assert exe.exists()
    # the DS variant is a define away, as the reference's second binary is
    src = tmp_path / "ds.cpp"
    src.write_text('#define K3DOM_B200_DSPHDMIB\n#include "k3dom_b200.hpp"\n'
                   'static_assert(dom::kDefaultVariant == K3DOM_VARIANT_DSPHDMIB, "variant");\n'
                   'int main() { dom::DOM::Params p; p.size = 12.8f; return p.seed == 0 ? 0 : 1; }\n')
    cuda = cuda_home()
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", str(ROOT / "include"), "-I",
                        str(cuda / "include"), str(src), "-o", str(tmp_path / "ds"), "-L", str(LIBDIR),
                        "-lk3dom_b200", "-L", str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_dom_matches_python_path(tmp_path):
    import k3dom_b200 as K
    from k3dom_b200 import scene

    exe = build_driver(tmp_path)
    cfg = scene.small(seed=21, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500, ego=1.0)
    cfg.params["seed"] = 99
    p = K.make_params("k3dom", **cfg.params)
    (tmp_path / "params.bin").write_bytes(bytes(p))
    frames = []
    lines = ["3"]
    for f in range(3):
        t = 0.1 + 0.1 * f
        s, pts = cfg.scene.scan(f, t, cfg.n_points)
        pts = np.ascontiguousarray(pts, np.float32)
        s = np.asarray(s, np.float32)
        (tmp_path / f"scan{f}.bin").write_bytes(pts.tobytes())
        # decimal forms of the float32 values that read back to the same floats
        lines.append(" ".join(repr(float(v)) for v in (np.float32(t), s[0], s[1], s[2])) + f" {pts.shape[0]}")
        frames.append((np.float32(t), s, pts))
    (tmp_path / "frames.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok ")

    dom = K.DOM(p, "k3dom")
    try:
        for t, s, pts in frames:
            dom.updatePose(float(s[0]), float(s[1]), float(s[2]))
            dom.updateGrid(float(t), pts[:, 0], pts[:, 1], pts[:, 2])
        cells = dom.get_gridcells()
        assert (tmp_path / "cells.bin").read_bytes() == cells.tobytes()
        mp = dom.get_mappoints()
        lib_pts = np.stack([mp[n] for n in mp.dtype.names], 1)
        node = np.fromfile(tmp_path / "mappoints_node.bin", np.float32).reshape(-1, 10)
        lib_cpp = np.fromfile(tmp_path / "mappoints_lib.bin", np.float32).reshape(-1, 10)
        np.testing.assert_array_equal(lib_cpp, lib_pts)
        np.testing.assert_array_equal(node, lib_pts)
        assert (cells["static_mass"] + cells["dynamic_mass"] > 0.01).sum() > 100
    finally:
        dom.close()

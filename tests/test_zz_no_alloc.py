"""The allocation-free prefix sum (k3dom_exact_prefix_sum_noalloc) against the update's own.

Some callers cannot allocate device memory at run time (a real-time callback with a memory
budget fixed at start-up, work recorded into a CUDA graph by a host framework, a plugin whose
memory belongs to another allocator). This entry point computes the exact prefix sum the
update uses for birth slots and ancestors with its scratch in a fixed array inside the
library. Here it must reproduce, bit for bit, the prefix sums a K3DOM handle formed in a frame
(born masses, and the joint persistent + birth weights), on two calls in a row.
This file is collected last so that a failure here cannot hide any other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_prefix_sum_matches_update():
    import torch

    import k3dom_b200 as K
    from k3dom_b200 import _native as N
    from k3dom_b200 import scene

    cfg = scene.small(seed=11, G=32, Gz=8, res=0.2, P=8192, B=2048, n_points=1500)
    cfg.params["seed"] = 17
    p = K.make_params("k3dom", **cfg.params)
    dom = K.DOM(p, "k3dom", device=0)
    lib = N.load()
    try:
        for f in range(3):
            t = 0.1 + 0.1 * f
            s, pts = cfg.scene.scan(f, t, cfg.n_points)
            dom.updatePose(*s)
            dom.updateGrid(t, pts)
        born = dom.get_cell_field("born_mass")
        joint_cum, born_cum, _ = dom.resampling_state()
        srt = dom.get_particles("sorted")["weight"]
        bw = dom.get_particles("birth")["weight"]
        joint = np.concatenate([srt, bw]).astype(np.float32)
        stream = torch.cuda.current_stream().cuda_stream
        for src, expected in ((born, born_cum), (joint, joint_cum)):  # two calls in a row
            d_in = torch.from_numpy(src).cuda()
            d_out = torch.full_like(d_in, float("nan"))
            torch.cuda.synchronize()
            st = lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(d_out), d_in.numel(), C.c_void_p(stream))
            assert st == 0, N.STATUS_NAMES.get(st)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(d_out.cpu().numpy(), expected)
        # beyond the fixed scratch: refused before any GPU work
        too_many = 33_554_432 + 1
        assert lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(d_out), too_many, None) == 4
    finally:
        dom.close()

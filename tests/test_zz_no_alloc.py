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
        inputs = [(torch.from_numpy(src).cuda(), expected) for src, expected in ((born, born_cum), (joint, joint_cum))]
        outs = [torch.full_like(d_in, float("nan")) for d_in, _ in inputs]
        torch.cuda.synchronize()
        for k, ((d_in, expected), d_out) in enumerate(zip(inputs, outs)):  # two calls in a row
            free0 = torch.cuda.mem_get_info()[0]
            st = lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(d_out), d_in.numel(), C.c_void_p(stream))
            assert st == 0, N.STATUS_NAMES.get(st)
            torch.cuda.synchronize()
            if k == 1:
                # the first call has looked up the scratch and loaded the kernels: the second
                # one takes no device memory at all
                assert torch.cuda.mem_get_info()[0] == free0
            np.testing.assert_array_equal(d_out.cpu().numpy(), expected)
        # beyond the fixed scratch: refused before any GPU work
        too_many = 33_554_432 + 1
        d_in, _ = inputs[0]
        assert lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(outs[0]), too_many, None) == 4
    finally:
        dom.close()


def test_noalloc_refused_elements_poison_the_rest():
    """Outside the exact domain (finite values in [0, 2^23)) an element is refused on the
    device: every prefix from it on is NaN, every prefix before it is the exact one."""
    import torch

    from k3dom_b200 import _native as N
    from oracle import binding as O

    lib = N.load()
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 4.0, 100_000).astype(np.float32)
    x[::97] = -0.0  # negative zero counts as zero
    exp = O.exact_scan(x)
    for bad_at, bad in ((70_001, np.float32(-1e-3)), (4_096, np.float32(np.nan)), (12, np.float32(np.inf)),
                        (99_999, np.float32(2.0 ** 23))):
        y = x.copy()
        y[bad_at] = bad
        d_in = torch.from_numpy(y).cuda()
        d_out = torch.zeros_like(d_in)
        assert lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(d_out), y.size, None) == 0
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        np.testing.assert_array_equal(got[:bad_at], exp[:bad_at])
        assert np.all(np.isnan(got[bad_at:])), bad
    # the largest value inside the domain is still exact
    y = x.copy()
    y[3] = np.nextafter(np.float32(2.0 ** 23), np.float32(0))
    d_in = torch.from_numpy(y).cuda()
    d_out = torch.zeros_like(d_in)
    assert lib.k3dom_exact_prefix_sum_noalloc(_ptr(d_in), _ptr(d_out), y.size, None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_out.cpu().numpy(), O.exact_scan(y))

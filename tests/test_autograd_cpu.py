"""Host logic of the differentiable path (no GPU): the plane lists handed to
the C ABI and the float64 torch reference the adjoint is checked against."""
import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from oracle import oracle as O
from oracle import torch_ref as TR


def test_plane_lists_follow_the_clip_end_clamp():
    import torch

    from dfttest2_b200 import autograd as A

    C, N, H, W, r = 2, 5, 8, 12, 1
    x, o, g, go = (torch.zeros(C, N, H, W) for _ in range(4))
    arr = A.frame_planes(x, o, r)
    garr = A.grad_planes(x, g, go, r)
    for c in range(C):
        for n in range(N):
            p, q = arr[c * N + n], garr[c * N + n]
            for t in range(2 * r + 1):
                k = min(max(n - r + t, 0), N - 1)
                assert p.src[t] == x[c, k].data_ptr() == q.src[t]
                assert q.grad_src[t] == g[c, k].data_ptr()
            assert p.dst == o[c, n].data_ptr() and q.grad_dst == go[c, n].data_ptr()
            assert p.src_stride == p.dst_stride == q.grad_src_stride == W * 4
            assert (p.width, p.height, q.width, q.height) == (W, H, W, H)


@pytest.mark.parametrize("kw", [dict(ftype=0, sigma=8.0, tbsize=3), dict(ftype=4, sigma=1.5, pmin=2.0, pmax=300.0),
                                dict(ftype=0, f0beta=0.7, sigma=5.0, tbsize=5, swin=2),
                                dict(ftype=2, sigma=0.7, sbsize=8, sosize=6, tbsize=1)])
def test_torch_reference_matches_fp64_oracle(kw):
    import torch

    args = plugin_arguments(full_sigma=True, **kw)
    T = 2 * args["radius"] + 1
    rng = np.random.default_rng(1)
    frames = rng.random((T, 37, 45)).astype(np.float32)
    a = O.fp64_plane(list(frames), args, 32)
    b = TR.dfttest_plane(torch.from_numpy(frames).double(), args).numpy()
    assert np.abs(a - b).max() < 1e-9


def test_torch_reference_gradients_are_finite_at_zero_psd():
    """The zero-mean DC bin has d = 0 exactly; the gains with square roots
    must give it a zero (not NaN) derivative."""
    import torch

    for kw in (dict(ftype=4, sigma=1.1, pmin=2.0, pmax=300.0), dict(ftype=0, f0beta=0.5, sigma=5.0),
               dict(ftype=0, f0beta=0.7, sigma=5.0)):
        args = plugin_arguments(full_sigma=True, **kw)
        x = torch.rand(3 if args["radius"] else 1, 32, 32, dtype=torch.float64, requires_grad=True)
        TR.dfttest_plane(x, args).sum().backward()
        assert torch.isfinite(x.grad).all()

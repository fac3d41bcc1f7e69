"""The allocation-free entry point, dfttest2_b200_process_plane_noalloc.

It serves hosts that cannot allocate GPU memory themselves (for example a
frame server that passes the filter frames out of a pool it reserved up
front, and that must not have cudaMalloc / cudaFree claim memory outside
that budget or stall its pipeline with the implicit device synchronisation
they can cause).  The entry point keeps its tables and overlap scratch in a
fixed-size device array inside the library.

Checked here through the C ABI: two calls in a row, on different inputs,
each match the regular entry point (dfttest2_b200_process_planes) within the
parity tolerance of the other GPU tests (1 LSB on integer planes, 2e-5 of
full scale on float planes); a plane that needs more scratch than the array
holds is rejected with a clear message, and so is a call inside a stream
capture; the kernels' error word, read by dfttest2_b200_noalloc_check,
reports no failure.  This file is collected last so that
a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from dfttest2_b200 import _lib
from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter

pytestmark = pytest.mark.gpu


def _params(args):
    p = _lib.Params()
    lib = _lib.load()
    lib.dfttest2_b200_params_init(ctypes.byref(p))
    keep = []
    w = _lib.as_double_array(args["window"])
    s = _lib.as_double_array(args["sigma"])
    keep += [w, s]
    p.window, p.window_len = w, len(w)
    p.sigma, p.sigma_len = s, len(s)
    p.sigma2, p.pmin, p.pmax = args["sigma2"], args["pmin"], args["pmax"]
    p.filter_type = args["filter_type"]
    p.radius = args["radius"]
    p.block_size = args["block_size"]
    p.block_step = args["block_step"]
    p.zero_mean = args["zero_mean"]
    if args["window_freq"] is not None:
        wf = _lib.as_double_array(args["window_freq"])
        keep.append(wf)
        p.window_freq, p.window_freq_len = wf, len(wf)
    p.device_id = 0
    return p, keep


def _plane(frames, n, radius, out):
    """C-ABI plane for output frame n of a (N, H, W) CUDA tensor."""
    N, h, w = frames.shape
    es = frames.element_size()
    pl = _lib.Plane()
    for t in range(2 * radius + 1):
        pl.src[t] = frames[min(max(n - radius + t, 0), N - 1)].data_ptr()
    pl.src_stride = w * es
    pl.dst = out.data_ptr()
    pl.dst_stride = w * es
    pl.width, pl.height = w, h
    return pl


def _close(a, b, is_float):
    if is_float:
        return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max()) <= 2e-5
    return int(np.abs(a.astype(np.int64) - b.astype(np.int64)).max()) <= 1


@pytest.mark.parametrize("fmt", ["u16", "f32"])
def test_noalloc_matches_regular_path_twice(fmt, cuda_device):
    import torch

    rng = np.random.default_rng(7)
    h, w, nfr = 480, 640, 4
    x = np.clip(0.5 + 0.2 * rng.standard_normal((2, nfr, h, w)), 0, 1)
    if fmt == "u16":
        host = np.round(x * 65535).astype(np.uint16)
        clips = [torch.from_numpy(host[i].view(np.int16)).to(cuda_device) for i in range(2)]
        st, bits = 0, 16
        args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3)
    else:
        host = x.astype(np.float32)
        clips = [torch.from_numpy(host[i]).to(cuda_device) for i in range(2)]
        st, bits = 1, 32
        args = plugin_arguments(ftype=1, sigma=12.0, sbsize=8, sosize=6, tbsize=5)
    r = args["radius"]
    n = 1

    # regular entry point (allocating filter object)
    flt = Filter(**args)
    try:
        ref = [flt.process_clip_device(c, st, bits) for c in clips]
        torch.cuda.synchronize()
        ref = [rr[n].cpu().numpy() for rr in ref]
    finally:
        flt.close()

    lib = _lib.load()
    p, keep = _params(args)
    stream = torch.cuda.current_stream(cuda_device).cuda_stream
    outs = []
    for c in clips:  # two calls in a row, different inputs
        out = torch.empty_like(c[0])
        pl = _plane(c, n, r, out)
        rc = lib.dfttest2_b200_process_plane_noalloc(ctypes.byref(p), ctypes.byref(pl), st, bits,
                                                     ctypes.c_void_p(stream))
        assert rc == 0, lib.dfttest2_b200_last_error().decode()
        outs.append(out)
    # the kernels' error word (in the same static array) reports no failure
    rc = lib.dfttest2_b200_noalloc_check(0, ctypes.c_void_p(stream))
    assert rc == 0, lib.dfttest2_b200_last_error().decode()
    torch.cuda.synchronize()
    for got, want in zip(outs, ref):
        assert _close(got.cpu().numpy(), want, fmt == "f32")
    del keep


def test_noalloc_rejects_planes_beyond_the_array(cuda_device):
    import torch

    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3)
    lib = _lib.load()
    p, keep = _params(args)
    # a 16384 x 8192 float plane needs far more overlap scratch than the array
    # holds.  The plane is a real allocation of that size (512 MiB) even though
    # the host-side check rejects the call before any launch: were the check
    # ever to regress, the kernels would still stay inside allocated memory.
    big = torch.zeros((8192, 16384), dtype=torch.float32, device=cuda_device)
    pl = _lib.Plane()
    for t in range(3):
        pl.src[t] = big.data_ptr()
    pl.src_stride = 16384 * 4
    pl.dst = big.data_ptr()
    pl.dst_stride = 16384 * 4
    pl.width, pl.height = 16384, 8192
    rc = lib.dfttest2_b200_process_plane_noalloc(ctypes.byref(p), ctypes.byref(pl), 1, 32, None)
    assert rc != 0
    msg = lib.dfttest2_b200_last_error().decode()
    assert "too large for the allocation-free path" in msg
    assert str(_lib.NOALLOC_SCRATCH_BYTES) in msg
    del keep


def test_noalloc_rejects_stream_capture(cuda_device):
    """Inside a stream capture the call is refused (its descriptor and table
    copies come from host memory that the call does not keep: its stack frame
    and a buffer the next call rewrites); the capture itself stays valid."""
    import torch

    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3)
    lib = _lib.load()
    p, keep = _params(args)
    frames = torch.zeros((3, 48, 64), dtype=torch.float32, device=cuda_device)
    out = torch.empty((48, 64), dtype=torch.float32, device=cuda_device)
    pl = _plane(frames, 1, 1, out)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream)
    assert lib.dfttest2_b200_process_plane_noalloc(ctypes.byref(p), ctypes.byref(pl), 1, 32, stream) == 0
    torch.cuda.synchronize()
    x = torch.zeros(16, device=cuda_device)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        x.add_(1.0)
        cs = ctypes.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream)
        rc = lib.dfttest2_b200_process_plane_noalloc(ctypes.byref(p), ctypes.byref(pl), 1, 32, cs)
        msg = lib.dfttest2_b200_last_error().decode()
    g.replay()
    torch.cuda.synchronize()
    assert rc != 0 and "stream capture" in msg
    assert float(x.sum()) == 16.0
    assert lib.dfttest2_b200_noalloc_check(0, stream) == 0
    del g, keep

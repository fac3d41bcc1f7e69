"""Parity with the reference's own CPU math at the benchmark configurations.

The checker is oracle/_ref: dfttest2_cpu's FFTW codelets, filter and fused
block pipeline (gcc_source/kernel.hpp of vs-dfttest2, compiled unchanged),
driven like cpu_source/getframe_impl.cpp:223-412.  Cases, with the seeded
synthetic generator (drifting sinusoids + noise) standing in for video:

* GRAYS float32 640x480, 8 frames, Gaussian noise 8/255; Wiener, sigma 8,
  sbsize 16 / sosize 12 / tbsize 3, Hanning spatial and rectangular temporal
  window, zero-mean, pmin 0, pmax 500: every frame, both clip ends included.
* YUV420P16 1920x1080 (chroma 960x540), Gaussian noise 4*257 codes plus 1 %
  salt-and-pepper, sigma from slocation (4 knots, 12 at DC to 4 at Nyquist),
  all three planes: frames 0, 1, 4 and 7 of an 8-frame clip (both clip ends),
  through the device-resident call and through the whole-clip host pipeline.

Bars: float planes max-abs <= 2e-5 of full scale; 16-bit planes within 1 LSB
with the exact-match fraction printed and >= 0.99.  The tensor-core form
(bf16 hi/lo x3) is held to the same 1 LSB bar on the 16-bit workload.
"""
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from dfttest2_b200.clip import GRAYS, YUV420P16
from dfttest2_b200.frontend import flatten, plugin_arguments, to_func
from dfttest2_b200.plugin import Filter
from dfttest2_b200.synth import make_clip
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")]

FLOAT_TOL = 2e-5
SLOCATION = [0.0, 12.0, 1 / 3, 28 / 3, 2 / 3, 20 / 3, 1.0, 4.0]


def _ref_frames(planes, frames, args, bits, threads=8):
    """Reference outputs {(plane index, frame): plane} over host threads."""
    jobs = [(p, n) for p in range(len(planes)) for n in frames]

    def one(job):
        p, n = job
        return job, O.ref_plane(O.clip_frames(planes[p], n, args["radius"]), args, bits)

    with ThreadPoolExecutor(threads) as ex:
        return dict(ex.map(one, jobs))


def _lsb(out, ref):
    d = np.abs(out.astype(np.int64) - ref.astype(np.int64))
    return int(d.max()), float(np.mean(d == 0))


def test_grays_640x480_against_reference(cuda_device):
    import torch

    noisy, _ = make_clip(GRAYS, 640, 480, 8, seed=1, noise_sigma=8 / 255)
    clip = noisy.planes[0]
    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3, swin=0, twin=7, zmean=True, pmin=0.0,
                            pmax=500.0)
    ref = _ref_frames([clip], range(8), args, 32)
    flt = Filter(device_id=0, synthesis_slice=2 * args["radius"], **args)
    try:
        dev = flt.process_clip_device(torch.from_numpy(clip).cuda(0), 1, 32)
        flt.check()
        dev = dev.cpu().numpy()
        host = flt.process_clip_host(clip, 1, 32)
    finally:
        flt.close()
    worst = 0.0
    for n in range(8):
        for out in (dev[n], host[n]):
            worst = max(worst, float(np.abs(out.astype(np.float64) - ref[(0, n)].astype(np.float64)).max()))
    print(f"GRAYS 640x480 x8: max-abs vs reference {worst:.3e}")
    assert worst <= FLOAT_TOL


@pytest.fixture(scope="module")
def yuv1080p():
    noisy, _ = make_clip(YUV420P16, 1920, 1080, 8, seed=1000, noise_sigma=4 * 257 / 65535, salt_pepper=0.01)
    sig = [to_func(flatten(SLOCATION), math.cbrt, 8.0)] * 3
    args = plugin_arguments(ftype=0, sigma=sig, sbsize=16, sosize=12, tbsize=3)
    frames = (0, 1, 4, 7)
    ref = _ref_frames(noisy.planes, frames, args, 16)
    return noisy.planes, args, frames, ref


def test_yuv420p16_1080p_against_reference(yuv1080p, cuda_device):
    import torch

    planes, args, frames, ref = yuv1080p
    flt = Filter(device_id=0, **args)
    try:
        dev = [flt.process_clip_device(torch.from_numpy(p.view(np.int16)).cuda(0), 0, 16) for p in planes]
        flt.check()
        dev = [d.cpu().numpy().view(np.uint16) for d in dev]
        host = flt.process_clip_planes_host(planes, 0, 16)
    finally:
        flt.close()
    for name, outs in (("device", dev), ("host pipeline", host)):
        worst, exact_sum, count = 0, 0.0, 0
        for p in range(3):
            for n in frames:
                m, e = _lsb(outs[p][n], ref[(p, n)])
                worst = max(worst, m)
                exact_sum += e * outs[p][n].size
                count += outs[p][n].size
        exact = exact_sum / count
        print(f"YUV420P16 1080p ({name}): max {worst} LSB vs reference, exact-match {exact:.5f}")
        assert worst <= 1 and exact >= 0.99


@pytest.mark.parametrize("mode", ["tc_fp16x3", "tc_bf16x3"])
def test_yuv420p16_1080p_tensor_core_against_reference(yuv1080p, mode, cuda_device):
    """The tensor-core strip form on the headline workload: within 1 LSB of the
    reference CPU math; fp16 hi/lo (about 22 bits, FP32 accumulation in tensor
    memory) also keeps >= 98 % of the samples exact (measured 98.8 %), bf16
    hi/lo (about 16 bits) is only held to 1 LSB."""
    import torch

    planes, args, frames, ref = yuv1080p
    flt = Filter(device_id=0, **args)
    try:
        flt.set_precision(mode)
        dev = [flt.process_clip_device(torch.from_numpy(p.view(np.int16)).cuda(0), 0, 16) for p in planes]
        flt.check()
        dev = [d.cpu().numpy().view(np.uint16) for d in dev]
    finally:
        flt.close()
    worst, exact_sum, count = 0, 0.0, 0
    for p in range(3):
        for n in frames:
            m, e = _lsb(dev[p][n], ref[(p, n)])
            worst = max(worst, m)
            exact_sum += e * dev[p][n].size
            count += dev[p][n].size
    exact = exact_sum / count
    print(f"YUV420P16 1080p tensor-core {mode}: max {worst} LSB vs reference, exact-match {exact:.5f}")
    assert worst <= 1
    if mode == "tc_fp16x3":
        assert exact >= 0.98

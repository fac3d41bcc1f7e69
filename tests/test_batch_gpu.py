"""Multi-clip batches (dfttest2_b200_batch_*): one graph launch over clips of
mixed size, length, format and block parameters must give what the plain
per-clip calls give (integers within 1 LSB, float within 2e-5 of full scale;
the unit split may differ, which reorders the overlap-add sums), and match
the FP64 oracle like the plain path does."""
import numpy as np
import pytest

from dfttest2_b200 import _lib
from dfttest2_b200.clip import GRAYS, YUV420P8, YUV420P16
from dfttest2_b200.frontend import plugin_arguments
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (width, height, frames, format, DFTTest arguments)
SPECS = [
    (160, 120, 5, YUV420P16, dict(sbsize=16, sosize=12, tbsize=3, ftype=0, sigma=8.0)),
    (200, 96, 4, GRAYS, dict(sbsize=8, sosize=6, tbsize=5, ftype=1, sigma=9.0)),
    (320, 180, 3, YUV420P8, dict(sbsize=32, sosize=24, tbsize=1, ftype=0, sigma=4.0)),
    (96, 72, 6, GRAYS, dict(sbsize=16, sosize=12, tbsize=3, ftype=0, sigma=12.0)),
    (176, 144, 4, YUV420P16, dict(sbsize=16, sosize=12, tbsize=3, ftype=0, sigma=5.0, zmean=False)),
    (192, 160, 7, YUV420P8, dict(sbsize=8, sosize=6, tbsize=3, ftype=0, sigma=6.0)),
    (256, 128, 2, GRAYS, dict(sbsize=32, sosize=24, tbsize=5, ftype=1, sigma=3.0)),
    # frequency-dependent sigma (12 at DC to 4 at Nyquist): the general kernel with asymmetric lanes
    (128, 128, 4, YUV420P16, dict(sbsize=16, sosize=12, tbsize=1, ftype=0, sigma=lambda f: 12.0 - 8.0 * f)),
]


def _build(torch, device, specs=SPECS, seed=0):
    from dfttest2_b200 import synth
    from dfttest2_b200.autograd import frame_planes
    from dfttest2_b200.plugin import Filter

    items, calls, pairs = [], [], []
    for i, (w, h, n, fmt, kw) in enumerate(specs):
        args = plugin_arguments(**kw)
        flt = Filter(device_id=0, **args)
        planes = synth.make_clip_device(fmt, w, h, n, seed * 100 + i, 0.04, device)
        arrs = []
        for src in planes:
            ob, os_ = torch.empty_like(src), torch.empty_like(src)
            items.append((flt, src, ob, fmt.sample_type, fmt.bits_per_sample))
            arrs.append(frame_planes(src[None], os_[None], args["radius"]))
            pairs.append((src, ob, os_, fmt, args))
        calls.append((flt, arrs, fmt))
    return items, calls, pairs


def _sequential(torch, calls):
    import ctypes

    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    for flt, arrs, fmt in calls:
        for a in arrs:
            _lib.check(lib.dfttest2_b200_process_planes(flt.handle, a, len(a), fmt.sample_type, fmt.bits_per_sample,
                                                        ctypes.c_void_p(st)))


def _value(torch, x):
    # 16-bit samples are int16 tensors holding the unsigned bit pattern
    return (x.to(torch.int32) & 0xFFFF if x.dtype == torch.int16 else x).to(torch.float32)


def _compare(torch, pairs):
    for src, ob, os_, fmt, _ in pairs:
        d = (_value(torch, ob) - _value(torch, os_)).abs().max().item()
        if fmt.sample_type == 1:
            assert d <= 2e-5, d
        else:
            assert d <= 1, d


@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_sequential_calls(tune, cuda_device):
    import torch

    from dfttest2_b200.batch import Batch

    items, calls, pairs = _build(torch, cuda_device)
    _sequential(torch, calls)
    b = Batch(items, tune=tune)
    try:
        launches, desc = b.describe()
        groups = desc.strip().split("\n")
        print(desc)
        assert 1 <= len(groups) <= len(SPECS)
        assert launches >= len(groups)
        if tune:
            assert all(("ms" in g) or ("cached" in g) for g in groups)
        b.run()
        torch.cuda.synchronize()
        _compare(torch, pairs)
        first = [ob.clone() for _, ob, _, _, _ in pairs]
        for _, ob, _, _, _ in pairs:
            ob.zero_()
        b.run()  # graph replay: identical
        torch.cuda.synchronize()
        for f, (_, ob, _, _, _) in zip(first, pairs):
            assert torch.equal(f, ob)
    finally:
        b.close()


def test_batch_against_fp64_oracle(cuda_device):
    import torch

    from dfttest2_b200.batch import Batch

    specs = [SPECS[0], SPECS[1], SPECS[5]]
    items, _, pairs = _build(torch, cuda_device, specs, seed=3)
    b = Batch(items, tune=False)
    b.run()
    torch.cuda.synchronize()
    b.close()
    for src, ob, _, fmt, args in pairs[:2] + pairs[-1:]:
        r = args["radius"]
        x = src.cpu().numpy()
        y = ob.cpu().numpy()
        if fmt.sample_type == 0 and fmt.bits_per_sample == 16:
            x, y = x.view(np.uint16), y.view(np.uint16)
        n = x.shape[0]
        for k in (0, n - 1):
            ref = O.fp64_plane(O.clip_frames(x, k, r), args, fmt.bits_per_sample if fmt.sample_type == 0 else 32)
            if fmt.sample_type == 1:
                assert np.abs(y[k].astype(np.float64) - ref).max() <= 2e-5
            else:
                q = O.quantize(ref, y.dtype, fmt.bits_per_sample)
                d = np.abs(y[k].astype(np.int64) - q.astype(np.int64))
                assert d.max() <= 1 and (d == 0).mean() > 0.98


def test_batch_rejects_bad_clips(cuda_device):
    import torch

    from dfttest2_b200.batch import Batch
    from dfttest2_b200.plugin import Filter

    flt = Filter(device_id=0, **plugin_arguments(sbsize=32, sosize=24, tbsize=1))
    tiny = torch.zeros((2, 20, 20), dtype=torch.float32, device=cuda_device)
    with pytest.raises(_lib.Error, match="too small"):
        Batch([(flt, tiny, torch.empty_like(tiny), 1, 32)])
    ok = torch.zeros((2, 64, 64), dtype=torch.float32, device=cuda_device)
    with pytest.raises(_lib.Error, match="32-bit float"):
        Batch([(flt, ok, torch.empty_like(ok), 1, 16)])
    with pytest.raises(_lib.Error):
        Batch([])
    flt.close()

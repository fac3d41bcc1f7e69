"""Tensor-core form of the block transforms (dfttest2_b200_set_precision):
error of each precision mode against the FP64 oracle, on float and 16-bit
planes, for every supported (block size, temporal size).

Stated bounds (max abs error, 0..1 sample scale, ~N(0.5, 0.15) content):
TC_BF16X3 (bf16 hi + lo, three products) 5e-5; TC_TF32 3e-3; TC_BF16 3e-2.
The plain FP32 path stays within 2e-5."""
import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BOUND = {"tc_bf16x3": 5e-5, "tc_tf32": 3e-3, "tc_bf16": 3e-2}
SHAPES = [(16, 1, 96, 72), (16, 3, 96, 72), (32, 1, 128, 96)]


def _run(torch, flt, clip, st, bits):
    dev = torch.from_numpy(clip).cuda(0)
    out = flt.process_clip_device(dev, st, bits)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"B{s[0]}T{s[1]}")
@pytest.mark.parametrize("mode", list(BOUND))
def test_tc_float_error_vs_fp64(shape, mode, cuda_device):
    import torch

    from dfttest2_b200.plugin import Filter

    B, T, W, H = shape
    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=B, sosize=B * 3 // 4, tbsize=T)
    rng = np.random.default_rng(B + T)
    clip = np.clip(0.5 + 0.15 * rng.standard_normal((4, H, W)), 0, 1).astype(np.float32)
    flt = Filter(device_id=0, **args)
    try:
        plain = _run(torch, flt, clip, 1, 32)
        flt.set_precision(mode)
        tc = _run(torch, flt, clip, 1, 32)
        flt.set_precision("fp32")
        again = _run(torch, flt, clip, 1, 32)
    finally:
        flt.close()
    assert np.array_equal(plain, again)
    r = args["radius"]
    worst_tc, worst_plain = 0.0, 0.0
    for n in range(clip.shape[0]):
        ref = O.fp64_plane(O.clip_frames(clip, n, r), args, 32)
        worst_tc = max(worst_tc, float(np.abs(tc[n] - ref).max()))
        worst_plain = max(worst_plain, float(np.abs(plain[n] - ref).max()))
    psnr = 10 * np.log10(1.0 / max(worst_tc, 1e-30) ** 2)
    print(f"B{B} T{T} {mode}: max abs {worst_tc:.3e} (plain fp32 {worst_plain:.3e}), PSNR(max) {psnr:.1f} dB")
    assert worst_plain <= 2e-5
    assert worst_tc <= BOUND[mode]


def test_tc_bf16x3_16bit_lsb(cuda_device):
    """1080p-like 16-bit content on the headline arguments: LSB error of the
    three-product bf16 form against the quantised FP64 oracle."""
    import torch

    from dfttest2_b200.plugin import Filter

    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3)
    rng = np.random.default_rng(7)
    v = np.clip(0.5 + 0.15 * rng.standard_normal((4, 120, 160)), 0, 1)
    clip = np.round(v * 65535).astype(np.uint16)
    flt = Filter(device_id=0, **args)
    try:
        flt.set_precision("tc_bf16x3")
        out = _run(torch, flt, clip.view(np.int16), 0, 16).view(np.uint16)
    finally:
        flt.close()
    d_all = []
    for n in range(4):
        ref = O.quantize(O.fp64_plane(O.clip_frames(clip, n, 1), args, 16), np.uint16, 16)
        d_all.append(np.abs(out[n].astype(np.int64) - ref.astype(np.int64)))
    d = np.concatenate([x.ravel() for x in d_all])
    print(f"tc_bf16x3 16-bit: max {d.max()} LSB, exact {np.mean(d == 0):.4f}, <=1 LSB {np.mean(d <= 1):.6f}")
    assert d.max() <= 1


def test_tc_rejects_unsupported_arguments(cuda_device):
    from dfttest2_b200 import _lib
    from dfttest2_b200.plugin import Filter

    flt = Filter(device_id=0, **plugin_arguments(sbsize=8, sosize=6, tbsize=3))
    with pytest.raises(_lib.Error, match="tensor-core form supports"):
        flt.set_precision("tc_bf16x3")
    with pytest.raises(_lib.Error, match="unknown precision"):
        flt.set_precision("fp8")
    flt.close()

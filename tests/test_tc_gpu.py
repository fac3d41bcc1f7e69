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

BOUND = {"tc_fp16x3": 2e-5, "tc_bf16x3": 5e-5, "tc_tf32": 3e-3, "tc_bf16": 3e-2}
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
    if mode == "tc_fp16x3" and B != 16:
        pytest.skip("the fp16 split form is the strip form: block_size 16")
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


@pytest.mark.parametrize("mode", ["tc_fp16x3", "tc_bf16x3"])
def test_tc_split_16bit_lsb(mode, cuda_device):
    """The split-product strip form against the quantised FP64 oracle on
    16-bit content: within 1 LSB; fp16 hi/lo keeps >= 98 % exact."""
    import torch

    from dfttest2_b200.plugin import Filter

    args = plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3)
    rng = np.random.default_rng(11)
    clip = np.round(np.clip(0.5 + 0.15 * rng.standard_normal((4, 120, 200)), 0, 1) * 65535).astype(np.uint16)
    flt = Filter(device_id=0, **args)
    try:
        flt.set_precision(mode)
        out = _run(torch, flt, clip.view(np.int16), 0, 16).view(np.uint16)
        flt.check()
    finally:
        flt.close()
    d = np.concatenate([np.abs(out[n].astype(np.int64) - O.quantize(O.fp64_plane(O.clip_frames(clip, n, 1), args, 16),
                                                                        np.uint16, 16).astype(np.int64)).ravel()
                        for n in range(4)])
    print(f"{mode} 16-bit: max {d.max()} LSB, exact {np.mean(d == 0):.4f}")
    assert d.max() <= 1
    if mode == "tc_fp16x3":
        assert np.mean(d == 0) >= 0.98


# (block step, radius, sample format, filter type, plane size): strips, segments, seams,
# clip ends, odd sizes and the general filter class of the strip form
STRIP_CASES = [
    (4, 1, "u16", 0, (360, 200)), (4, 1, "u8", 0, (97, 61)), (4, 1, "f32", 0, (250, 130)),
    (4, 0, "u16", 0, (180, 90)), (2, 1, "u16", 0, (150, 70)), (1, 1, "f32", 0, (70, 40)),
    (4, 1, "f32", 1, (200, 100)), (4, 1, "f32", 2, (130, 90)), (4, 1, "f32", 4, (140, 80)),
]


@pytest.mark.parametrize("case", STRIP_CASES, ids=lambda c: f"S{c[0]}r{c[1]}{c[2]}ft{c[3]}_{c[4][0]}x{c[4][1]}")
def test_strip_form_matches_fp32(case, cuda_device):
    """Strip form (tc_fp16x3) against the FP32 kernel on the same frames, every
    frame of a 5-frame clip (both clip ends): float max abs <= 2e-5 of full
    scale, integers within 1 LSB."""
    import torch

    from dfttest2_b200.plugin import Filter

    S, r, kind, ft, (W, H) = case
    args = plugin_arguments(ftype=ft, sigma=8.0, sigma2=4.0, pmin=1.0, pmax=400.0, sbsize=16, sosize=16 - S,
                            tbsize=2 * r + 1)
    rng = np.random.default_rng(S * 100 + W)
    v = np.clip(0.5 + 0.2 * rng.standard_normal((5, H, W)), 0, 1)
    if kind == "f32":
        clip, st, bits = v.astype(np.float32), 1, 32
    elif kind == "u16":
        clip, st, bits = np.round(v * 65535).astype(np.uint16).view(np.int16), 0, 16
    else:
        clip, st, bits = np.round(v * 255).astype(np.uint8), 0, 8
    flt = Filter(device_id=0, **args)
    try:
        plain = _run(torch, flt, clip, st, bits)
        flt.set_precision("tc_fp16x3")
        tc = _run(torch, flt, clip, st, bits)
        flt.check()
    finally:
        flt.close()
    if kind == "f32":
        d = float(np.abs(tc - plain).max())
        print(f"strip form {case}: max abs {d:.3e}")
        assert d <= 2e-5
    else:
        d = np.abs(tc.astype(np.int64) - plain.astype(np.int64)) if kind == "u8" else \
            np.abs(tc.view(np.uint16).astype(np.int64) - plain.view(np.uint16).astype(np.int64))
        print(f"strip form {case}: max {d.max()} LSB, exact {np.mean(d == 0):.4f}")
        assert d.max() <= 1


def test_tc_rejects_unsupported_arguments(cuda_device):
    from dfttest2_b200 import _lib
    from dfttest2_b200.plugin import Filter

    flt = Filter(device_id=0, **plugin_arguments(sbsize=8, sosize=6, tbsize=3))
    with pytest.raises(_lib.Error, match="tensor-core form supports"):
        flt.set_precision("tc_bf16x3")
    with pytest.raises(_lib.Error, match="strip form needs block_size 16"):
        flt.set_precision("tc_fp16x3")
    with pytest.raises(_lib.Error, match="unknown precision"):
        flt.set_precision("fp8")
    flt.close()

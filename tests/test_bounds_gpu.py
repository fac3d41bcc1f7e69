"""Memory-safety checks of the kernels without a sanitizer.

* Guard bands: every plane is written into a device buffer whose rows are
  wider than the plane and which has guard rows above and below, all filled
  with a canary byte; after filtering, every byte outside the plane must
  still hold the canary.  Odd plane sizes, every block size / temporal size,
  sample types u8 / u16 / f32, row offsets that defeat the vector stores and
  the TMA staging (and aligned ones that use them).  Outputs must equal a
  run on dense planes bit for bit.  The FP32 kernels and the tensor-core
  strip form.
* The checked build (libdfttest2_b200_checked.so, -DDFT_CHECKS): the unit
  and fix-up kernels test every ring, staging, block-buffer, band-record and
  output index before the access, the strip form its band-record indices,
  and a failing test records kernel error 3 instead of the access; the same
  cases (both forms) run through it in a child process (the library is
  chosen at load time) and dfttest2_b200_check must report nothing.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter

pytestmark = pytest.mark.gpu

CANARY = 0xA5
SHAPES = [(8, 6, 1), (8, 4, 3), (8, 6, 7), (16, 12, 3), (16, 8, 5), (16, 12, 7), (16, 0, 3), (32, 24, 1),
          (32, 24, 3), (32, 28, 5), (32, 24, 5), (32, 16, 5), (32, 31, 3), (32, 24, 7)]
SIZES = [(71, 53), (130, 97)]
KINDS = [(np.uint8, 0, 8), (np.uint16, 0, 16), (np.float32, 1, 32)]
GUARD_ROWS = 3


def _clip(rng, n, h, w, dtype, bits):
    x = np.clip(0.5 + 0.2 * rng.standard_normal((n, h, w)), 0, 1)
    return x.astype(np.float32) if dtype == np.float32 else np.round(x * ((1 << bits) - 1)).astype(dtype)


def _run_guarded(flt, clip, st, bits, aligned, torch):
    """Filters every frame of `clip` into guard-banded buffers; returns
    (outputs, intact) where intact says every guard byte kept the canary.
    aligned: rows start on 16-byte boundaries (TMA staging, vector stores);
    else one sample of guard before each row and odd row strides."""
    n, h, w = clip.shape
    esz = clip.dtype.itemsize
    if aligned:
        xoff = 16 // esz
        stride = w * esz + 16
        stride += (-stride) % 16
    else:
        xoff = 1
        stride = w * esz + 37
        stride += (-stride) % esz
    rows = h + 2 * GUARD_ROWS
    src = torch.from_numpy(clip.view(np.uint8).reshape(n, h, w * esz)).cuda()
    src_strided = torch.zeros((n, h, stride), dtype=torch.uint8, device="cuda")
    src_strided[:, :, xoff * esz:xoff * esz + w * esz] = src
    frame_bytes = rows * stride + 64  # 64 guard bytes after the last guard row
    dst = torch.full((n, frame_bytes), CANARY, dtype=torch.uint8, device="cuda")
    r = flt.radius
    planes = []
    for i in range(n):
        ptrs = [src_strided[min(max(i - r + t, 0), n - 1)].data_ptr() + xoff * esz for t in range(2 * r + 1)]
        planes.append(dict(src=ptrs, src_stride=stride, dst=dst[i].data_ptr() + GUARD_ROWS * stride + xoff * esz,
                           dst_stride=stride, width=w, height=h))
    flt.process_planes_device(planes, st, bits, torch.cuda.current_stream().cuda_stream)
    flt.check()
    d = dst.cpu().numpy()
    inside = np.zeros(d.shape, bool)
    starts = []
    for y in range(h):
        s0 = (GUARD_ROWS + y) * stride + xoff * esz
        inside[:, s0:s0 + w * esz] = True
        starts.append(s0)
    intact = bool(np.all(d[~inside] == CANARY))
    out = np.stack([np.stack([d[i, s0:s0 + w * esz] for s0 in starts]).view(clip.dtype) for i in range(n)])
    return out, intact


# the tensor-core strip form (16x16 blocks, block steps 1, 2, 4, radius 0 or 1)
STRIP_SHAPES = [(16, 12, 3), (16, 14, 3), (16, 15, 1), (16, 12, 1)]


@pytest.mark.parametrize("B,sosize,tb,precision", [s + ("fp32",) for s in SHAPES] +
                         [s + ("tc_fp16x3",) for s in STRIP_SHAPES])
def test_guard_bands(B, sosize, tb, precision, cuda_device):
    import torch

    args = plugin_arguments(ftype=0, sigma=6.0, sbsize=B, sosize=sosize, tbsize=tb)
    rng = np.random.default_rng(B * 100 + sosize * 10 + tb)
    flt = Filter(device_id=0, **args)
    flt.set_precision(precision)
    try:
        for (w, h) in SIZES:
            for dtype, st, bits in KINDS:
                clip = _clip(rng, 3, h, w, dtype, bits)
                dense = flt.process_clip_device(torch.from_numpy(clip.view(np.uint8)).cuda().view(
                    {1: torch.uint8, 2: torch.int16, 4: torch.float32}[clip.dtype.itemsize]), st, bits)
                flt.check()
                dense = dense.cpu().numpy().view(clip.dtype)
                for aligned in (True, False):
                    out, intact = _run_guarded(flt, clip, st, bits, aligned, torch)
                    what = f"B{B} sosize {sosize} T{tb} {precision} {w}x{h} {dtype.__name__} aligned {aligned}"
                    assert intact, f"guard bytes overwritten: {what}"
                    assert np.array_equal(out.view(np.uint8), dense.view(np.uint8)), f"{what}: differs from dense planes"
    finally:
        flt.close()


CHILD = r"""
import sys
sys.path[:0] = [{root!r}, {pkg!r}]
import numpy as np, torch
from dfttest2_b200 import _lib
assert _lib.LIB_PATH.endswith("libdfttest2_b200_checked.so"), _lib.LIB_PATH
from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter
from oracle import oracle as O
rng = np.random.default_rng(3)
worst = 0
for B, sosize, tb, precision in {shapes!r}:
    args = plugin_arguments(ftype=0, sigma=6.0, sbsize=B, sosize=sosize, tbsize=tb)
    flt = Filter(device_id=0, **args)
    flt.set_precision(precision)
    for (w, h) in {sizes!r}:
        x = np.round(np.clip(0.5 + 0.2 * rng.standard_normal((3, h, w)), 0, 1) * 65535).astype(np.uint16)
        out = flt.process_clip_device(torch.from_numpy(x.view(np.int16)).cuda(), 0, 16)
        flt.check()  # raises on kernel error 3 (an index outside its buffer)
        got = out.cpu().numpy().view(np.uint16)[1]
        ref = O.quantize(O.fp64_plane(O.clip_frames(x, 1, args["radius"]), args, 16), np.uint16, 16)
        worst = max(worst, int(np.abs(got.astype(np.int64) - ref.astype(np.int64)).max()))
        host = flt.process_clip_host(x, 0, 16)  # host pipeline (reads the word itself)
    flt.close()
print("checked build: max", worst, "LSB")
assert worst <= 1
"""


def test_checked_build_reports_no_out_of_range_index(cuda_device):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "vs-dfttest2_b200")
    lib = os.path.join(pkg, "dfttest2_b200", "libdfttest2_b200_checked.so")
    if not os.path.exists(lib):
        pytest.fail("the checked build is missing: run `make checked` in vs-dfttest2_b200/")
    shapes = [s + ("fp32",) for s in SHAPES] + [s + ("tc_fp16x3",) for s in STRIP_SHAPES]
    code = CHILD.format(root=root, pkg=pkg, shapes=shapes, sizes=SIZES)
    env = dict(os.environ, DFTTEST2_B200_LIB="checked")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    print(res.stdout[-2000:], res.stderr[-2000:])
    assert res.returncode == 0

"""Precision report of the block-transform arithmetic (FP32 codelets and the
tensor-core forms) against an FP64 reference of the same pipeline, on the
4K precision workload: GRAYS float32 3840x2160, 32 frames, seeded drifting
sinusoids + Gaussian noise sigma 0.03, two setups (sbsize 16 / sosize 12 /
tbsize 3 and sbsize 32 / sosize 24 / tbsize 1), ftype 0, sigma 8.

The FP64 reference is oracle/torch_ref.py (float64 torch on the GPU; it
matches the FP64 C oracle to 1e-15).  Max-abs error and PSNR (peak 1.0,
MSE over all frames) are printed per setup and mode; the bounds asserted
are those stated for each mode in tests/test_tc_gpu.py.
"""
import os

import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from oracle import torch_ref as TR

pytestmark = pytest.mark.gpu

SETUPS = [dict(sbsize=16, sosize=12, tbsize=3), dict(sbsize=32, sosize=24, tbsize=1)]
MODES = {"fp32": 2e-5, "tc_fp16x3": 2e-5, "tc_bf16x3": 5e-5, "tc_tf32": 3e-3, "tc_bf16": 3e-2}


def test_precision_report_4k(cuda_device):
    import torch

    from dfttest2_b200 import synth
    from dfttest2_b200.clip import GRAYS
    from dfttest2_b200.plugin import Filter

    clip = synth.make_clip_device(GRAYS, 3840, 2160, 32, 2024, 0.03, cuda_device)[0]
    lines = []
    for setup in SETUPS:
        args = plugin_arguments(ftype=0, sigma=8.0, **setup)
        ref = torch.empty((clip.shape[0],) + tuple(clip.shape[1:]), dtype=torch.float64, device=cuda_device)
        r = args["radius"]
        n = clip.shape[0]
        x64 = clip.double()
        for k in range(n):
            idx = [min(max(k - r + t, 0), n - 1) for t in range(2 * r + 1)]
            ref[k] = TR.dfttest_plane(x64[idx], args)
        flt = Filter(device_id=0, **args)
        try:
            for mode, bound in MODES.items():
                if mode == "tc_fp16x3" and setup["sbsize"] != 16:
                    continue  # the fp16 split runs the strip form: 16x16 blocks
                flt.set_precision(mode)
                out = flt.process_clip_device(clip, 1, 32)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                flt.process_clip_device(clip, 1, 32, out=out)
                e1.record()
                torch.cuda.synchronize()
                err = (out.double() - ref).abs()
                mx = err.max().item()
                mse = (err * err).mean().item()
                psnr = 10 * np.log10(1.0 / max(mse, 1e-300))
                lines.append(f"sbsize {setup['sbsize']} tbsize {setup['tbsize']} {mode:10s} max-abs {mx:.3e} "
                             f"PSNR {psnr:6.1f} dB  {n / (e0.elapsed_time(e1) * 1e-3):8.1f} frames/s")
                assert mx <= bound, lines[-1]
        finally:
            flt.close()
    print("\n" + "\n".join(lines))
    # DFTTEST2_B200_REPORT_DIR=<dir>: the report also goes to <dir>/precision_report_4k.txt
    out_dir = os.environ.get("DFTTEST2_B200_REPORT_DIR")
    if out_dir:
        with open(os.path.join(out_dir, "precision_report_4k.txt"), "w") as f:
            f.write("\n".join(lines) + "\n")

"""Parity with the reference's own GPU algorithm for general block sizes.

dfttest2_cpu accepts only 16x16 blocks; block sizes 8 and 32 exist in the
reference only on its cuFFT backend (dfttest2_cuda: im2col, cuFFT R2C,
frequency filter, cuFFT C2R, col2im; cuda_source/kernels.cu:84-406 and
cuda_source/source.cpp:515-662).  oracle/_ref/libdfttest_ref_cufft.so is
that backend's kernels.cu compiled unchanged, driven like source.cpp by
oracle/ref_cufft.cu.  Bars as for the CPU reference: float planes max-abs
<= 2e-5 of full scale, integer planes within 1 LSB with the exact-match
fraction >= 0.99.
"""
import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_cufft_available(), reason="oracle/_ref cuFFT checker not built")]

CASES = [
    # B, sosize, tbsize, ftype, full sigma array
    (8, 6, 3, 0, False), (8, 6, 1, 0, False), (8, 4, 5, 1, True), (8, 6, 7, 0, True),
    (32, 24, 1, 0, False), (32, 24, 3, 0, True), (32, 16, 5, 2, False), (32, 28, 3, 0, False),
    (16, 12, 3, 0, False), (16, 8, 5, 4, True),
]
FORMATS = [(np.uint16, 16), (np.float32, 32), (np.uint8, 8)]


@pytest.mark.parametrize("B,sosize,tb,ftype,full", CASES)
@pytest.mark.parametrize("dtype,bits", FORMATS)
def test_against_reference_cufft_path(B, sosize, tb, ftype, full, dtype, bits, cuda_device):
    rng = np.random.default_rng(B * 31 + sosize + tb)
    w, h = 3 * B + 29, 2 * B + 37
    x = np.clip(0.5 + 0.2 * rng.standard_normal((tb, h, w)), 0, 1)
    frames = x.astype(np.float32) if dtype == np.float32 else np.round(x * ((1 << bits) - 1)).astype(dtype)
    sigma = 0.9 if ftype in (2, 3, 4) else 6.0
    args = plugin_arguments(ftype=ftype, sigma=sigma, pmin=1.0, pmax=300.0, sbsize=B, sosize=sosize, tbsize=tb,
                            full_sigma=full)
    ref = O.ref_cufft_plane(list(frames), args, bits)
    flt = Filter(device_id=0, **args)
    try:
        out = flt.process_plane_host(list(frames), 1 if dtype == np.float32 else 0, bits)
    finally:
        flt.close()
    if dtype == np.float32:
        err = float(np.abs(out.astype(np.float64) - ref.astype(np.float64)).max())
        print(f"B{B} sosize {sosize} T{tb} ft{ftype} float: max-abs {err:.2e}")
        assert err <= 2e-5
    else:
        d = np.abs(out.astype(np.int64) - ref.astype(np.int64))
        print(f"B{B} sosize {sosize} T{tb} ft{ftype} {dtype.__name__}: max {d.max()} LSB, exact {np.mean(d == 0):.4f}")
        assert d.max() <= 1 and np.mean(d == 0) >= 0.99

"""Pinning the FP64 oracle (oracle/dfttest_oracle.c) against the reference.

The reference has no tests or golden vectors of its own, so parity is pinned
on the reference's own CPU math: committed fixtures generated with it
(tests/golden/gen_golden.py) and, when available, the live build in
oracle/_ref.  Tolerances: float planes 1e-5 of full scale (the oracle is FP64,
the reference FP32), integer planes within 1 LSB with >= 99% exact.
"""
import numpy as np
import pytest

from conftest import golden_planes, load_case, load_plane
from oracle import oracle as O


def _compare(ref_out, f64, bits):
    if ref_out.dtype == np.float32:
        err = np.abs(ref_out.astype(np.float64) - f64).max()
        assert err <= 1e-5, err
        return 1.0
    q = O.quantize(f64, ref_out.dtype, bits).astype(np.int64)
    d = np.abs(q - ref_out.astype(np.int64))
    assert d.max() <= 1
    exact = float(np.mean(d == 0))
    assert exact >= 0.99, exact
    return exact


@pytest.mark.parametrize("case", golden_planes())
def test_fp64_oracle_matches_reference_fixture(case):
    rec, args = load_case(case)
    frames, out = load_plane(case)
    f64 = O.fp64_plane(list(frames), args, rec["bits"], synthesis_slice=2 * args["radius"])
    _compare(out, f64, rec["bits"])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("dtype,bits", [(np.float32, 32), (np.uint16, 16), (np.uint8, 8), (np.uint16, 10)])
@pytest.mark.parametrize("tb,ftype,swin,twin,sosize", [(3, 0, 0, 7, 12), (1, 0, 1, 7, 8), (5, 1, 2, 0, 12),
                                                        (7, 0, 4, 9, 12), (3, 4, 6, 7, 4), (3, 5, 11, 3, 12)])
def test_fp64_oracle_matches_reference_build(dtype, bits, tb, ftype, swin, twin, sosize):
    from dfttest2_b200.frontend import plugin_arguments
    rng = np.random.default_rng(tb * 100 + ftype)
    h, w = 53, 71
    n = tb
    base = rng.random((n, h, w))
    if dtype == np.float32:
        frames = base.astype(np.float32)
    else:
        frames = np.round(base * ((1 << bits) - 1)).astype(dtype)
    f0 = 0.7 if ftype == 5 else 1.0
    args = plugin_arguments(ftype=min(ftype, 4), f0beta=f0, sigma=4.0, pmin=1.0, pmax=300.0, tbsize=tb, swin=swin,
                            twin=twin, sosize=sosize, full_sigma=True)
    src = list(frames)
    ref = O.ref_plane(src, args, bits)
    f64 = O.fp64_plane(src, args, bits, synthesis_slice=2 * args["radius"])
    _compare(ref, f64, bits)


def test_fp64_oracle_identity():
    # multiplier 1 everywhere with a rectangular temporal window reproduces the input
    from dfttest2_b200.frontend import plugin_arguments
    rng = np.random.default_rng(3)
    frames = rng.random((3, 40, 56)).astype(np.float32)
    args = plugin_arguments(ftype=2, sigma=1.0, tbsize=3, full_sigma=True)
    f64 = O.fp64_plane(list(frames), args, 32)
    # the window table is FP32 (as the plugin stores it), so the identity holds to ~1e-7
    assert np.abs(f64 - frames[1]).max() < 2e-7

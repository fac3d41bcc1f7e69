"""Host logic: window / sigma construction and parameter translation against
the reference's own Python (recorded in tests/golden/)."""
import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases, load_case
from dfttest2_b200 import GRAYS, YUV420P16, Backend, Clip, DFTTest, select_backend
from dfttest2_b200 import helpers
from dfttest2_b200.backends import as_b200
from dfttest2_b200.frontend import plugin_arguments


def _rfftn_rdft(data, shape):
    a = np.asarray(data, dtype=np.float64).reshape(shape)
    out = np.fft.rfftn(a)
    return list(np.stack([out.real, out.imag], axis=-1).ravel())


def test_windows_match_reference_helpers():
    with open(os.path.join(GOLDEN, "helpers.json")) as f:
        ref = json.load(f)
    for key, vals in ref["windows"].items():
        mode, size = map(int, key.split("_"))
        got = [helpers.get_window_value(i + 0.5, size, mode, 2.5) for i in range(size)]
        np.testing.assert_allclose(got, vals, rtol=0, atol=1e-15, err_msg=key)
    for length, vals in ref["locations"].items():
        got = [helpers.get_location(i, int(length)) for i in range(int(length))]
        np.testing.assert_allclose(got, vals, rtol=0, atol=1e-15)
    cases = {"r1_16_4_0_7": (1, 16, 4, 0, 2.5, 7, 2.5), "r2_8_2_4_0": (2, 8, 2, 4, 3.0, 0, 2.5),
             "r0_32_8_9_7": (0, 32, 8, 9, 2.5, 7, 2.5)}
    for key, a in cases.items():
        np.testing.assert_allclose(helpers.get_window(*a), ref["get_window"][key], rtol=0, atol=1e-15)


@pytest.mark.parametrize("case", golden_cases())
def test_plugin_arguments_match_reference_translation(case):
    rec, ref_args = load_case(case)
    kw = dict(rec["dfttest_kwargs"])
    # DFTTest's own sigma-function construction, then DFTTest2's translation
    import dfttest2_b200.frontend as fe

    captured = {}

    def fake_dfttest2(**k):
        captured.update(k)

    real = fe.DFTTest2
    fe.DFTTest2 = fake_dfttest2
    try:
        fmt = GRAYS
        clip = Clip([np.zeros((1, 48, 64), np.float32)], fmt)
        fe.DFTTest(clip, backend=Backend.B200(), **kw)
    finally:
        fe.DFTTest2 = real
    captured.pop("clip")
    captured.pop("planes")
    captured.pop("backend")
    full = rec["backend"] in ("CPU", "GCC")
    got = plugin_arguments(full_sigma=full, rdft=_rfftn_rdft, **captured)
    np.testing.assert_allclose(got["window"], ref_args["window"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(got["sigma"], ref_args["sigma"], rtol=1e-13, atol=0)
    for k in ("sigma2", "pmin", "pmax"):
        assert math.isclose(got[k], ref_args[k], rel_tol=1e-13), k
    for k in ("filter_type", "radius", "block_size", "block_step"):
        assert got[k] == ref_args[k], k
    if ref_args["window_freq"] is not None and (rec["backend"] != "CPU" or got["zero_mean"]):
        np.testing.assert_allclose(got["window_freq"], ref_args["window_freq"], rtol=0, atol=1e-9)


def test_dfttest_validation_messages():
    clip = Clip([np.zeros((2, 32, 32), np.float32)], GRAYS)
    with pytest.raises(ValueError, match="ftype must be 0, 1, 2, 3, or 4"):
        DFTTest(clip, ftype=5)
    with pytest.raises(ValueError, match='"smode" must be 1'):
        DFTTest(clip, smode=0)
    with pytest.raises(ValueError, match="spatial overlap greater than 50%"):
        DFTTest(clip, sbsize=16, sosize=11)
    with pytest.raises(ValueError, match="swin must be between 0 and 11"):
        DFTTest(clip, swin=12)
    with pytest.raises(ValueError, match="multiple of 2"):
        DFTTest(clip, slocation=[0.0, 1.0, 0.5])
    with pytest.raises(ValueError, match='"nlocation" must be None'):
        DFTTest(clip, nlocation=[1, 2, 3, 4])
    with pytest.raises(ValueError, match="invalid radius"):
        DFTTest(clip, tbsize=9, backend=Backend.B200())
    with pytest.raises(RuntimeError, match="No backend are available"):
        DFTTest(clip, tbsize=9)


def test_backend_selection():
    assert isinstance(select_backend(None, 16, 3), Backend.B200)
    assert isinstance(select_backend(None, 32, 1), Backend.B200)
    with pytest.raises(RuntimeError):
        select_backend(None, 12, 3)
    b = as_b200(Backend.NVRTC(device_id=1, num_streams=3))
    assert (b.device_id, b.num_streams) == (1, 3)
    with pytest.raises(TypeError):
        as_b200(Backend.CPU())


def test_clip_container_checks_plane_shapes():
    with pytest.raises(ValueError):
        Clip([np.zeros((2, 32, 32), np.uint16)] * 3, YUV420P16)

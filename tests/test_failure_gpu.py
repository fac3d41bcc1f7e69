"""Kernel failures reach the caller as DFTTEST2_B200_EKERNEL.

The kernels never trap: an internal failure is written to an error word that
the host reads (after its own wait in the host-memory calls, through
dfttest2_b200_check for the asynchronous device calls), as the reference
turns every CUDA failure into setFilterError (cuda_source/source.cpp:124-138).

The failure made here is a bounded wait that runs out: with the wait limit
set to 0, the tensor-core kernel's wait for its products gives up at once;
the kernel then drains the products still in flight with the full limit,
frees its tensor memory and returns early.  Nothing faults: the products are
valid and complete, only the wait is cut short.  Afterwards the same filter
runs normally again.
"""
import numpy as np
import pytest

from dfttest2_b200._lib import Error
from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter

pytestmark = pytest.mark.gpu


def _frames(seed, n=3, h=72, w=96):
    rng = np.random.default_rng(seed)
    return np.round(np.clip(0.5 + 0.2 * rng.standard_normal((n, h, w)), 0, 1) * 65535).astype(np.uint16)


def test_tc_wait_timeout_reports_ekernel_host_path(cuda_device):
    frames = _frames(1)
    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=8.0, tbsize=3))
    try:
        flt.set_precision("tc_bf16x3")
        good = flt.process_plane_host(list(frames), 0, 16)
        flt.set_wait_limit(0)
        with pytest.raises(Error, match="kernel error 2"):
            flt.process_plane_host(list(frames), 0, 16)
        flt.set_wait_limit(-1)
        again = flt.process_plane_host(list(frames), 0, 16)
        flt.check()
    finally:
        flt.close()
    # the tensor-core form sums overlapping blocks with float atomics, whose
    # order varies from run to run: equal within 1 LSB
    assert np.abs(good.astype(np.int64) - again.astype(np.int64)).max() <= 1


def test_tc_wait_timeout_reports_ekernel_device_path(cuda_device):
    import torch

    clip = torch.from_numpy(_frames(2, n=4).view(np.int16)).cuda(0)
    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=8.0, tbsize=3))
    try:
        flt.set_precision("tc_bf16x3")
        good = flt.process_clip_device(clip, 0, 16)
        flt.check()  # nothing reported by a normal run
        flt.set_wait_limit(0)
        flt.process_clip_device(clip, 0, 16)
        with pytest.raises(Error, match="kernel error 2"):
            flt.check()
        flt.check()  # the word was cleared by the report
        flt.set_wait_limit(-1)
        again = flt.process_clip_device(clip, 0, 16)
        flt.check()
        d = ((good.to(torch.int32) & 0xFFFF) - (again.to(torch.int32) & 0xFFFF)).abs().max().item()
        assert d <= 1  # float atomics of the tensor-core form: run-to-run order varies
    finally:
        flt.close()


def test_fp32_paths_report_no_failure(cuda_device):
    frames = _frames(3, n=5)
    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=8.0, tbsize=3))
    try:
        flt.process_clip_host(frames, 0, 16)
        flt.process_plane_host(list(frames[:3]), 0, 16)
        flt.process_frame_host_cached(frames, 2, 0, 0, 16)
        flt.check()
    finally:
        flt.close()

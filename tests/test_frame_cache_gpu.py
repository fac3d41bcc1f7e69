"""Frame-by-frame host path with the device frame cache
(dfttest2_b200_process_plane_host_cached): results equal the uncached
per-plane host path for in-order, shuffled and concurrent requests, for
every plane of a YUV clip and for float planes."""
import threading

import numpy as np
import pytest

from dfttest2_b200.frontend import plugin_arguments
from dfttest2_b200.plugin import Filter

pytestmark = pytest.mark.gpu


def _clip(rng, n, h, w, dtype, peak):
    v = np.clip(0.5 + 0.2 * rng.standard_normal((n, h, w)), 0, 1)
    return v.astype(np.float32) if dtype == np.float32 else np.round(v * peak).astype(dtype)


def _uncached(flt, clip, n, st, bits):
    from oracle import oracle as O

    return flt.process_plane_host(O.clip_frames(clip, n, flt.radius), st, bits)


@pytest.mark.parametrize("order", ["in_order", "shuffled"])
def test_cached_equals_uncached_yuv(order, cuda_device):
    rng = np.random.default_rng(5)
    planes = [_clip(rng, 9, 96, 160, np.uint16, 65535), _clip(rng, 9, 48, 80, np.uint16, 65535),
              _clip(rng, 9, 48, 80, np.uint16, 65535)]
    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=8.0, sbsize=16, sosize=12, tbsize=3))
    try:
        frames = list(range(9))
        if order == "shuffled":
            rng.shuffle(frames)
        for n in frames:
            for p, clip in enumerate(planes):
                got = flt.process_frame_host_cached(clip, n, p, 0, 16)
                assert np.array_equal(got, _uncached(flt, clip, n, 0, 16)), (n, p)
    finally:
        flt.close()


def test_frame_call_equals_uncached_planes(cuda_device):
    """All planes of each frame in one call (one launch) give the per-plane results."""
    rng = np.random.default_rng(7)
    planes = [_clip(rng, 7, 96, 160, np.uint8, 255), _clip(rng, 7, 48, 80, np.uint8, 255),
              _clip(rng, 7, 48, 80, np.uint8, 255)]
    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=6.0, sbsize=16, sosize=12, tbsize=3))
    try:
        for n in (0, 1, 2, 6, 3, 5, 4):
            got = flt.process_frame_planes_host_cached(planes, n, 0, 8)
            for p, clip in enumerate(planes):
                want = _uncached(flt, clip, n, 0, 8)
                d = np.abs(got[p].astype(np.int64) - want.astype(np.int64))
                assert d.max() <= 1 and (d == 0).mean() > 0.99, (n, p)
    finally:
        flt.close()


def test_cached_concurrent_float(cuda_device):
    rng = np.random.default_rng(6)
    clip = _clip(rng, 12, 72, 96, np.float32, 1.0)
    flt = Filter(device_id=0, num_streams=3, **plugin_arguments(ftype=0, sigma=6.0, tbsize=5))
    try:
        want = [_uncached(flt, clip, n, 1, 32) for n in range(12)]
        got = [None] * 12
        errors = []

        def worker(ns):
            try:
                for n in ns:
                    got[n] = flt.process_frame_host_cached(clip, n, 0, 1, 32)
            except Exception as e:  # noqa: BLE001 - reported below
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(list(range(k, 12, 3)),)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        for n in range(12):
            assert np.array_equal(got[n], want[n]), n
    finally:
        flt.close()


def test_cached_call_rejects_bad_planes(cuda_device):
    import ctypes

    from dfttest2_b200 import _lib

    flt = Filter(device_id=0, **plugin_arguments(ftype=0, sigma=8.0, tbsize=3))
    lib = _lib.load()
    try:
        src = np.zeros((72, 96), np.uint16)
        out = np.zeros_like(src)
        pl = _lib.Plane()
        for t in range(3):
            pl.src[t] = src.ctypes.data
        pl.src_stride, pl.dst, pl.dst_stride, pl.width, pl.height = 192, None, 192, 96, 72
        ids = (ctypes.c_int * 3)(0, 0, 1)
        with pytest.raises(_lib.Error, match="null destination"):
            _lib.check(lib.dfttest2_b200_process_plane_host_cached(flt.handle, ctypes.byref(pl), ids, 0, 0, 16))
        pl.dst, pl.src_stride = out.ctypes.data, 100
        with pytest.raises(_lib.Error, match="invalid stride"):
            _lib.check(lib.dfttest2_b200_process_plane_host_cached(flt.handle, ctypes.byref(pl), ids, 0, 0, 16))
    finally:
        flt.close()

"""ctypes binding of the C ABI declared in include/dfttest2_b200.h.

The shared library is built in-tree (``make`` in vs-dfttest2_b200/, or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_ssize_t, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
# DFTTEST2_B200_LIB=checked loads the bounds-checked build (make checked),
# whose kernels record out-of-range indices as kernel error 3
LIB_PATH = os.path.join(_HERE, "libdfttest2_b200_checked.so" if os.environ.get("DFTTEST2_B200_LIB") == "checked"
                        else "libdfttest2_b200.so")

NOALLOC_SCRATCH_BYTES = 8 * 1024 * 1024
OK = 0
EINVAL = 1
ECUDA = 2
ENOMEM = 3
EKERNEL = 4
INTEGER = 0
FLOAT = 1


class Params(ctypes.Structure):
    _fields_ = [
        ("window", POINTER(c_double)),
        ("window_len", c_int),
        ("sigma", POINTER(c_double)),
        ("sigma_len", c_int),
        ("sigma2", c_double),
        ("pmin", c_double),
        ("pmax", c_double),
        ("filter_type", c_int),
        ("radius", c_int),
        ("block_size", c_int),
        ("block_step", c_int),
        ("zero_mean", c_int),
        ("window_freq", POINTER(c_double)),
        ("window_freq_len", c_int),
        ("device_id", c_int),
        ("num_streams", c_int),
        ("synthesis_slice", c_int),
    ]


class Plane(ctypes.Structure):
    _fields_ = [
        ("src", c_void_p * 7),
        ("src_stride", c_ssize_t),
        ("dst", c_void_p),
        ("dst_stride", c_ssize_t),
        ("width", c_int),
        ("height", c_int),
    ]


class GradPlane(ctypes.Structure):
    _fields_ = [
        ("src", c_void_p * 7),
        ("grad_src", c_void_p * 7),
        ("grad_dst", c_void_p),
        ("src_stride", c_ssize_t),
        ("grad_src_stride", c_ssize_t),
        ("grad_dst_stride", c_ssize_t),
        ("width", c_int),
        ("height", c_int),
    ]


class HostPlane(ctypes.Structure):
    """dfttest2_b200_host_plane: one plane of a clip in host memory."""

    _fields_ = [
        ("src", c_void_p),
        ("src_stride", c_ssize_t),
        ("src_frame_bytes", c_ssize_t),
        ("dst", c_void_p),
        ("dst_stride", c_ssize_t),
        ("dst_frame_bytes", c_ssize_t),
        ("width", c_int),
        ("height", c_int),
    ]


class Clip(ctypes.Structure):
    """dfttest2_b200_clip: one device-resident clip of a multi-clip batch."""

    _fields_ = [
        ("filter", c_void_p),
        ("src", c_void_p),
        ("src_stride", c_ssize_t),
        ("src_frame_bytes", c_ssize_t),
        ("dst", c_void_p),
        ("dst_stride", c_ssize_t),
        ("dst_frame_bytes", c_ssize_t),
        ("nframes", c_int),
        ("width", c_int),
        ("height", c_int),
        ("sample_type", c_int),
        ("bits_per_sample", c_int),
    ]


BATCH_TUNE = 1

# dfttest2_b200_set_precision modes
PRECISION = {"fp32": 0, "tc_bf16x3": 1, "tc_tf32": 2, "tc_bf16": 3, "tc_fp16x3": 4}

# every symbol include/dfttest2_b200.h declares, with its ctypes signature
SIGNATURES = {
    "dfttest2_b200_params_init": (None, [POINTER(Params)]),
    "dfttest2_b200_create": (c_int, [POINTER(Params), POINTER(c_void_p)]),
    "dfttest2_b200_free": (None, [c_void_p]),
    "dfttest2_b200_process_planes": (c_int, [c_void_p, POINTER(Plane), c_int, c_int, c_int, c_void_p]),
    "dfttest2_b200_process_plane_host": (c_int, [c_void_p, POINTER(Plane), c_int, c_int]),
    "dfttest2_b200_process_clip_host": (
        c_int,
        [c_void_p, c_void_p, c_ssize_t, c_ssize_t, c_void_p, c_ssize_t, c_ssize_t, c_int, c_int, c_int, c_int, c_int],
    ),
    "dfttest2_b200_process_plane_host_cached": (c_int, [c_void_p, POINTER(Plane), POINTER(c_int), c_int, c_int, c_int]),
    "dfttest2_b200_process_frame_host_cached": (
        c_int, [c_void_p, POINTER(Plane), c_int, POINTER(c_int), POINTER(c_int), c_int, c_int]),
    "dfttest2_b200_process_clip_planes_host": (c_int, [c_void_p, POINTER(HostPlane), c_int, c_int, c_int, c_int]),
    "dfttest2_b200_process_planes_sigma": (c_int, [c_void_p, POINTER(Plane), c_int, c_int, c_int, c_void_p, c_void_p]),
    "dfttest2_b200_backward_planes": (c_int, [c_void_p, POINTER(GradPlane), c_int, c_void_p, c_void_p, c_void_p]),
    "dfttest2_b200_set_precision": (c_int, [c_void_p, c_int]),
    "dfttest2_b200_check": (c_int, [c_void_p]),
    "dfttest2_b200_set_wait_limit": (c_int, [c_void_p, c_int]),
    "dfttest2_b200_noalloc_check": (c_int, [c_int, c_void_p]),
    "dfttest2_b200_batch_create": (c_int, [POINTER(Clip), c_int, c_int, POINTER(c_void_p)]),
    "dfttest2_b200_batch_run": (c_int, [c_void_p, c_void_p]),
    "dfttest2_b200_batch_describe": (c_int, [c_void_p, ctypes.c_char_p, c_int]),
    "dfttest2_b200_batch_free": (None, [c_void_p]),
    "dfttest2_b200_process_plane_noalloc": (c_int, [POINTER(Params), POINTER(Plane), c_int, c_int, c_void_p]),
    "dfttest2_b200_rdft": (c_int, [POINTER(c_double), c_int, POINTER(c_int), c_int, POINTER(c_double), c_int]),
    "dfttest2_b200_version": (c_char_p, []),
    "dfttest2_b200_last_error": (c_char_p, []),
}

_lib = None


class Error(Exception):
    """Raised for every failing call (mirrors vapoursynth.Error)."""


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is not built: run `make` in vs-dfttest2_b200/ or __graft_entry__.build() "
            "(there is no CPU fallback)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != OK:
        msg = load().dfttest2_b200_last_error().decode()
        raise Error(msg or f"dfttest2_b200 error {rc}")


def as_double_array(values):
    arr = (c_double * len(values))(*[float(v) for v in values])
    return arr

"""Backend selection, mirroring the reference's ``python/backends.py``.

``Backend.B200`` is the new entry; it takes the same options as the
reference's NVRTC backend (``device_id``, ``num_streams``).  The reference's
other backend classes are kept by name so that scripts that name them keep
working: the CUDA ones (NVRTC, cuFFT) run on this implementation with their
device, the CPU / AMD ones raise because this package does not carry them.
``select_backend`` puts B200 first for every block size it supports
(python/backends.py:39-63 lists NVRTC first for sbsize 16).
"""
from __future__ import annotations

from dataclasses import dataclass


class Backend:
    @dataclass(frozen=False)
    class B200:
        device_id: int = 0
        num_streams: int = 1

    @dataclass(frozen=False)
    class cuFFT:
        device_id: int = 0
        in_place: bool = True

    @dataclass(frozen=False)
    class NVRTC:
        device_id: int = 0
        num_streams: int = 1

    @dataclass(frozen=False)
    class CPU:
        opt: int = 0

    @dataclass(frozen=False)
    class GCC: ...

    @dataclass(frozen=False)
    class hipFFT:
        device_id: int = 0
        in_place: bool = True

    @dataclass(frozen=False)
    class HIPRTC:
        device_id: int = 0
        num_streams: int = 1


SUPPORTED_BLOCK_SIZES = (8, 16, 32)
SUPPORTED_TBSIZE = (1, 3, 5, 7)


def select_backend(backend, sbsize: int, tbsize: int):
    if backend is not None:
        return backend
    if sbsize in SUPPORTED_BLOCK_SIZES and tbsize in SUPPORTED_TBSIZE:
        return Backend.B200()
    raise RuntimeError("No backend are available")


def as_b200(backend) -> "Backend.B200":
    """Map a backend instance onto the B200 implementation (or raise)."""
    inst = backend() if isinstance(backend, type) else backend
    if isinstance(inst, Backend.B200):
        return inst
    if isinstance(inst, Backend.NVRTC):
        return Backend.B200(device_id=inst.device_id, num_streams=inst.num_streams)
    if isinstance(inst, Backend.cuFFT):
        return Backend.B200(device_id=inst.device_id)
    raise TypeError(f"Unknown backend: {inst}")

"""dfttest2_b200: DFTTest's per-plane denoising hot path on B200 (sm_100a).

Public API (mirrors the reference vs-dfttest2 Python package):

* ``DFTTest`` / ``DFTTest2``   user-level filter (python/dfttest2.py)
* ``Backend`` / ``select_backend``  backend table (python/backends.py)
* ``dfttest2_b200``            plugin namespace: DFTTest / RDFT / Version
* ``Clip`` and formats         stand-in for a VapourSynth clip
"""
from .backends import Backend, select_backend
from .clip import GRAY8, GRAY16, GRAYS, YUV420P8, YUV420P10, YUV420P16, YUV444PS, Clip, VideoFormat
from .frontend import DFTTest, DFTTest2, plugin_arguments
from .plugin import Error, Filter, dfttest2_b200

__all__ = [
    "Backend", "select_backend", "Clip", "VideoFormat", "GRAY8", "GRAY16", "GRAYS", "YUV420P8", "YUV420P10",
    "YUV420P16", "YUV444PS", "DFTTest", "DFTTest2", "plugin_arguments", "Error", "Filter", "dfttest2_b200",
]

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "vs-dfttest2_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_case(name):
    """Recorded plugin arguments of a golden case, with the plugin defaults
    filled in (the CPU backend always runs zero-mean, block_step defaults to
    block_size)."""
    with open(os.path.join(GOLDEN, f"args_{name}.json")) as f:
        rec = json.load(f)
    args = dict(rec["args"])
    # backend-specific options of the reference plugins (CPU ISA dispatch,
    # cuFFT in-place, device selection) are not filter arguments
    for k in ("opt", "in_place", "device_id", "num_streams"):
        args.pop(k, None)
    args.setdefault("zero_mean", 1)
    args.setdefault("window_freq", None)
    args.setdefault("radius", 0)
    args.setdefault("block_size", 16)
    args.setdefault("block_step", args["block_size"])
    return rec, args


def golden_cases():
    return sorted(f[5:-5] for f in os.listdir(GOLDEN) if f.startswith("args_") and f.endswith(".json"))


def golden_planes():
    return sorted(f[6:-4] for f in os.listdir(GOLDEN) if f.startswith("plane_") and f.endswith(".npz"))


def load_plane(name):
    d = np.load(os.path.join(GOLDEN, f"plane_{name}.npz"))
    return d["frames"], d["out"]


@pytest.fixture(scope="session")
def cuda_device():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")

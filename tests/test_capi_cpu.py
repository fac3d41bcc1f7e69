"""C ABI without a GPU: symbols, argument validation and RDFT (host-only)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from dfttest2_b200 import _lib, dfttest2_b200
from dfttest2_b200.plugin import Filter

HEADER = os.path.join(ROOT, "include", "dfttest2_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dfttest2_b200_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 9
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "binding and header disagree"


def test_version_string():
    v = dfttest2_b200.Version()["version"]
    assert "dfttest2_b200" in v and "sm_100a" in v


@pytest.mark.parametrize("shape", [(16,), (8, 16), (3, 16, 16), (5, 8, 8), (1, 32, 32), (7, 16, 16)])
def test_rdft_matches_numpy(shape):
    rng = np.random.default_rng(len(shape))
    data = rng.standard_normal(int(np.prod(shape)))
    got = np.asarray(dfttest2_b200.RDFT(list(data), list(shape)))
    ref = np.fft.rfftn(data.reshape(shape))
    ref = np.stack([ref.real, ref.imag], axis=-1).ravel()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-9 * max(1.0, np.abs(ref).max()))


def test_rdft_errors():
    with pytest.raises(_lib.Error, match="shape"):
        dfttest2_b200.RDFT([1.0] * 16, [2, 2, 2, 2])
    with pytest.raises(_lib.Error, match="cannot reshape array"):
        dfttest2_b200.RDFT([1.0] * 15, [16])


def _base(radius=1, B=16):
    T = 2 * radius + 1
    X = B // 2 + 1
    return dict(window=[0.1] * (T * B * B), sigma=[1.0], sigma2=1.0, pmin=0.0, pmax=500.0, filter_type=0,
                radius=radius, block_size=B, block_step=B // 4, zero_mean=1, window_freq=[1.0] * (T * B * X * 2))


@pytest.mark.parametrize("change,msg", [
    (dict(radius=4), '"radius" must be in [0, 1, 2, 3]'),
    (dict(block_size=12), '"block_size" must be 8, 16 or 32'),
    (dict(window=[0.1] * 10), "invalid window size"),
    (dict(sigma=[]), "sigma must not be empty"),
    (dict(sigma=[1.0, 2.0]), "invalid sigma array size"),
    (dict(window_freq=[1.0] * 3), "invalid window_freq size"),
    (dict(filter_type=9), '"filter_type" must be in [0, 6]'),
    (dict(block_step=0), '"block_step" must be in [1, block_size]'),
])
def test_create_validation_matches_reference_messages(change, msg):
    kw = _base()
    kw.update(change)
    if change.get("radius") == 4:
        kw["window"] = [0.1] * (9 * 256)
    with pytest.raises(_lib.Error) as e:
        Filter(**kw)
    assert msg in str(e.value)


def test_plugin_plane_checks():
    from dfttest2_b200 import GRAYS, Clip
    clip = Clip([np.zeros((1, 32, 32), np.float32)], GRAYS)
    kw = _base()
    with pytest.raises(_lib.Error, match="plane index out of range"):
        dfttest2_b200.DFTTest(clip, planes=[1], **kw)


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof / offsetof of every C-ABI struct (compiled from the header with
    gcc) equal the ctypes mirrors the Python side passes."""
    import subprocess

    structs = {"dfttest2_b200_params": _lib.Params, "dfttest2_b200_plane": _lib.Plane,
               "dfttest2_b200_grad_plane": _lib.GradPlane, "dfttest2_b200_clip": _lib.Clip,
               "dfttest2_b200_host_plane": _lib.HostPlane}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dfttest2_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)

"""The generated DFT codelets: exactness in FP64 and freshness of codelets.cuh."""
import importlib.util
import os

from conftest import PKG_DIR

GEN = os.path.join(PKG_DIR, "csrc", "gen_codelets.py")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_codelets", GEN)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_codelets_match_numpy_fft():
    assert _gen().check()


def test_codelets_header_is_current(tmp_path):
    out = tmp_path / "codelets.cuh"
    _gen().write(str(out))
    with open(os.path.join(PKG_DIR, "csrc", "codelets.cuh")) as f:
        assert f.read() == out.read_text(), "codelets.cuh is stale: run csrc/gen_codelets.py"


def test_codelet_instruction_counts():
    # op counts of the emitted codelets stay close to the best known FMA counts
    counts = {(k, n): c for k, n, (_, _, c) in _gen().all_codelets()}
    instr = {key: c["add"] + c["fma"] + c["mul"] for key, c in counts.items()}
    assert instr[("r2c", 16)] <= 60
    assert instr[("c2r", 16)] <= 60
    assert instr[("cdft_fwd", 16)] <= 148
    assert instr[("cdft_fwd", 3)] <= 12

"""CPU checks of the drop-in boundary: the C-ABI library builds, loads and
exports every entry point include/csrst.h declares.  No compute calls."""
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared():
    txt = (ROOT / "include" / "csrst.h").read_text()
    return sorted(set(re.findall(r"\b(csrst_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_the_loop(gpu_lib):
    names = declared()
    for must in ("csrst_create", "csrst_push", "csrst_drift", "csrst_step_first", "csrst_step_second",
                 "csrst_move_window", "csrst_gather", "csrst_deposit", "csrst_diag_wake"):
        assert must in names


def test_library_exports_every_declared_symbol(gpu_lib):
    so = ROOT / "csrst_b200" / "libcsrst_gpu.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (csrst_[a-z_0-9]+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    for n in declared():
        assert hasattr(gpu_lib, n)


def test_binding_matches_header(gpu_lib):
    from csrst_b200 import _lib
    src = (ROOT / "csrst_b200" / "_lib.py").read_text()
    bound = set(re.findall(r'"(csrst_[a-z_0-9]+)"', src))
    assert set(declared()) <= bound


def test_built_for_sm100a():
    from csrst_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert "--fmad=false" in build.FLAGS


def test_config_struct_layout():
    # csrst_config in include/csrst.h and the ctypes mirror must agree
    import ctypes as C
    from csrst_b200._lib import Config
    assert C.sizeof(Config) == 4 * 4 + 8 * 8

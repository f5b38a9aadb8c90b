"""The C-ABI library loads and exports every function include/topgpu.h declares."""
import ctypes
import re
from pathlib import Path

from top_gpu_on_matlab_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "topgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(top_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 25
    so = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_error_plumbing():
    assert _lib.lib().top_version() >= 1
    assert isinstance(_lib.last_error(), str)

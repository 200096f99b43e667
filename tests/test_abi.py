"""The C-ABI library loads and exports every entry point include/mcs.h declares."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "mcs.h").read_text()
    return sorted(set(re.findall(r"MCS_API\s+[\w\s\*]+?\b(mcs_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mcs_advance" in syms and "mcs_pop_create" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(str(built_lib))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from mcstreamer_b200 import _lib
    missing = [s for s in declared_symbols() if s not in _lib.SIGNATURES]
    assert not missing, missing
    L = _lib.lib()
    assert L.mcs_version() == 1


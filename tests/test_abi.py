"""The C ABI library loads and exports every entry point include/mcpet.h declares."""
import ctypes
import os
import re

import mcpet
from mcpet import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mcpet.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mcpet_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mcpet_scene_load" in syms and "mcpet_run" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libmcpet.so lacks {missing}"


def test_binding_covers_every_declared_symbol():
    assert set(declared_symbols()) <= set(mcpet.EXPORTED)


def test_version_and_error_text():
    assert "sm_100a" in mcpet.version()
    assert isinstance(_abi.lib().mcpet_last_error(), bytes)


def test_struct_layouts_match_header_sizes():
    # field order and types mirror include/mcpet.h; spot-check a few offsets
    assert _abi.Config.seed.offset == 0
    assert _abi.Config.acquisition_time_ps.offset == 16
    assert _abi.Tallies.psf_capacity.offset == 6 * 8
    assert ctypes.sizeof(_abi.Counters) == 10 * 8
    assert mcpet.PSF_DTYPE.itemsize == 44

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


def test_struct_layouts_equal_the_c_compilers(tmp_path):
    """Every field offset and struct size of the ctypes binding equals what a
    C compiler makes of include/mcpet.h (fields appended to a struct must
    be appended to the binding too)."""
    import subprocess
    structs = {"mcpet_config": _abi.Config, "mcpet_scene_info": _abi.SceneInfo, "mcpet_run_opts": _abi.RunOpts,
               "mcpet_counters": _abi.Counters, "mcpet_tallies": _abi.Tallies, "mcpet_grad_args": _abi.GradArgs,
               "mcpet_tune_result": _abi.TuneResult}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mcpet.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            cname, f, v = ln.split()
            got[(cname, f)] = int(v)
    for cname, cls in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)

"""The drop-in command line (mcpet.x) on its failure paths, which need no GPU:
usage, a missing input file, a malformed input file.  Errors are reported
with a status and a non-zero exit code, as the reference's exit(-1/-2)."""
import os
import subprocess

import pytest

from mcpet import _abi, inputs
import scenes

CLI = os.path.join(os.path.dirname(_abi.LIB_PATH), "mcpet.x")
pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="command line not built")


def _run(*args, cwd=None):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120, cwd=cwd)


def test_usage():
    r = _run()
    assert r.returncode != 0 and "usage" in (r.stdout + r.stderr)


def test_missing_input(workdir):
    r = _run(os.path.join(workdir, "no_such.in"))
    assert r.returncode != 0 and "not found" in (r.stdout + r.stderr)


def test_malformed_input(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "cli_bad", mat, rho, act, vs)
    text = open(inp).read().replace("SECTION SINOGRAM PARAMETERS", "SECTION REMOVED")
    bad = os.path.join(workdir, "cli_bad_missing_section.in")
    open(bad, "w").write(text)
    r = _run(bad, cwd=workdir)
    out = r.stdout + r.stderr
    assert r.returncode != 0 and "lacks" in out and "status 3" in out

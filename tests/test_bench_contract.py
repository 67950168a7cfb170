"""bench.py's reference arm runs the reference's own CPU path (its loaders and
its transport kernel compiled for the host), loads no library of this
project, and prints the JSON line the benchmark contract asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_DRIVER = """
import json, os, sys
sys.path.insert(0, {root!r})
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample-decays", "1e6"]
import bench
rc = bench.main()
libs = sorted({{ln.split()[-1] for ln in open("/proc/self/maps") if ".so" in ln.split()[-1]}})
print("LIBS " + json.dumps(libs))
sys.exit(rc)
"""


def test_reference_arm_json_line_and_libraries():
    out = subprocess.run([sys.executable, "-c", _DRIVER.format(root=ROOT)], cwd=ROOT, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "coincidences/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert "workload" in d["config"] and "head-like phantom" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert "read_input" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    libs = json.loads([l for l in out.stdout.splitlines() if l.startswith("LIBS ")][0][5:])
    ours = [l for l in libs if os.path.basename(l) == "libmcpet.so"]
    assert not ours, ours
    names = {os.path.basename(l) for l in libs}
    assert {"libref_prog.so", "libref_cpu.so"} <= names

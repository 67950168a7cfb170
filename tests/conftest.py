import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "mcgpu-pet_b200"), ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line(
        "markers", "needs_ref(*names): the test compares against these reference builds under oracle/_ref and "
                   "fails (does not skip) when one is missing")


def pytest_runtest_setup(item):
    """A parity test whose reference build is missing fails: a box without
    the reference libraries must not turn every comparison into a skip."""
    for m in item.iter_markers("needs_ref"):
        for name in m.args:
            if not os.path.exists(os.path.join(REF_DIR, name)):
                pytest.fail(f"reference build oracle/_ref/{name} is missing: build it with `make -C oracle/ref` "
                            f"(or __graft_entry__.build()) where the reference sources are present",
                            pytrace=False)


def has_reference_sources() -> bool:
    return os.path.isdir("/root/reference")


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("mcpet"))

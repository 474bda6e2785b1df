import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def driver(tmp_path_factory):
    """tests/cpp/host_driver.cc compiled against the built libcffc_e2d.so."""
    from cffc_b200 import capi
    capi.load_library()  # the library must exist (built by __graft_entry__.build)
    libdir = os.path.join(ROOT, "cffc_b200")
    exe = str(tmp_path_factory.mktemp("host") / "host_driver")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "host_driver.cc"), "-o", exe, "-L", libdir, "-lcffc_e2d",
           "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True)
    return exe

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "louvain-community-detection_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "oracle"), os.path.join(PKG, "python"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


def _ensure_built():
    lib = os.path.join(PKG, "lib", "liblouvain_b200.so")
    cli = os.path.join(PKG, "bin", "louvain")
    orc = os.path.join(ROOT, "oracle", "liblvoracle.so")
    if not (os.path.exists(lib) and os.path.exists(cli)):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


def golden_names():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)["graphs"]


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def golden_mtx(name):
    return os.path.join(GOLDEN, name + ".mtx")


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(n) for n in golden_names()}

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gaugefix-coulomb_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def _ensure(path, cmd):
    if not os.path.exists(path):
        subprocess.run(cmd, check=True, cwd=ROOT, stdout=subprocess.DEVNULL)


# The library and the oracle are normally built by __graft_entry__.build(); build
# them here only if they are missing (fresh checkout).
_ensure(os.path.join(PKG, "lib", "libgfc.so"), ["make", "-C", PKG, "-j8"])
_ensure(os.path.join(ROOT, "oracle", "liboracle.so"), ["make", "-C", os.path.join(ROOT, "oracle"), "oracle"])


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than ~30 s")


@pytest.fixture(scope="session")
def cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return {c["name"]: c for c in json.load(f)}


@pytest.fixture(scope="session")
def param_files():
    with open(os.path.join(GOLDEN, "param_files.json")) as f:
        return json.load(f)

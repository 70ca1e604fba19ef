"""The reference arm of bench.py on CPU: the reference's own half-sweep loop (built
from its sources into oracle/_ref) timed on this host, printed as one JSON line by
rank 0; other ranks exit without work."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
HAVE_REF = any(os.path.exists(os.path.join(REF, n)) for n in ("ref_harness", "ref_harness_v3"))
ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
        "--cpu-half-sweeps", "2", "--ns", "8", "--nt", "16"]


def run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run(ARGS, capture_output=True, text=True, env=env, timeout=300)


@pytest.mark.skipif(not HAVE_REF, reason="the reference harness is not built here")
def test_reference_arm_line():
    p = run({"WORLD_SIZE": "1", "RANK": "0"})
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "site-updates/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 1
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["lattice"] == [8, 16]


def test_reference_arm_other_ranks_do_no_work():
    p = run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


@pytest.mark.skipif(not HAVE_REF, reason="the reference harness is not built here")
def test_reference_arm_loads_no_product_library():
    """The reference arm makes its input with the oracle's generator: the product
    library (gaugefix-coulomb_b200/lib/libgfc.so) is never mapped into its process."""
    code = ("import runpy, sys; sys.argv = %r; runpy.run_path(%r, run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT-LOADED' if 'libgfc' in maps else 'CLEAN', 'oracle' in maps)"
            % (ARGS[1:], ARGS[1]))
    env = dict(os.environ, WORLD_SIZE="1", RANK="0")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip().splitlines()[-1] == "CLEAN True"

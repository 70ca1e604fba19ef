"""The drop-in program on the GPU against the reference program's recorded output:
identical stdout text, gauge-transformation bytes and side file."""
import os
import subprocess

import numpy as np
import pytest

import gfc
import oracle_ref as orc
from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu
CLI = os.path.join(PKG, "bin", "gauge_fix_coulomb")


def write_case(c, d):
    U = gfc.synth_config(c["ns"], c["nt"], c["seed"], c["scale"])
    (d / f"{c['name']}.cfg").write_bytes(U.astype(">f8" if c["in_bytes"] == 8 else ">f4").tobytes())
    (d / f"{c['name']}.par").write_text("#generic parameters\n" + "".join(
        f"{k}:   {v}\n" for k, v in c["params"].items()))


@pytest.mark.parametrize("name", ["l4x8", "cfg0_8x16", "l4x8_f32in"])
def test_cli_matches_reference(cases, tmp_path, name):
    c = cases[name]
    write_case(c, tmp_path)
    env = dict(os.environ)
    if c["in_bytes"] == 4:
        env["GFC_CFG_IN"] = "f32"
    p = subprocess.run([CLI, f"{name}.cfg", f"{name}.gt_cli", str(c["ns"]), str(c["nt"]), f"{name}.par"],
                       capture_output=True, text=True, cwd=tmp_path, env=env, timeout=600)
    assert p.returncode == c["cli_exit"], p.stderr
    assert p.stdout == open(os.path.join(GOLDEN, f"{name}_stdout.txt")).read()
    assert p.stderr == open(os.path.join(GOLDEN, f"{name}_stderr.txt")).read()
    G = np.fromfile(tmp_path / f"{name}.gt_cli", dtype=np.float64)
    assert orc.sha(G) == c["cli_gt_sha256"]
    side = (tmp_path / f"sweeps_to_gaugefix_{c['ns']}x{c['nt']}.txt").read_text()
    assert side == c["side_file"]


def test_cli_not_converged_exit(cases, tmp_path):
    c = cases["l4x8_maxsweeps"]
    write_case(c, tmp_path)
    p = subprocess.run([CLI, f"{c['name']}.cfg", "g.out", "4", "8", f"{c['name']}.par"], capture_output=True,
                       text=True, cwd=tmp_path, timeout=300)
    assert p.returncode == 1
    assert "could not be gauge-fixed within the maximum number of sweeps" in p.stderr
    assert not (tmp_path / "g.out").exists()


def test_cli_writes_the_fixed_config_when_asked(cases, tmp_path):
    """GFC_WRITE_CONFIG=1: the gauge-fixed configuration (the writeConfig call the
    reference's main has commented out) goes to <config>fixed, every link (temporal
    ones included) equal to G(x) U(x) G(x+mu)^dagger of the reunitarised input with
    the G written beside it; GFC_CFG_OUT=f32 with GFC_CFG_SWAP_OUT=1 writes the same
    links as big-endian FP32."""
    c = cases["l4x8"]
    ns, nt = c["ns"], c["nt"]
    write_case(c, tmp_path)
    U0 = gfc.synth_config(ns, nt, c["seed"], c["scale"])
    orc.reunitarize(U0)
    out = {}
    for tag, extra in (("f64", {}), ("f32", {"GFC_CFG_OUT": "f32", "GFC_CFG_SWAP_OUT": "1"})):
        env = dict(os.environ, GFC_WRITE_CONFIG="1", **extra)
        p = subprocess.run([CLI, f"{c['name']}.cfg", "g.out", str(ns), str(nt), f"{c['name']}.par"],
                           capture_output=True, text=True, cwd=tmp_path, env=env, timeout=600)
        assert p.returncode == 0, p.stderr
        assert f"U fixed written for config {c['name']}.cfg." in p.stdout
        raw = (tmp_path / f"{c['name']}.cfgfixed").read_bytes()
        out[tag] = np.frombuffer(raw, dtype=np.float64 if tag == "f64" else ">f4").astype(np.float64)
        G = np.fromfile(tmp_path / "g.out", dtype=np.float64)
    assert out["f64"].size == ns ** 3 * nt * 4 * 18
    U1 = U0.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(out["f64"], U1, atol=1e-12)
    np.testing.assert_array_equal(out["f32"], out["f64"].astype(np.float32).astype(np.float64))

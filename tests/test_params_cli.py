"""Parameter parsing and the command line's early exits, against the reference
program's own output (tests/golden/param_files.json, recorded from the unmodified
program built from source).  The cases stop at "Loading of file ... failed."
before any GPU work, so they run on CPU."""
import os
import subprocess

import pytest

import gfc
from conftest import PKG

CLI = os.path.join(PKG, "bin", "gauge_fix_coulomb")


def run_cli(args, cwd):
    return subprocess.run([CLI] + args, capture_output=True, text=True, cwd=cwd, timeout=120)


@pytest.mark.parametrize("name", ["comments_unknown", "bad_proxy", "bad_omega", "negative_tol", "zero_reunit",
                                  "estimate_key", "missing_par", "no_par"])
def test_cli_parameter_text_matches_reference(param_files, tmp_path, name):
    case = param_files[name]
    args = ["missing.cfg", "x.gt", "4", "8"]
    if case["text"] is not None:
        (tmp_path / f"{name}.par").write_text(case["text"])
        args.append(f"{name}.par")
    elif name == "missing_par":
        args.append("nope.par")
    p = run_cli(args, tmp_path)
    assert p.stdout == case["stdout"]
    assert p.stderr == case["stderr"]
    assert p.returncode == case["exit"]


def test_parser_values(tmp_path):
    f = tmp_path / "p.par"
    f.write_text("# c\n gfix_proxy : theta\ntolerance: 1e-14\nhits: 3.7\nomega_OR: 1.5\n"
                 "max_sweeps_to_fix: 1234.9\nestimate_sweeps_to_gfixprogress: 55\nsweeps_to_reunitarization: 9\n")
    p = gfc.parse_params(str(f))
    assert p.gfix_proxy == gfc.PROXY_THETA
    assert p.tolerance == 1e-14
    assert p.hits == 3                       # atof then unsigned conversion
    assert p.omega_OR == pytest.approx(1.5)
    assert p.max_sweeps_to_fix == 1234
    assert p.estimate_sweeps_to_gf_progress == 55  # print-label spelling accepted
    assert p.sweeps_to_reunitarization == 9
    assert p.error == 0


def test_defaults_and_validity():
    p = gfc.default_params()
    assert (p.tolerance, p.max_sweeps_to_fix, p.estimate_sweeps_to_gf_progress, p.sweeps_to_reunitarization,
            p.hits) == (1e-16, 100000, 1000, 250, 2)
    assert p.omega_OR == pytest.approx(1.95) and float(p.omega_OR) != 1.95  # stored as float
    assert gfc.lib.gfc_params_valid(p) == 1
    for k, v in [("omega_OR", 2.0), ("omega_OR", 0.99), ("tolerance", 0.0), ("sweeps_to_reunitarization", 0),
                 ("error", 1)]:
        q = gfc.default_params(**{k: v})
        assert gfc.lib.gfc_params_valid(q) == 0, k


def test_cli_wrong_argc_and_geometry(tmp_path):
    p = run_cli(["a.cfg", "b.gt", "4"], tmp_path)
    assert p.returncode == 1 and "Bad input." in p.stderr
    p = run_cli(["a.cfg", "b.gt", "0", "8"], tmp_path)
    assert p.returncode == 1 and "n_SPC: 0" in p.stderr


def test_cli_short_and_long_files(tmp_path):
    V = 2 ** 3 * 2
    (tmp_path / "short.cfg").write_bytes(b"\0" * (V * 4 * 144 - 8))
    (tmp_path / "long.cfg").write_bytes(b"\0" * (V * 4 * 144 + 1))
    p = run_cli(["short.cfg", "g", "2", "2"], tmp_path)
    assert p.returncode == 1 and "Error: Reading from file short.cfg." in p.stderr
    p = run_cli(["long.cfg", "g", "2", "2"], tmp_path)
    assert p.returncode == 1 and "File has not been read till the end" in p.stderr

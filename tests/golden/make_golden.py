"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference built from its own sources (oracle/Makefile -> oracle/_ref/) on
seeded synthetic configurations and records, per case:
  - the sha256 of the input file and of the reference's final G and U bytes
    (bit-exact parity targets),
  - sweep count / return code, final residue, e2, theta, F, plaquettes,
  - for small cases the e2 and F trace after every half-sweep and the full G,
  - the reference program's stdout for a few cases (CLI drop-in text).

Needs the reference sources (only in the build container); the fixtures are
committed so the tests run anywhere.  Usage:  python tests/golden/make_golden.py

  --full   instead runs the reference's complete fix of the two full-size workloads
           (32^3x64 FP64, seed 2, H 0.5; 48^3x96 stored FP32, seed 3, H 0.7; tolerance
           1e-15) through oracle/_ref/ref_harness (ref_harness_f32in for FP32 files)
           and writes full_cases.json (sweep count, return code, final residue, e2, F,
           theta, plaquettes before and after, sha256 of G and of the spatial links),
           <name>_trace.npy (e2 and F after the first 20 half-sweeps and after every
           50th) and <name>_gt_sample.npy (G at every sample_stride-th site, after
           half-sweep dump_sweep and at the end).  About 10 min (32^3x64) and 40 min
           (48^3x96) on 8 host cores.
"""
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle_ref as orc  # noqa: E402  (the oracle's restatement of the workload generator)

REF = os.path.join(ROOT, "oracle", "_ref")

# name, ns, nt, seed, scale, in_bytes, params, keep_trace, keep_g, keep_stdout
CASES = [
    ("cfg0_8x16", 8, 16, 1, 0.5, 8, dict(tolerance="1.0E-16", omega_OR="1.95"), True, False, True),
    ("l4x8", 4, 8, 11, 0.5, 8, dict(tolerance="1.0E-15"), True, True, True),
    ("l4x8_theta", 4, 8, 11, 0.5, 8, dict(gfix_proxy="theta", tolerance="1.0E-17"), True, False, False),
    ("l4x5_oddnt", 4, 5, 12, 0.5, 8, dict(tolerance="1.0E-15"), True, True, False),
    ("l3x4_oddns", 3, 4, 13, 0.5, 8, dict(tolerance="1.0E-14"), True, True, False),
    ("l5x4_oddns", 5, 4, 14, 0.5, 8, dict(tolerance="1.0E-14"), True, True, False),
    ("l2x4", 2, 4, 15, 0.5, 8, dict(tolerance="1.0E-15"), True, True, False),
    ("l6x6_params", 6, 6, 16, 0.5, 8,
     dict(tolerance="1.0E-14", omega_OR="1.7", hits="1", sweeps_to_reunitarization="10",
          estimate_sweeps_to_gf_progress="100"), True, True, False),
    ("l4x8_maxsweeps", 4, 8, 17, 0.5, 8, dict(tolerance="1.0E-15", max_sweeps_to_fix="40"), True, True, False),
    ("l8x8_scale07", 8, 8, 3, 0.7, 8, dict(tolerance="1.0E-15"), True, False, False),
    ("l6x12_hits3", 6, 12, 18, 0.5, 8, dict(tolerance="1.0E-15", hits="3", omega_OR="1.99"), True, False, False),
    ("l4x8_f32in", 4, 8, 19, 0.5, 4, dict(tolerance="1.0E-15"), False, True, True),
]


def sha(b):
    return hashlib.sha256(b).hexdigest()


def write_params(path, kv):
    with open(path, "w") as f:
        f.write("#generic parameters\n")
        for k, v in kv.items():
            f.write(f"{k}:   {v}\n")


def config_bytes(ns, nt, seed, scale, in_bytes):
    U = orc.synth_config(ns, nt, seed, scale)
    return U.astype(">f8" if in_bytes == 8 else ">f4").tobytes()


def normalise_stdout(text, tmp):
    return text.replace(tmp + "/", "")


def run_case(name, ns, nt, seed, scale, in_bytes, params, keep_trace, keep_g, keep_stdout, tmp):
    rec = dict(name=name, ns=ns, nt=nt, seed=seed, scale=scale, in_bytes=in_bytes, params=params)
    raw = config_bytes(ns, nt, seed, scale, in_bytes)
    rec["cfg_sha256"] = sha(raw)
    cfg = os.path.join(tmp, f"{name}.cfg")
    with open(cfg, "wb") as f:
        f.write(raw)
    par = os.path.join(tmp, f"{name}.par")
    write_params(par, params)
    V = ns ** 3 * nt
    if in_bytes == 8:
        prefix = os.path.join(tmp, name)
        subprocess.run([os.path.join(REF, "ref_harness"), "trace", cfg, str(ns), str(nt), par, prefix],
                       check=True, capture_output=True, cwd=tmp)
        summ = {}
        for line in open(prefix + ".summary"):
            k, v = line.split()
            summ[k] = float(v) if "." in v or "e" in v else int(v)
        rec.update(summ)
        gt = open(prefix + ".gt", "rb").read()
        u = open(prefix + ".u", "rb").read()
        rec["gt_sha256"] = sha(gt)
        rec["u_sha256"] = sha(u)
        ua = np.frombuffer(u, dtype=np.float64).reshape(V, 4, 18)
        rec["u_spatial_sha256"] = sha(np.ascontiguousarray(ua[:, 1:4, :]).tobytes())
        if keep_trace:
            tr = np.loadtxt(prefix + ".trace")
            np.save(os.path.join(HERE, f"{name}_trace.npy"), tr)
        if keep_g:
            np.save(os.path.join(HERE, f"{name}_gt.npy"), np.frombuffer(gt, dtype=np.float64))
    # the unmodified program (FP32-input build for FP32 files)
    prog = "gauge_fix_coulomb" if in_bytes == 8 else "gauge_fix_coulomb_f32in"
    gtout = os.path.join(tmp, f"{name}.gt_cli")
    p = subprocess.run([os.path.join(REF, prog), cfg, gtout, str(ns), str(nt), par], capture_output=True,
                       text=True, cwd=tmp)
    rec["cli_exit"] = p.returncode
    if os.path.exists(gtout):
        g2 = open(gtout, "rb").read()
        rec["cli_gt_sha256"] = sha(g2)
        if in_bytes == 4 and keep_g:
            np.save(os.path.join(HERE, f"{name}_gt.npy"), np.frombuffer(g2, dtype=np.float64))
    m = re.search(r"Sweeps needed to gauge-fix config from file .*: (-?\d+)\. residue: (\S+)", p.stdout)
    if m:
        rec["cli_sweeps"] = int(m.group(1))
        rec["cli_residue_text"] = m.group(2)
    if keep_stdout:
        with open(os.path.join(HERE, f"{name}_stdout.txt"), "w") as f:
            f.write(normalise_stdout(p.stdout, tmp))
        with open(os.path.join(HERE, f"{name}_stderr.txt"), "w") as f:
            f.write(normalise_stdout(p.stderr, tmp))
    side = os.path.join(tmp, f"sweeps_to_gaugefix_{ns}x{nt}.txt")
    if os.path.exists(side):
        rec["side_file"] = normalise_stdout(open(side).read(), tmp)
        os.remove(side)
    return rec


def param_file_cases(tmp):
    """The reference's parser on awkward parameter files, via the unmodified program
    (a missing config makes it stop right after printing the parameters)."""
    files = {
        "comments_unknown": "# comment line\n\ngfix_proxy :  theta \n tolerance: 1e-14\nfoo: 3\n"
                            "hits: 3.7\nomega_OR: 1.5\nmax_sweeps_to_fix: 1234.9\n",
        "bad_proxy": "gfix_proxy: e3\nomega_OR: 1.8\n",
        "bad_omega": "omega_OR: 2.5\ntolerance: 1e-10\n",
        "negative_tol": "tolerance: -1\n",
        "zero_reunit": "sweeps_to_reunitarization: 0\n",
        "estimate_key": "estimate_sweeps_to_gf_progress: 77\nsweeps_to_reunitarization: 12\n",
    }
    out = {}
    for name, text in files.items():
        par = os.path.join(tmp, name + ".par")
        with open(par, "w") as f:
            f.write(text)
        p = subprocess.run([os.path.join(REF, "gauge_fix_coulomb"), os.path.join(tmp, "missing.cfg"),
                            os.path.join(tmp, "x.gt"), "4", "8", par], capture_output=True, text=True, cwd=tmp)
        out[name] = dict(text=text, stdout=normalise_stdout(p.stdout, tmp), stderr=normalise_stdout(p.stderr, tmp),
                         exit=p.returncode)
    # missing parameter file, wrong argument count
    p = subprocess.run([os.path.join(REF, "gauge_fix_coulomb"), os.path.join(tmp, "missing.cfg"),
                        os.path.join(tmp, "x.gt"), "4", "8", os.path.join(tmp, "nope.par")],
                       capture_output=True, text=True, cwd=tmp)
    out["missing_par"] = dict(text=None, stdout=normalise_stdout(p.stdout, tmp),
                              stderr=normalise_stdout(p.stderr, tmp), exit=p.returncode)
    p = subprocess.run([os.path.join(REF, "gauge_fix_coulomb"), os.path.join(tmp, "missing.cfg"),
                        os.path.join(tmp, "x.gt"), "4", "8"], capture_output=True, text=True, cwd=tmp)
    out["no_par"] = dict(text=None, stdout=normalise_stdout(p.stdout, tmp), stderr=normalise_stdout(p.stderr, tmp),
                         exit=p.returncode)
    return out


# name, ns, nt, seed, scale, in_bytes, params, dense trace length, trace stride, dump sweep, sample stride
FULL_CASES = [
    ("cfg1_32x64", 32, 64, 2, 0.5, 8, dict(tolerance="1.0E-15"), 20, 50, 700, 2039),
    ("cfg2_48x96_f32in", 48, 96, 3, 0.7, 4, dict(tolerance="1.0E-15"), 20, 50, 700, 10337),
]


def run_full_case(name, ns, nt, seed, scale, in_bytes, params, dense, every, dump, stride, tmp):
    import time
    rec = dict(name=name, ns=ns, nt=nt, seed=seed, scale=scale, in_bytes=in_bytes, params=params,
               dump_sweep=dump, sample_stride=stride)
    raw = config_bytes(ns, nt, seed, scale, in_bytes)
    rec["cfg_sha256"] = sha(raw)
    cfg = os.path.join(tmp, f"{name}.cfg")
    with open(cfg, "wb") as f:
        f.write(raw)
    del raw
    par = os.path.join(tmp, f"{name}.par")
    write_params(par, params)
    V = ns ** 3 * nt
    prefix = os.path.join(tmp, name)
    prog = "ref_harness" if in_bytes == 8 else "ref_harness_f32in"
    t0 = time.time()
    subprocess.run([os.path.join(REF, prog), "trace", cfg, str(ns), str(nt), par, prefix, str(dense), str(every),
                    str(dump)], check=True, capture_output=True, cwd=tmp)
    rec["reference_seconds"] = round(time.time() - t0, 1)
    for line in open(prefix + ".summary"):
        k, v = line.split()
        rec[k] = float(v) if "." in v or "e" in v else int(v)
    gt = np.fromfile(prefix + ".gt", dtype=np.float64)
    rec["gt_sha256"] = sha(gt.tobytes())
    u = np.fromfile(prefix + ".u", dtype=np.float64).reshape(V, 4, 18)
    rec["u_spatial_sha256"] = sha(np.ascontiguousarray(u[:, 1:4, :]).tobytes())
    del u
    gd = np.fromfile(prefix + ".gt_dump", dtype=np.float64)
    sites = np.arange(0, V, stride)
    sample = np.stack([gd.reshape(V, 18)[sites], gt.reshape(V, 18)[sites]])
    np.save(os.path.join(HERE, f"{name}_gt_sample.npy"), sample)
    np.save(os.path.join(HERE, f"{name}_trace.npy"), np.loadtxt(prefix + ".trace"))
    for ext in (".gt", ".gt_dump", ".u", ".cfg"):
        os.remove(prefix + ext if ext != ".cfg" else cfg)
    return rec


def main_full():
    if not os.path.exists(os.path.join(REF, "ref_harness_f32in")):
        sys.exit("oracle/_ref is not built (make -C oracle REF=<reference tree>)")
    recs = []
    with tempfile.TemporaryDirectory() as tmp:
        for c in FULL_CASES:
            recs.append(run_full_case(*c, tmp=tmp))
            print(recs[-1]["name"], recs[-1]["sweeps"], recs[-1]["final_residue"], recs[-1]["reference_seconds"],
                  flush=True)
            with open(os.path.join(HERE, "full_cases.json"), "w") as f:
                json.dump(recs, f, indent=1)


def main():
    if "--full" in sys.argv:
        return main_full()
    if not os.path.exists(os.path.join(REF, "ref_harness")):
        sys.exit("oracle/_ref is not built (make -C oracle with the reference sources present)")
    with tempfile.TemporaryDirectory() as tmp:
        recs = [run_case(*c, tmp=tmp) for c in CASES]
        params = param_file_cases(tmp)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(recs, f, indent=1)
    with open(os.path.join(HERE, "param_files.json"), "w") as f:
        json.dump(params, f, indent=1)
    for r in recs:
        print(r["name"], r.get("sweeps"), r.get("cli_sweeps"), r.get("final_residue"), r.get("cli_exit"))


if __name__ == "__main__":
    main()

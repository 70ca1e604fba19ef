"""ctypes view of oracle/liboracle.so -- the CPU restatement used as the checker.

Test infrastructure only (the product never loads it).
"""
import ctypes
import hashlib
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
_P, _I, _D, _U = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint
_lib.orc_fix.argtypes = [_P, _P, _I, _I, _D, _I, _U, _U, _U, ctypes.c_float, _U, _P, _P, _I, _P, _I]
_lib.orc_fix.restype = _I
_lib.orc_halfsweep.argtypes = [_P, _P, _I, _I, _I, _D, _U]
_lib.orc_reunitarize.argtypes = [_P, ctypes.c_size_t]
_lib.orc_reunitarize.restype = _I
_lib.orc_e2.argtypes = [_P, _I, _I, _P]
_lib.orc_e2.restype = _D
_lib.orc_theta.argtypes = [_P, _I, _I]
_lib.orc_theta.restype = _D
_lib.orc_functional.argtypes = [_P, _I, _I]
_lib.orc_functional.restype = _D
_lib.orc_plaquette.argtypes = [_P, _I, _I, _I]
_lib.orc_plaquette.restype = _D
_lib.orc_apply_gt.argtypes = [_P, _P, _I, _I]
_lib.orc_synth_config.argtypes = [_I, _I, ctypes.c_ulonglong, _D, _P]
_lib.orc_synth_config.restype = _I


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def reunitarize(M):
    n = M.size // 18
    return _lib.orc_reunitarize(M.ctypes.data, n)


def e2(U, ns, nt, slices=False):
    if slices:
        out = np.empty(nt)
        tot = _lib.orc_e2(U.ctypes.data, ns, nt, out.ctypes.data)
        return tot, out
    return _lib.orc_e2(U.ctypes.data, ns, nt, None)


def theta(U, ns, nt):
    return _lib.orc_theta(U.ctypes.data, ns, nt)


def functional(U, ns, nt):
    return _lib.orc_functional(U.ctypes.data, ns, nt)


def plaquette(U, ns, nt, which):
    """which: 0 spatial, 1 temporal, 2 total"""
    return _lib.orc_plaquette(U.ctypes.data, ns, nt, which)


def halfsweep(U, G, ns, nt, sweep, omega=1.95, hits=2):
    _lib.orc_halfsweep(U.ctypes.data, G.ctypes.data, ns, nt, sweep, float(np.float32(omega)), hits)


def apply_gt(U, G, ns, nt):
    _lib.orc_apply_gt(U.ctypes.data, G.ctypes.data, ns, nt)


def fix(U, G, ns, nt, tol=1e-16, theta_proxy=False, max_sweeps=100000, estimate=1000, reunit=250,
        omega=1.95, hits=2, trace_len=0):
    """gaugefixOverrelaxation restated; returns (rc, final_residue, e2_trace, F_trace)."""
    tr = np.zeros(max(trace_len, 1))
    ftr = np.zeros(max(trace_len, 1))
    fr = np.zeros(1)
    rc = _lib.orc_fix(U.ctypes.data, G.ctypes.data, ns, nt, tol, int(theta_proxy), max_sweeps, estimate, reunit,
                      omega, hits, tr.ctypes.data if trace_len else None, ftr.ctypes.data if trace_len else None,
                      trace_len, fr.ctypes.data, 0)
    return rc, fr[0], tr[:trace_len], ftr[:trace_len]


def synth_config(ns, nt, seed, scale):
    """The seeded workload construction restated in the oracle (same bytes as the
    product's generator for the same arguments)."""
    U = np.empty(ns ** 3 * nt * 4 * 18)
    if _lib.orc_synth_config(ns, nt, seed, scale, U.ctypes.data) != 0:
        raise MemoryError("orc_synth_config")
    return U


def case_params(case):
    """Parameters of a golden case as oracle keyword arguments (defaults of
    initParametersORDefault, gauge_fixing.c:72-84)."""
    p = case["params"]
    return dict(tol=float(p.get("tolerance", 1e-16)), theta_proxy=p.get("gfix_proxy", "e2") == "theta",
                max_sweeps=int(float(p.get("max_sweeps_to_fix", 100000))),
                estimate=int(float(p.get("estimate_sweeps_to_gf_progress", 1000))),
                reunit=int(float(p.get("sweeps_to_reunitarization", 250))),
                omega=float(p.get("omega_OR", 1.95)), hits=int(float(p.get("hits", 2))))

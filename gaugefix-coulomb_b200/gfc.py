"""ctypes binding of libgfc.so (include/gfc.h), the B200 Coulomb gauge fixer.

The product is the C library and the ``bin/gauge_fix_coulomb`` program; this module
is the Python view of the same C ABI, used by the tests and the benchmark.  It
mirrors the reference's in-process interface: ``gaugefix_overrelaxation`` has the
meaning and return codes of ``gaugefixOverrelaxation`` (gauge_fixing.c:713-826),
``Params`` is ``ORGaugeFixingParameters`` (gauge_fixing.h:30-54), and the
observables are ``calculate_e2`` / ``calculateTheta`` / ``calculateF`` /
``averagePlaquette``.

There is no fallback: if the library is missing, importing this module raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgfc.so")
CLI_PATH = os.path.join(_HERE, "bin", "gauge_fix_coulomb")

GFC_OK = 0
FIX_NOT_CONVERGED = -1
FIX_BAD_PARAMS = -2
PROXY_E2, PROXY_THETA = 0, 1
PREC_FP64_EXACT, PREC_FP64_FAST, PREC_MIXED, PREC_FP64_FULL = 0, 1, 2, 3
STOP_REFERENCE, STOP_EVERY = 0, 1
CTX_MIXED = 1


class Params(ctypes.Structure):
    """ORGaugeFixingParameters; omega_OR is a float like the reference's."""

    _fields_ = [
        ("tolerance", ctypes.c_double),
        ("gfix_proxy", ctypes.c_int),
        ("max_sweeps_to_fix", ctypes.c_uint),
        ("estimate_sweeps_to_gf_progress", ctypes.c_uint),
        ("sweeps_to_reunitarization", ctypes.c_uint),
        ("error", ctypes.c_int),
        ("omega_OR", ctypes.c_float),
        ("hits", ctypes.c_uint),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("stop_rule", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("switch_e2", ctypes.c_double),
        ("refine_reunit", ctypes.c_uint),
        ("block_threads", ctypes.c_int),
        ("dense_check", ctypes.c_int),
        ("warm_start", ctypes.c_int),
        ("fp32_refresh", ctypes.c_int),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("sweeps", ctypes.c_int),
        ("sweeps_fp32", ctypes.c_int),
        ("first_below_tol", ctypes.c_int),
        ("initial_residue", ctypes.c_double),
        ("final_residue", ctypes.c_double),
        ("e2", ctypes.c_double),
        ("theta", ctypes.c_double),
        ("functional", ctypes.c_double),
        ("seconds_sweeps", ctypes.c_double),
        ("seconds_total", ctypes.c_double),
        ("site_updates", ctypes.c_longlong),
        ("kernel_launches", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GFCError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise GFCError(f"{LIB_PATH} is not built (run __graft_entry__.build() or make -C gaugefix-coulomb_b200)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D, U, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint, ctypes.c_size_t
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "gfc_params_default": (None, [ctypes.POINTER(Params)]),
        "gfc_params_valid": (I, [ctypes.POINTER(Params)]),
        "gfc_params_parse_file": (I, [ctypes.c_char_p, ctypes.POINTER(Params)]),
        "gfc_params_print": (None, [ctypes.POINTER(Params)]),
        "gfc_options_default": (None, [ctypes.POINTER(Options)]),
        "gfc_synth_config": (I, [I, I, ctypes.c_uint64, D, P]),
        "gfc_read_exact": (I, [ctypes.c_char_p, P, S, I]),
        "gfc_write_all": (I, [ctypes.c_char_p, P, S]),
        "gfc_byteswap": (I, [P, S, S]),
        "gfc_last_error": (ctypes.c_char_p, []),
        "gfc_device_code_version": (I, [I, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "gfc_check_division": (I, [I, ctypes.c_ulonglong, ctypes.c_longlong, ctypes.POINTER(ctypes.c_ulonglong)]),
        "gfc_host_alloc": (P, [S]),
        "gfc_host_free": (None, [P]),
        "gfc_ctx_create": (I, [I, I, I, I, ctypes.POINTER(P)]),
        "gfc_ctx_destroy": (I, [P]),
        "gfc_ctx_kernel_launches": (ctypes.c_longlong, [P]),
        "gfc_ctx_stream": (P, [P]),
        "gfc_ctx_sync": (I, [P]),
        "gfc_ctx_upload_links": (I, [P, P, I, I]),
        "gfc_ctx_download_links": (I, [P, P, I, I]),
        "gfc_ctx_upload_gt": (I, [P, P, I, I]),
        "gfc_ctx_download_gt": (I, [P, P, I, I]),
        "gfc_ctx_download_gt_async": (I, [P, P, I, I]),
        "gfc_ctx_get_link": (I, [P, S, I, DP]),
        "gfc_ctx_reunitarize": (I, [P]),
        "gfc_ctx_reunitarize_gt": (I, [P]),
        "gfc_ctx_save_links": (I, [P]),
        "gfc_ctx_restore_links": (I, [P]),
        "gfc_ctx_set_identity_gt": (I, [P]),
        "gfc_ctx_status": (I, [P, ctypes.POINTER(U)]),
        "gfc_ctx_e2": (I, [P, DP, DP]),
        "gfc_ctx_e2_slices": (I, [P, P]),
        "gfc_ctx_functional": (I, [P, DP]),
        "gfc_ctx_plaquette": (I, [P, DP, DP]),
        "gfc_ctx_halfsweeps": (I, [P, I, I, ctypes.c_float, U, I]),
        "gfc_ctx_finalize_temporal": (I, [P]),
        "gfc_ctx_fix": (I, [P, ctypes.POINTER(Params), ctypes.POINTER(Options), ctypes.POINTER(Report)]),
        "gfc_ctx_apply_gt": (I, [P]),
        "gfc_ctx_upload_links_reunit": (I, [P, P, I, I]),
        "gfc_gaugefix_overrelaxation": (I, [I, I, P, P, ctypes.POINTER(Params), ctypes.POINTER(Options),
                                            ctypes.POINTER(Report), I]),
        "gfc_e2_theta_device_noalloc": (I, [I, I, P, P, DP, DP]),
        "gfc_ctx_autotune": (I, [P, I, P]),
        "gfc_ctx_get_shapes": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I)]),
        "gfc_ctx_set_shapes": (I, [P, I, I, I]),
        "gfc_ctx_set_blocking": (I, [P, I, I, I]),
        "gfc_ctx_get_blocking": (I, [P] + [ctypes.POINTER(I)] * 4),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def last_error():
    return lib.gfc_last_error().decode(errors="replace")


def _check(rc, what):
    if rc != GFC_OK:
        raise GFCError(f"{what} failed ({rc}): {last_error()}")


def default_params(**kw):
    p = Params()
    lib.gfc_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def parse_params(path):
    p = Params()
    lib.gfc_params_parse_file(None if path is None else path.encode(), ctypes.byref(p))
    return p


def options(**kw):
    o = Options()
    lib.gfc_options_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def device_code_version(device=0):
    """(binaryVersion, ptxVersion) of the library's kernels as loaded on `device`."""
    b, p = ctypes.c_int(), ctypes.c_int()
    _check(lib.gfc_device_code_version(device, ctypes.byref(b), ctypes.byref(p)), "gfc_device_code_version")
    return b.value, p.value


def check_division(count, seed=1, device=0):
    """Quotients, of `count` pseudo-random pairs, on which the exact path's shared-
    divisor division differs from IEEE division (0 expected)."""
    bad = ctypes.c_ulonglong()
    _check(lib.gfc_check_division(device, seed, count, ctypes.byref(bad)), "gfc_check_division")
    return bad.value


def synth_config(ns, nt, seed, scale):
    """Links in the reference layout, float64 array of shape (V*4*18,)."""
    V = ns ** 3 * nt
    U = np.empty(V * 4 * 18, dtype=np.float64)
    _check(lib.gfc_synth_config(ns, nt, seed, scale, U.ctypes.data), "gfc_synth_config")
    return U


class PinnedBuffer:
    """Page-locked host memory viewed as a numpy array."""

    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        self.ptr = lib.gfc_host_alloc(self.nbytes)
        if not self.ptr:
            raise GFCError("gfc_host_alloc failed")
        self.array = np.ctypeslib.as_array((ctypes.c_uint8 * self.nbytes).from_address(self.ptr))

    def view(self, dtype):
        return self.array.view(dtype)

    def close(self):
        if getattr(self, "ptr", None):   # None too when __init__ failed
            lib.gfc_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


class Lattice:
    """One lattice resident on one GPU (a gfc_ctx)."""

    def __init__(self, ns, nt, device=0, mixed=False):
        self.ns, self.nt = ns, nt
        self.V = ns ** 3 * nt
        h = ctypes.c_void_p()
        _check(lib.gfc_ctx_create(ns, nt, device, CTX_MIXED if mixed else 0, ctypes.byref(h)), "gfc_ctx_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):   # None too when __init__ failed
            lib.gfc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- transfers
    def upload_links(self, buf, elem_bytes=8, byteswap=False):
        a = np.ascontiguousarray(buf)
        assert a.nbytes == self.V * 4 * 18 * elem_bytes, "link buffer size"
        _check(lib.gfc_ctx_upload_links(self.h, a.ctypes.data, elem_bytes, int(byteswap)), "upload_links")

    def upload_links_reunit(self, buf, elem_bytes=8, byteswap=False):
        """upload_links + reunitarize in one pass over the links."""
        a = np.ascontiguousarray(buf)
        assert a.nbytes == self.V * 4 * 18 * elem_bytes, "link buffer size"
        _check(lib.gfc_ctx_upload_links_reunit(self.h, a.ctypes.data, elem_bytes, int(byteswap)), "upload_links_reunit")

    def download_links(self, elem_bytes=8, byteswap=False, out=None):
        dt = np.float64 if elem_bytes == 8 else np.float32
        out = np.empty(self.V * 4 * 18, dtype=dt) if out is None else out
        _check(lib.gfc_ctx_download_links(self.h, out.ctypes.data, elem_bytes, int(byteswap)), "download_links")
        return out

    def upload_gt(self, buf, elem_bytes=8, byteswap=False):
        a = np.ascontiguousarray(buf)
        assert a.nbytes == self.V * 18 * elem_bytes
        _check(lib.gfc_ctx_upload_gt(self.h, a.ctypes.data, elem_bytes, int(byteswap)), "upload_gt")

    def download_gt(self, elem_bytes=8, byteswap=False, out=None):
        dt = np.float64 if elem_bytes == 8 else np.float32
        out = np.empty(self.V * 18, dtype=dt) if out is None else out
        _check(lib.gfc_ctx_download_gt(self.h, out.ctypes.data, elem_bytes, int(byteswap)), "download_gt")
        return out

    def download_gt_async(self, out, elem_bytes=8, byteswap=False):
        """Queue the download of G into `out` (page-locked, e.g. a PinnedBuffer view)
        and return at once; sync() completes it."""
        _check(lib.gfc_ctx_download_gt_async(self.h, out.ctypes.data, elem_bytes, int(byteswap)),
               "download_gt_async")
        return out

    def get_link(self, site, mu):
        out = (ctypes.c_double * 18)()
        _check(lib.gfc_ctx_get_link(self.h, site, mu, out), "get_link")
        return np.array(out[:])

    # ---- fields
    def reunitarize(self):
        _check(lib.gfc_ctx_reunitarize(self.h), "reunitarize")

    def reunitarize_gt(self):
        _check(lib.gfc_ctx_reunitarize_gt(self.h), "reunitarize_gt")

    def save_links(self):
        _check(lib.gfc_ctx_save_links(self.h), "save_links")

    def restore_links(self):
        _check(lib.gfc_ctx_restore_links(self.h), "restore_links")

    def set_identity_gt(self):
        _check(lib.gfc_ctx_set_identity_gt(self.h), "set_identity_gt")

    def status(self):
        s = ctypes.c_uint()
        _check(lib.gfc_ctx_status(self.h, ctypes.byref(s)), "status")
        return s.value

    def halfsweeps(self, first, n, omega=1.95, hits=2, precision=PREC_FP64_EXACT):
        _check(lib.gfc_ctx_halfsweeps(self.h, first, n, omega, hits, precision), "halfsweeps")

    def apply_gt(self):
        """applyGaugeTransformationU with the resident G on all links."""
        _check(lib.gfc_ctx_apply_gt(self.h), "apply_gt")

    def finalize_temporal(self):
        _check(lib.gfc_ctx_finalize_temporal(self.h), "finalize_temporal")

    def sync(self):
        _check(lib.gfc_ctx_sync(self.h), "sync")

    def autotune(self, which=0):
        """Time every compiled launch shape on this lattice; keep the fastest.
        The links are kept in the save_links() slot (replacing a copy saved there
        before) and restored from it afterwards.
        Returns seconds per half-sweep: {"exact": [...], "fast64": [...], "fast32": [...]}."""
        t = np.zeros(49)
        _check(lib.gfc_ctx_autotune(self.h, which, t.ctypes.data), "autotune")
        return {"exact": t[0:5].tolist(), "fast64": t[5:23].tolist(), "fast32": t[23:41].tolist(),
                "fast64_blocked": t[41:45].tolist(), "fast32_blocked": t[45:49].tolist()}

    def set_blocking(self, precision_bits, slices, sweeps):
        _check(lib.gfc_ctx_set_blocking(self.h, precision_bits, slices, sweeps), "set_blocking")

    def blocking(self):
        v = [ctypes.c_int() for _ in range(4)]
        _check(lib.gfc_ctx_get_blocking(self.h, *[ctypes.byref(x) for x in v]), "get_blocking")
        return tuple(x.value for x in v)

    def shapes(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.gfc_ctx_get_shapes(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "get_shapes")
        return a.value, b.value, c.value

    def set_shapes(self, exact=-1, fast64=-1, fast32=-1):
        _check(lib.gfc_ctx_set_shapes(self.h, exact, fast64, fast32), "set_shapes")

    @property
    def kernel_launches(self):
        return lib.gfc_ctx_kernel_launches(self.h)

    @property
    def stream(self):
        return lib.gfc_ctx_stream(self.h)

    # ---- observables
    def e2_theta(self):
        e2, th = ctypes.c_double(), ctypes.c_double()
        _check(lib.gfc_ctx_e2(self.h, ctypes.byref(e2), ctypes.byref(th)), "e2")
        return e2.value, th.value

    def e2_slices(self):
        out = np.empty(self.nt, dtype=np.float64)
        _check(lib.gfc_ctx_e2_slices(self.h, out.ctypes.data), "e2_slices")
        return out

    def functional(self):
        f = ctypes.c_double()
        _check(lib.gfc_ctx_functional(self.h, ctypes.byref(f)), "functional")
        return f.value

    def plaquette(self):
        s, t = ctypes.c_double(), ctypes.c_double()
        _check(lib.gfc_ctx_plaquette(self.h, ctypes.byref(s), ctypes.byref(t)), "plaquette")
        return s.value, t.value

    # ---- the fix
    def fix(self, params=None, opts=None):
        """gaugefixOverrelaxation on the resident lattice; returns (rc, report)."""
        p = params if params is not None else default_params()
        o = opts if opts is not None else options()
        r = Report()
        rc = lib.gfc_ctx_fix(self.h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(r))
        if rc < FIX_BAD_PARAMS:
            raise GFCError(f"gfc_ctx_fix failed ({rc}): {last_error()}")
        return rc, r


def gaugefix_overrelaxation(U, G, ns, nt, params=None, opts=None, device=0):
    """Drop-in of gaugefixOverrelaxation(U, G, params) on host arrays
    (gfc_gaugefix_overrelaxation).

    U: float64 array of 4V*18 (reference layout), fixed in place; G: float64 array
    of V*18, overwritten with the gauge transformation.  Returns the reference's
    return value (sweeps, -1 or -2) and the run report.
    """
    p = params if params is not None else default_params()
    o = opts if opts is not None else options()
    assert U.dtype == np.float64 and U.flags.c_contiguous and U.size == ns ** 3 * nt * 72
    assert G.dtype == np.float64 and G.flags.c_contiguous and G.size == ns ** 3 * nt * 18
    rep = Report()
    rc = lib.gfc_gaugefix_overrelaxation(ns, nt, U.ctypes.data, G.ctypes.data, ctypes.byref(p), ctypes.byref(o),
                                         ctypes.byref(rep), device)
    if rc < FIX_BAD_PARAMS:
        raise GFCError(f"gfc_gaugefix_overrelaxation failed ({rc}): {last_error()}")
    return rc, rep


# ---------------------------------------------------------------- batches --
def _batch_tune_times(t):
    return {"fp32_minb_2_3_4": list(t[0:3]), "fp64_minb_staged_20_30_40_21_31": list(t[3:8]),
            "round_4_8_16": list(t[8:11]), "fp32_warp_ctas_8_11_12": list(t[11:14]),
            "fp64_warp_ctas_8_11_12": list(t[14:17])}


def _bind_batch():
    P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    IP = ctypes.POINTER(ctypes.c_int)
    RP = ctypes.POINTER(Report)
    sig = {
        "gfc_batch_create": (I, [I, S, I, I, ctypes.POINTER(P)]),
        "gfc_batch_destroy": (I, [P]),
        "gfc_batch_slot_bytes": (S, [I, I]),
        "gfc_batch_add": (I, [P, I, I, IP]),
        "gfc_batch_remove": (I, [P, I]),
        "gfc_batch_upload": (I, [P, I, P, I, I]),
        "gfc_batch_synth": (I, [P, I, ctypes.c_uint64, D]),
        "gfc_batch_activate": (I, [P, I, I]),
        "gfc_batch_round": (I, [P, ctypes.POINTER(Params), ctypes.POINTER(Options), IP]),
        "gfc_batch_slot_done": (I, [P, I, IP]),
        "gfc_batch_finalize": (I, [P, I, RP]),
        "gfc_batch_plaquette": (I, [P, I, ctypes.POINTER(D), ctypes.POINTER(D)]),
        "gfc_batch_download_gt": (I, [P, I, P, I, I]),
        "gfc_batch_download_links": (I, [P, I, P, I, I]),
        "gfc_batch_status": (I, [P, ctypes.POINTER(ctypes.c_uint)]),
        "gfc_batch_slice_sweeps": (I, [P, I, P]),
        "gfc_batch_kernel_launches": (ctypes.c_longlong, [P]),
        "gfc_batch_stream": (P, [P]),
        "gfc_batch_set_shape": (I, [P, I, I, I]),
        "gfc_batch_set_staging": (I, [P, I]),
        "gfc_batch_hold": (I, [P, I, I]),
        "gfc_batch_get_shape": (I, [P] + [IP] * 4),
        "gfc_batch_autotune": (I, [P, I, I, ctypes.POINTER(D)]),
        "gfc_batch_fix_all": (I, [P, ctypes.POINTER(Params), ctypes.POINTER(Options), RP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


_bind_batch()


class Batch:
    """Many lattices on one GPU, swept timeslice by timeslice (a gfc_batch)."""

    def __init__(self, max_sites, max_slots=128, max_nt=128, device=0):
        h = ctypes.c_void_p()
        _check(lib.gfc_batch_create(device, int(max_sites), max_slots, max_nt, ctypes.byref(h)), "gfc_batch_create")
        self.h = h
        self.max_slots = max_slots
        self.geom = {}

    def close(self):
        if getattr(self, "h", None):   # None too when __init__ failed
            lib.gfc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def slot_bytes(ns, nt):
        return lib.gfc_batch_slot_bytes(ns, nt)

    def add(self, ns, nt):
        s = ctypes.c_int()
        _check(lib.gfc_batch_add(self.h, ns, nt, ctypes.byref(s)), "gfc_batch_add")
        self.geom[s.value] = (ns, nt)
        return s.value

    def remove(self, slot):
        _check(lib.gfc_batch_remove(self.h, slot), "gfc_batch_remove")
        self.geom.pop(slot, None)

    def upload(self, slot, buf, elem_bytes=8, byteswap=False):
        a = np.ascontiguousarray(buf)
        ns, nt = self.geom[slot]
        assert a.nbytes == ns ** 3 * nt * 4 * 18 * elem_bytes
        _check(lib.gfc_batch_upload(self.h, slot, a.ctypes.data, elem_bytes, int(byteswap)), "gfc_batch_upload")

    def synth(self, slot, seed, scale):
        _check(lib.gfc_batch_synth(self.h, slot, seed, scale), "gfc_batch_synth")

    def activate(self, slot, precision=PREC_MIXED):
        _check(lib.gfc_batch_activate(self.h, slot, precision), "gfc_batch_activate")

    def round(self, params, opts):
        a = ctypes.c_int()
        _check(lib.gfc_batch_round(self.h, ctypes.byref(params), ctypes.byref(opts), ctypes.byref(a)), "round")
        return a.value

    def slot_done(self, slot):
        d = ctypes.c_int()
        _check(lib.gfc_batch_slot_done(self.h, slot, ctypes.byref(d)), "slot_done")
        return bool(d.value)

    def finalize(self, slot):
        r = Report()
        _check(lib.gfc_batch_finalize(self.h, slot, ctypes.byref(r)), "finalize")
        return r

    def plaquette(self, slot):
        s, t = ctypes.c_double(), ctypes.c_double()
        _check(lib.gfc_batch_plaquette(self.h, slot, ctypes.byref(s), ctypes.byref(t)), "plaquette")
        return s.value, t.value

    def download_gt(self, slot, elem_bytes=8, byteswap=False):
        ns, nt = self.geom[slot]
        out = np.empty(ns ** 3 * nt * 18, dtype=np.float64 if elem_bytes == 8 else np.float32)
        _check(lib.gfc_batch_download_gt(self.h, slot, out.ctypes.data, elem_bytes, int(byteswap)), "download_gt")
        return out

    def download_links(self, slot, elem_bytes=8, byteswap=False):
        ns, nt = self.geom[slot]
        out = np.empty(ns ** 3 * nt * 4 * 18, dtype=np.float64 if elem_bytes == 8 else np.float32)
        _check(lib.gfc_batch_download_links(self.h, slot, out.ctypes.data, elem_bytes, int(byteswap)),
               "download_links")
        return out

    def slice_sweeps(self, slot):
        ns, nt = self.geom[slot]
        out = np.empty(nt, dtype=np.int32)
        _check(lib.gfc_batch_slice_sweeps(self.h, slot, out.ctypes.data), "slice_sweeps")
        return out

    def status(self):
        s = ctypes.c_uint()
        _check(lib.gfc_batch_status(self.h, ctypes.byref(s)), "status")
        return s.value

    def set_shape(self, minb32=4, minb64=3, round_sweeps=8):
        _check(lib.gfc_batch_set_shape(self.h, minb32, minb64, round_sweeps), "set_shape")

    def hold(self, slot, hold=True):
        _check(lib.gfc_batch_hold(self.h, slot, int(hold)), "gfc_batch_hold")

    def set_staging(self, stage64):
        _check(lib.gfc_batch_set_staging(self.h, int(stage64)), "set_staging")

    def shape(self):
        v = [ctypes.c_int() for _ in range(4)]
        _check(lib.gfc_batch_get_shape(self.h, *[ctypes.byref(x) for x in v]), "get_shape")
        return dict(minb32=v[0].value, minb64=v[1].value, stage64=v[2].value, round_sweeps=v[3].value)

    def autotune(self, ns, nt):
        """Time the launch shapes on a scratch ns^3 x nt lattice; keep the fastest."""
        t = (ctypes.c_double * 17)()
        _check(lib.gfc_batch_autotune(self.h, ns, nt, t), "gfc_batch_autotune")
        return _batch_tune_times(t)

    @property
    def kernel_launches(self):
        return lib.gfc_batch_kernel_launches(self.h)

    @property
    def stream(self):
        return lib.gfc_batch_stream(self.h)

    def fix_all(self, params, opts):
        reports = (Report * self.max_slots)()
        rounds = lib.gfc_batch_fix_all(self.h, ctypes.byref(params), ctypes.byref(opts), reports)
        if rounds < 0:
            raise GFCError(f"gfc_batch_fix_all failed ({rounds}): {last_error()}")
        return rounds, {s: reports[s] for s in list(self.geom)}


def _bind_server():
    P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    IP, DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    sig = {
        "gfc_server_create": (I, [I, S, D, I, I, ctypes.POINTER(P)]),
        "gfc_server_destroy": (I, [P]),
        "gfc_server_capacity_sites": (S, [P]),
        "gfc_server_submit": (I, [P, I, I, P, I, I, ctypes.c_uint64, D, I, ctypes.POINTER(ctypes.c_int64)]),
        "gfc_server_step": (I, [P, ctypes.POINTER(Params), ctypes.POINTER(Options), IP, IP]),
        "gfc_server_poll": (I, [P, ctypes.c_int64, IP, DP, DP, ctypes.POINTER(Report)]),
        "gfc_server_fetch": (I, [P, ctypes.c_int64, P, I, I]),
        "gfc_server_result": (I, [P, ctypes.c_int64, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                  ctypes.POINTER(ctypes.c_size_t)]),
        "gfc_server_batch": (P, [P]),
        "gfc_server_reserve_host": (I, [P, S, I]),
        "gfc_server_set_policy": (I, [P, I, S]),
        "gfc_server_stats": (I, [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


_bind_server()

REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FETCHED = 0, 1, 2, 3
SERVE_ALL, SERVE_SMALLEST_FIRST = 0, 1


class Server:
    """Request loop with continuous batching over one Batch (a gfc_server).

    submit() queues a lattice; step() admits what fits in free device memory,
    runs one round and finalises finished requests; fetch() returns G and frees
    the request's device memory."""

    def __init__(self, max_sites=0, mem_fraction=0.85, max_slots=256, max_nt=128, device=0):
        h = ctypes.c_void_p()
        _check(lib.gfc_server_create(device, int(max_sites), mem_fraction, max_slots, max_nt, ctypes.byref(h)),
               "gfc_server_create")
        self.h = h
        self.geom = {}

    def close(self):
        if getattr(self, "h", None):   # None too when __init__ failed
            lib.gfc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def capacity_sites(self):
        return lib.gfc_server_capacity_sites(self.h)

    def submit(self, ns, nt, links=None, elem_bytes=8, byteswap=False, seed=0, scale=0.5, precision=PREC_MIXED):
        rid = ctypes.c_int64()
        ptr = None
        if links is not None:
            links = np.ascontiguousarray(links)
            assert links.nbytes == ns ** 3 * nt * 4 * 18 * elem_bytes
            ptr = links.ctypes.data
        _check(lib.gfc_server_submit(self.h, ns, nt, ptr, elem_bytes, int(byteswap), seed, scale, precision,
                                     ctypes.byref(rid)), "gfc_server_submit")
        self.geom[rid.value] = (ns, nt)
        return rid.value

    def step(self, params, opts):
        r, q = ctypes.c_int(), ctypes.c_int()
        _check(lib.gfc_server_step(self.h, ctypes.byref(params), ctypes.byref(opts), ctypes.byref(r),
                                   ctypes.byref(q)), "gfc_server_step")
        return r.value, q.value

    def poll(self, rid):
        st, ta, td = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        rep = Report()
        _check(lib.gfc_server_poll(self.h, rid, ctypes.byref(st), ctypes.byref(ta), ctypes.byref(td),
                                   ctypes.byref(rep)), "gfc_server_poll")
        return st.value, ta.value, td.value, rep

    def fetch(self, rid, elem_bytes=8, release=True, want_gt=True):
        out = None
        if want_gt:
            ns, nt = self.geom[rid]
            out = np.empty(ns ** 3 * nt * 18, dtype=np.float64 if elem_bytes == 8 else np.float32)
        _check(lib.gfc_server_fetch(self.h, rid, None if out is None else out.ctypes.data, elem_bytes,
                                    int(release)), "gfc_server_fetch")
        return out

    def result_view(self, rid):
        """G of a done request as a read-only view of the server's host copy
        (valid until fetch(..., release=True))."""
        p, n = ctypes.POINTER(ctypes.c_double)(), ctypes.c_size_t()
        _check(lib.gfc_server_result(self.h, rid, ctypes.byref(p), ctypes.byref(n)), "gfc_server_result")
        a = np.ctypeslib.as_array(p, shape=(n.value,))
        a.flags.writeable = False
        return a

    def set_policy(self, policy, work_sites=0):
        """SERVE_ALL: every admitted request sweeps each round; SERVE_SMALLEST_FIRST:
        the smallest running requests, up to work_sites sites, the others wait."""
        _check(lib.gfc_server_set_policy(self.h, policy, int(work_sites)), "gfc_server_set_policy")

    def reserve_host(self, buffer_bytes, count):
        """Pin host result buffers ahead of time."""
        _check(lib.gfc_server_reserve_host(self.h, int(buffer_bytes), count), "gfc_server_reserve_host")

    def stats(self):
        """Host seconds per phase of step() and the rounds run."""
        sec, n = (ctypes.c_double * 4)(), ctypes.c_longlong()
        _check(lib.gfc_server_stats(self.h, sec, ctypes.byref(n)), "gfc_server_stats")
        return dict(release_s=sec[0], admission_s=sec[1], rounds_s=sec[2], finalize_s=sec[3], rounds=n.value)

    def release(self, rid):
        _check(lib.gfc_server_fetch(self.h, rid, None, 8, 1), "gfc_server_fetch")

    def autotune(self, ns, nt):
        """Launch shapes of the server's batch, timed on a scratch ns^3 x nt lattice
        (before requests are admitted)."""
        t = (ctypes.c_double * 17)()
        _check(lib.gfc_batch_autotune(lib.gfc_server_batch(self.h), ns, nt, t), "gfc_batch_autotune")
        return _batch_tune_times(t)

    def batch_stream(self):
        return lib.gfc_batch_stream(lib.gfc_server_batch(self.h))

    def kernel_launches(self):
        return lib.gfc_batch_kernel_launches(lib.gfc_server_batch(self.h))

"""The C-ABI library loads without a GPU and exports every function the public
headers declare; the drop-in program and the oracle are built."""
import ctypes
import os
import re
import subprocess

import gfc
from conftest import PKG, ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(", text):
        name = m.group(1)
        start = text.rfind("\n", 0, m.start()) + 1
        line = text[start:m.start()]
        if line.lstrip().startswith("#") or "typedef" in line:
            continue
        if name in ("if", "for", "while", "return", "sizeof", "defined"):
            continue
        # a declaration: preceded on its line by a type (not an expression)
        if re.search(r"(void|int|double|float|char|long|unsigned|size_t|gfc_\w+|\*|[A-Z]\w+)\s*\**\s*$", line):
            names.add(name)
    return names


def test_headers_exist():
    assert any(h.endswith("gfc.h") for h in HEADERS)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(gfc.LIB_PATH)
    missing = []
    for h in HEADERS:
        for name in sorted(declared_functions(h)):
            if not hasattr(lib, name):
                missing.append(f"{os.path.basename(h)}:{name}")
    assert not missing, missing


def test_exports_via_nm():
    out = subprocess.run(["nm", "-D", "--defined-only", gfc.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for h in HEADERS:
        for name in declared_functions(h):
            assert name in exported, name


def test_cli_built_and_linked():
    cli = os.path.join(PKG, "bin", "gauge_fix_coulomb")
    assert os.access(cli, os.X_OK)
    out = subprocess.run(["ldd", cli], capture_output=True, text=True).stdout
    assert "libgfc.so" in out and "not found" not in out


def test_build_targets_sm100a_only():
    """The build recipe compiles device code for sm_100a and nothing else (the
    loaded architecture itself is checked on a GPU by
    tests/test_gpu_observables_io.py::test_device_code_is_sm100a)."""
    import re

    mk = open(os.path.join(PKG, "Makefile")).read()
    arch = re.search(r"^ARCH\s*:=\s*(.*)$", mk, re.M).group(1).split()
    assert arch == ["-gencode", "arch=compute_100a,code=sm_100a"]


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_no_gpu_fails_loudly():
    """Without a GPU there is no fallback: creating a context, a batch or a server
    returns an error code with a message, and the binding raises."""
    import pytest

    if _has_gpu():
        pytest.skip("a GPU is present")
    lib = ctypes.CDLL(gfc.LIB_PATH)
    h = ctypes.c_void_p()
    for call in (lambda: lib.gfc_ctx_create(4, 8, 0, 0, ctypes.byref(h)),
                 lambda: lib.gfc_batch_create(0, ctypes.c_size_t(4096), 2, 8, ctypes.byref(h)),
                 lambda: lib.gfc_server_create(0, ctypes.c_size_t(4096), ctypes.c_double(0.5), 2, 8,
                                               ctypes.byref(h))):
        rc = call()
        assert rc < 0 and not h.value
        assert gfc.last_error()
    with pytest.raises(gfc.GFCError):
        gfc.Lattice(4, 8)
    with pytest.raises(gfc.GFCError):
        gfc.Batch(max_sites=4096, max_slots=2, max_nt=8)


def test_bad_arguments_rejected_before_any_device_work():
    lib = ctypes.CDLL(gfc.LIB_PATH)
    h = ctypes.c_void_p()
    assert lib.gfc_ctx_create(4, 8, 0, 0, None) < 0
    assert lib.gfc_batch_create(0, ctypes.c_size_t(0), 2, 8, ctypes.byref(h)) == -10   # max_sites 0
    assert lib.gfc_batch_create(0, ctypes.c_size_t(4096), 0, 8, ctypes.byref(h)) == -10  # no slots
    assert lib.gfc_server_create(0, ctypes.c_size_t(4096), ctypes.c_double(0.5), 0, 8, ctypes.byref(h)) == -10
    assert lib.gfc_gaugefix_overrelaxation(4, 8, None, None, None, None, None, 0) == -10


def test_geometry_limits_rejected_before_any_device_work():
    """Extents the 32-bit site indexing cannot address, and empty extents, are refused
    with GFC_ERR_GEOMETRY before anything touches a device."""
    lib = ctypes.CDLL(gfc.LIB_PATH)
    h = ctypes.c_void_p()
    assert lib.gfc_ctx_create(512, 512, 0, 0, ctypes.byref(h)) == -13   # 4V > 2^31
    assert lib.gfc_ctx_create(0, 8, 0, 0, ctypes.byref(h)) == -13
    assert lib.gfc_ctx_create(4, -1, 0, 0, ctypes.byref(h)) == -13
    assert "too large" in gfc.last_error() or "extents" in gfc.last_error()

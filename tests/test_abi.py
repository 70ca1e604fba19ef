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


def test_library_is_sm100a():
    """The library carries sm_100a device code (cuobjdump is not used: the
    embedded architecture list is read from the ELF notes via the build flags)."""
    mk = open(os.path.join(PKG, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk

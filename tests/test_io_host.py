"""Host-side file access: the reference's size checks and return codes
(loadConfig, fields_io.c:216-305) and the byte swap (fields_io.c:42-96)."""
import ctypes

import numpy as np

import gfc


def test_read_exact_codes(tmp_path):
    buf = np.zeros(64, dtype=np.uint8)
    f = tmp_path / "f.bin"
    f.write_bytes(bytes(range(64)))
    assert gfc.lib.gfc_read_exact(str(f).encode(), buf.ctypes.data, 64, 0) == 0
    assert bytes(buf) == bytes(range(64))
    assert gfc.lib.gfc_read_exact(str(tmp_path / "none").encode(), buf.ctypes.data, 64, 0) == -1
    assert gfc.lib.gfc_read_exact(str(f).encode(), buf.ctypes.data, 65, 0) == -2   # short
    assert gfc.lib.gfc_read_exact(str(f).encode(), buf.ctypes.data, 63, 0) == -3   # longer than the lattice
    assert gfc.lib.gfc_read_exact(str(f).encode(), buf.ctypes.data, 63, 1) == -2   # GT flavour


def test_write_all(tmp_path):
    a = np.arange(10, dtype=np.float64)
    p = tmp_path / "w.bin"
    assert gfc.lib.gfc_write_all(str(p).encode(), a.ctypes.data, a.nbytes) == 0
    assert np.array_equal(np.fromfile(p, dtype=np.float64), a)
    assert gfc.lib.gfc_write_all(str(tmp_path / "no" / "dir.bin").encode(), a.ctypes.data, a.nbytes) == -1


def test_byteswap_roundtrip():
    rng = np.random.default_rng(0)
    for dt, w in ((np.float64, 8), (np.float32, 4)):
        a = rng.standard_normal(1001).astype(dt)
        b = a.copy()
        assert gfc.lib.gfc_byteswap(b.ctypes.data, w, b.nbytes) == 0
        assert b.tobytes() == a.byteswap().tobytes()   # compare bits: swapped words can be NaN
        assert gfc.lib.gfc_byteswap(b.ctypes.data, w, b.nbytes) == 0
        assert b.tobytes() == a.tobytes()
    c = np.arange(6, dtype=np.uint8)
    assert gfc.lib.gfc_byteswap(c.ctypes.data, 3, 6) == -1
    assert gfc.lib.gfc_byteswap(c.ctypes.data, 1, 6) == 0 and list(c) == list(range(6))

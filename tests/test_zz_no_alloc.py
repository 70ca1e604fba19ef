"""The allocation-free e2/theta entry point (gfc_e2_theta_device_noalloc).

It serves callers that cannot let the library allocate device memory: their own
allocator owns the GPU, or a cudaFree's device-wide synchronisation would stall
other work sharing the GPU.  It takes links that already live in device memory
(the caller's buffer) and keeps its scratch in a fixed array inside the library.

Checked here through the C ABI against the context entry point (gfc_ctx_e2, which
allocates its own scratch) and against the CPU oracle's calculate_e2 and
calculateTheta, on two calls in a row so that the second call sees the scratch the
first one left behind.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import gfc
import oracle_ref as orc

pytestmark = pytest.mark.gpu


def noalloc(ns, nt, ptr, stream=None):
    e2, th = ctypes.c_double(), ctypes.c_double()
    rc = gfc.lib.gfc_e2_theta_device_noalloc(ns, nt, ptr, stream, ctypes.byref(e2), ctypes.byref(th))
    return rc, e2.value, th.value


@pytest.mark.parametrize("ns,nt,seed", [(8, 8, 61), (6, 12, 62)])
def test_noalloc_matches_context_entry_point(ns, nt, seed):
    import torch

    U = gfc.synth_config(ns, nt, seed, 0.6)
    with gfc.Lattice(ns, nt) as lat:      # the existing entry point
        lat.upload_links(U, 8, False)
        e2_ref, th_ref = lat.e2_theta()
    u_dev = torch.from_numpy(U).to("cuda:0")   # the caller's own device buffer
    torch.cuda.synchronize()
    for _ in range(2):                          # two calls in a row share the scratch
        rc, e2, th = noalloc(ns, nt, u_dev.data_ptr())
        assert rc == gfc.GFC_OK, gfc.last_error()
        assert e2 == pytest.approx(e2_ref, rel=1e-13)
        assert th == pytest.approx(th_ref, rel=1e-13)
        assert e2 == pytest.approx(orc.e2(U, ns, nt), rel=1e-12)
        assert th == pytest.approx(orc.theta(U, ns, nt), rel=1e-12)
    # a second, different lattice right after: no stale partial sums are reused
    U2 = gfc.synth_config(4, 5, seed + 100, 0.4)
    with gfc.Lattice(4, 5) as lat:
        lat.upload_links(U2, 8, False)
        e2b_ref, thb_ref = lat.e2_theta()
    u2_dev = torch.from_numpy(U2).to("cuda:0")
    torch.cuda.synchronize()
    rc, e2b, thb = noalloc(4, 5, u2_dev.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == gfc.GFC_OK
    assert e2b == pytest.approx(e2b_ref, rel=1e-13) and thb == pytest.approx(thb_ref, rel=1e-13)
    assert e2b == pytest.approx(orc.e2(U2, 4, 5), rel=1e-12) and thb == pytest.approx(orc.theta(U2, 4, 5), rel=1e-12)


def test_noalloc_rejects_what_does_not_fit():
    """Too many timeslices for the fixed scratch, a misaligned pointer, or links
    that are not in this GPU's memory: a clear error, no kernel launched (the
    pointer is never dereferenced)."""
    import torch

    buf = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    rc, _, _ = noalloc(1, 20000, buf.data_ptr())
    assert rc == -10 and "scratch" in gfc.last_error()
    rc, _, _ = noalloc(2, 2, buf.data_ptr() + 8)
    assert rc == -10 and "aligned" in gfc.last_error()
    # page-locked host memory is reachable from the GPU, but it is not device memory
    # of this GPU: refused before any launch
    host = torch.zeros(2 ** 3 * 2 * 4 * 18, dtype=torch.float64).pin_memory()
    rc, _, _ = noalloc(2, 2, host.data_ptr())
    assert rc == -10 and "device memory" in gfc.last_error()

"""The seeded synthetic configuration generator (host/gfc_synth.c)."""
import os
import subprocess
import sys

import numpy as np

import gfc
from conftest import PKG


def as_matrices(U):
    M = U.reshape(-1, 9, 2)
    return (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)


def test_links_are_su3():
    M = as_matrices(gfc.synth_config(4, 4, 7, 0.5))
    eye = np.eye(3)
    assert np.abs(M @ M.conj().transpose(0, 2, 1) - eye).max() < 1e-13
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-13


def test_deterministic_and_seeded():
    a = gfc.synth_config(4, 4, 7, 0.5)
    b = gfc.synth_config(4, 4, 7, 0.5)
    c = gfc.synth_config(4, 4, 8, 0.5)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


def test_thread_count_independent():
    code = ("import sys; sys.path.insert(0, %r); import gfc, hashlib; "
            "print(hashlib.sha256(gfc.synth_config(6, 4, 3, 0.7).tobytes()).hexdigest())" % PKG)
    outs = set()
    for n in ("1", "5"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        outs.add(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                check=True).stdout.strip())
    assert len(outs) == 1


def test_pure_gauge_limit():
    """scale 0: U_mu(x) = g(x) g(x+mu)^dagger, a pure gauge whose plaquettes are 1."""
    ns, nt = 4, 4
    M = as_matrices(gfc.synth_config(ns, nt, 5, 0.0)).reshape(nt, ns, ns, ns, 4, 3, 3)
    # plaquette in the (x, y) plane at the origin: U_x(0) U_y(0+x) U_x(0+y)^dag U_y(0)^dag
    ux, uy = M[..., 3, :, :], M[..., 2, :, :]
    p = ux[0, 0, 0, 0] @ uy[0, 0, 0, 1] @ ux[0, 0, 1, 0].conj().T @ uy[0, 0, 0, 0].conj().T
    assert abs(np.trace(p).real / 3 - 1) < 1e-13

"""Comparison of gauge transformations up to the residual gauge freedom of Coulomb
gauge (test infrastructure).

Coulomb gauge fixes G only up to a rotation that is constant in space on each
timeslice: G(x) -> h(t) G(x) leaves div A = 0, e2, theta and the gauge functional
unchanged.  Paths that round differently from the reference (the FP32 phase of the
mixed path above all) drift along that flat direction, so their G is compared with
the reference's after removing the best-fitting h(t) of each timeslice.
"""
import numpy as np


def mats(G):
    M = np.asarray(G).reshape(-1, 9, 2)
    return (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)


def global_rotation_residual(G, Gref, t_of_site):
    """(max |G(x) - h(t) Gref(x)|, max |h(t) - 1|) with h(t) the unitary polar factor
    of sum over the timeslice of G(x) Gref(x)^dagger."""
    A, B = mats(G), mats(Gref)
    t_of_site = np.asarray(t_of_site)
    res, drift = 0.0, 0.0
    for t in np.unique(t_of_site):
        sel = t_of_site == t
        M = np.einsum("nij,nkj->ik", A[sel], B[sel].conj())
        w, _, vh = np.linalg.svd(M)
        h = w @ vh
        res = max(res, np.abs(A[sel] - h @ B[sel]).max())
        drift = max(drift, np.abs(h - np.eye(3)).max())
    return res, drift

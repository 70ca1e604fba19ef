"""Edge lattices on the GPU: the smallest extents (ns = 2, where a site's forward and
backward neighbours coincide; ns = 1), a single timeslice (nt = 1, the temporal
link closes on its own site), odd nt, and odd ns (7, 9: sites swept in parallel by
boundary level, which must give the oracle's sequential z, y, x order bit for bit),
on the exact, fast, mixed and batch paths."""
import numpy as np
import pytest

import gfc
import oracle_ref as orc

pytestmark = pytest.mark.gpu
TOL = 1e-15


def su3_error(G):
    M = G.reshape(-1, 9, 2)
    M = (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)
    return max(np.abs(M @ M.conj().transpose(0, 2, 1) - np.eye(3)).max(), np.abs(np.linalg.det(M) - 1).max())


def unfixed(ns, nt, seed):
    U = gfc.synth_config(ns, nt, seed, 0.5)
    orc.reunitarize(U)
    return U


@pytest.mark.parametrize("ns,nt", [(2, 1), (4, 1), (2, 3), (6, 1), (1, 4), (7, 5), (9, 6)])
def test_exact_oracle_fix_bit_for_bit(ns, nt):
    """The reference-arithmetic fix with the reference schedule against the oracle."""
    U = unfixed(ns, nt, 61)
    V = ns ** 3 * nt
    Uo = U.copy()
    Go = np.zeros(V * 18)
    rc_o = orc.fix(Uo, Go, ns, nt, tol=1e-14)[0]
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        rc, rep = lat.fix(gfc.default_params(tolerance=1e-14))
        G = lat.download_gt()
        Ug = lat.download_links()
    assert rc == rc_o
    assert orc.sha(G) == orc.sha(Go)
    assert orc.sha(Ug.reshape(-1, 4, 18)[:, 1:4, :]) == orc.sha(Uo.reshape(-1, 4, 18)[:, 1:4, :])


@pytest.mark.parametrize("ns,nt", [(2, 1), (4, 1), (2, 5), (6, 3), (5, 4)])
@pytest.mark.parametrize("prec", [gfc.PREC_FP64_FAST, gfc.PREC_MIXED, gfc.PREC_FP64_FULL])
def test_fast_paths_on_edge_lattices(ns, nt, prec):
    U0 = unfixed(ns, nt, 62)
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        ps0, pt0 = lat.plaquette()
        rc, rep = lat.fix(gfc.default_params(tolerance=TOL), gfc.options(precision=prec, stop_rule=gfc.STOP_EVERY))
        G = lat.download_gt()
        U = lat.download_links()
        ps1, pt1 = lat.plaquette()
    assert rc >= 0 and rep.final_residue <= TOL
    assert su3_error(G) < 1e-13
    assert abs(ps1 - ps0) < 1e-13 and abs(pt1 - pt0) < 1e-13
    U1 = U0.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(U1, U, atol=1e-12)


def test_batch_edge_lattices_alone_and_mixed():
    """Tiny and single-timeslice lattices beside a larger one retire correctly and
    give the same G as when fixed alone."""
    geoms = [(2, 1, 63), (4, 1, 64), (2, 3, 65), (6, 4, 66), (1, 4, 67)]
    p, o = gfc.default_params(tolerance=TOL), gfc.options(precision=gfc.PREC_MIXED)
    alone = {}
    for ns, nt, seed in geoms:
        with gfc.Batch(max_sites=10 ** 5, max_slots=2, max_nt=8) as b:
            s = b.add(ns, nt)
            b.upload(s, gfc.synth_config(ns, nt, seed, 0.5), 8, False)
            b.activate(s, gfc.PREC_MIXED)
            _, reps = b.fix_all(p, o)
            assert reps[s].e2 <= TOL
            alone[(ns, nt)] = b.download_gt(s)
    with gfc.Batch(max_sites=10 ** 5, max_slots=8, max_nt=8) as b:
        slots = {}
        for ns, nt, seed in geoms:
            s = b.add(ns, nt)
            b.upload(s, gfc.synth_config(ns, nt, seed, 0.5), 8, False)
            b.activate(s, gfc.PREC_MIXED)
            slots[(ns, nt)] = s
        _, reps = b.fix_all(p, o)
        for g, s in slots.items():
            assert reps[s].e2 <= TOL
            G = b.download_gt(s)
            assert su3_error(G) < 1e-13
            assert G.tobytes() == alone[g].tobytes()
            # the links returned are G U G^dagger of the uploaded ones (ns = 1: unchanged)
            ns, nt = g
            U0 = unfixed(ns, nt, dict((k[:2], k[2]) for k in geoms)[g])
            orc.apply_gt(U0, G, ns, nt)
            np.testing.assert_allclose(b.download_links(s), U0, atol=1e-12)


@pytest.mark.parametrize("ns,nt", [(1, 4), (3, 2), (5, 3)])
@pytest.mark.parametrize("prec", [gfc.PREC_FP64_EXACT, gfc.PREC_FP64_FAST])
def test_half_sweeps_on_odd_ns(ns, nt, prec):
    """Half-sweeps on odd ns (the fix of ns = 1 never sweeps: its e2 vanishes
    identically): the exact path gives the oracle's links and G bit for bit after each
    half-sweep, ns = 1 included, where a link is its site's forward and backward link
    and is updated twice in turn; the fast path gives them to rounding."""
    U = unfixed(ns, nt, 71)
    V = ns ** 3 * nt
    Uo, Go = U.copy(), np.zeros(V * 18)
    Go[0::18] = Go[8::18] = Go[16::18] = 1.0
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        lat.set_identity_gt()
        for k in range(4):
            lat.halfsweeps(k, 1, 1.95, 2, prec)
            orc.halfsweep(Uo, Go, ns, nt, k)
            G = lat.download_gt()
            Ug = lat.download_links()
            if prec == gfc.PREC_FP64_EXACT or ns == 1:
                assert orc.sha(G) == orc.sha(Go), k
                assert orc.sha(Ug.reshape(-1, 4, 18)[:, 1:4, :]) == orc.sha(Uo.reshape(-1, 4, 18)[:, 1:4, :]), k
            else:
                np.testing.assert_allclose(G, Go, atol=1e-13)
                np.testing.assert_allclose(Ug.reshape(-1, 4, 18)[:, 1:4, :], Uo.reshape(-1, 4, 18)[:, 1:4, :],
                                           atol=1e-13)

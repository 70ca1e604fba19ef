"""The fast FP64 path and the FP32-bulk / FP64-refine path.

They do not round like the reference, so parity is stated through what the fix
must deliver: e2 <= tolerance, G in SU(3), G U0 G^dagger = the returned links,
plaquettes unchanged to 1e-13, and the same Coulomb gauge as the oracle (the
functional F agrees to 1e-10 relative and the half-sweep count to within 1 %)."""
import numpy as np
import pytest

import gfc
import oracle_ref as orc

pytestmark = pytest.mark.gpu


def su3_error(G):
    M = G.reshape(-1, 9, 2)
    M = (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)
    unit = np.abs(M @ M.conj().transpose(0, 2, 1) - np.eye(3)).max()
    det = np.abs(np.linalg.det(M) - 1).max()
    return max(unit, det)


def first_below(ns, nt, U0, tol, omega=1.95, hits=2):
    """Half-sweeps until the oracle's e2 first reaches tol (checked every half-sweep)."""
    U = U0.copy()
    V = ns ** 3 * nt
    G = np.zeros(V * 18)
    G.reshape(V, 9, 2)[:, [0, 4, 8], 0] = 1.0
    k = 0
    while orc.e2(U, ns, nt) > tol:
        orc.halfsweep(U, G, ns, nt, k, omega, hits)
        k += 1
        if k % 250 == 0:
            orc.reunitarize(U)
            orc.reunitarize(G)
    return k, U, G


@pytest.mark.parametrize("prec", [gfc.PREC_FP64_FAST, gfc.PREC_FP64_EXACT, gfc.PREC_MIXED])
def test_every_sweep_stopping(prec):
    ns, nt, tol = 8, 8, 1e-15
    U0 = gfc.synth_config(ns, nt, 51, 0.5)
    orc.reunitarize(U0)
    k_ref, Uref, Gref = first_below(ns, nt, U0, tol)
    with gfc.Lattice(ns, nt, mixed=(prec == gfc.PREC_MIXED)) as lat:
        lat.upload_links(U0, 8, False)
        ps0, pt0 = lat.plaquette()
        p = gfc.default_params(tolerance=tol)
        rc, rep = lat.fix(p, gfc.options(precision=prec, stop_rule=gfc.STOP_EVERY))
        ps1, pt1 = lat.plaquette()
        G = lat.download_gt()
        U = lat.download_links()
        e2, _ = lat.e2_theta()
    assert rc > 0 and rep.first_below_tol >= 0
    assert e2 <= tol and rep.final_residue <= tol
    assert su3_error(G) < 1e-13
    assert abs(ps1 - ps0) < 1e-13 and abs(pt1 - pt0) < 1e-13
    # the returned links are G U0 G^dagger
    U1 = U0.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(U1, U, atol=1e-12)
    # same gauge functional as the FP64 oracle at its stopping point
    assert rep.functional == pytest.approx(orc.functional(Uref, ns, nt), rel=1e-10)
    if prec != gfc.PREC_MIXED:
        # the fused test sees e2 one half-sweep late (see gfc_fast.cu)
        assert abs(rep.first_below_tol - k_ref) <= max(1, 0.01 * k_ref)


def test_fast_tracks_exact_per_sweep():
    """The fast update follows the reference update to rounding for many sweeps."""
    ns, nt = 8, 8
    U0 = gfc.synth_config(ns, nt, 52, 0.5)
    orc.reunitarize(U0)
    out = {}
    for prec in (gfc.PREC_FP64_EXACT, gfc.PREC_FP64_FAST):
        with gfc.Lattice(ns, nt) as lat:
            lat.upload_links(U0, 8, False)
            lat.set_identity_gt()
            e2 = []
            for k in range(200):
                lat.halfsweeps(k, 1, 1.95, 2, prec)
                e2.append(lat.e2_theta()[0])
            out[prec] = (np.array(e2), lat.functional())
    np.testing.assert_allclose(out[gfc.PREC_FP64_FAST][0], out[gfc.PREC_FP64_EXACT][0], rtol=1e-6)
    assert out[gfc.PREC_FP64_FAST][1] == pytest.approx(out[gfc.PREC_FP64_EXACT][1], rel=1e-12)


# shape indices by kernel body: plain, all six links staged in shared memory, four
# staged, two staged (gfc_ctx_autotune's order)
BODIES = [range(0, 9), range(9, 15), range(15, 17), range(17, 18)]


def test_every_launch_shape_gives_the_same_fix():
    """The autotuner may pick any compiled shape.  Shapes of one kernel body compute
    the same bits for the same half-sweeps: checked on a fixed number of half-sweeps
    (exact and FP64 fast), and on the fixes of one body that stop at the same
    half-sweep (the fused e2 is summed in a shape-dependent order, so a fix may stop
    one half-sweep apart).  Across bodies the staged forms evaluate the same
    expressions but may be scheduled differently, so the fix agrees to rounding: the
    same gauge functional, G to the accuracy e2 allows, the sweep count to one
    half-sweep."""
    ns, nt = 8, 8
    U0 = gfc.synth_config(ns, nt, 53, 0.5)
    orc.reunitarize(U0)
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        lat.save_links()
        times = lat.autotune()
        assert all(t > 0 for t in times["exact"] + times["fast64"] + times["fast32"])
        assert lat.download_links().tobytes() == U0.tobytes()   # restored after tuning
        for kind in ("exact", "fast64", "fast32"):
            prec = {"exact": gfc.PREC_FP64_EXACT, "fast64": gfc.PREC_FP64_FAST, "fast32": gfc.PREC_MIXED}[kind]
            runs, fixed = [], []
            for s in range(len(times[kind])):
                lat.set_shapes(**{kind: s})
                lat.restore_links()
                rc, rep = lat.fix(gfc.default_params(tolerance=1e-14),
                                  gfc.options(precision=prec, stop_rule=gfc.STOP_EVERY))
                assert rc > 0
                runs.append((rc, rep.functional, lat.download_gt()))
                if kind != "fast32":
                    lat.restore_links()
                    lat.set_identity_gt()
                    lat.halfsweeps(0, 24, 1.95, 2, prec)
                    fixed.append(orc.sha(lat.download_gt()) + orc.sha(lat.download_links()))
            bodies = [range(len(runs))] if kind == "exact" else BODIES
            assert sum(len(b) for b in bodies) == len(runs)
            for body in bodies:
                if fixed:
                    assert len({fixed[i] for i in body}) == 1, kind
                for rc in {runs[i][0] for i in body}:
                    assert len({orc.sha(runs[i][2]) for i in body if runs[i][0] == rc}) == 1, kind
            for rc, F, G in runs:
                assert abs(rc - runs[0][0]) <= 1
                assert F == pytest.approx(runs[0][1], rel=1e-12)
                np.testing.assert_allclose(G, runs[0][2], atol=1e-6)

def test_slice_blocking_same_results():
    """Timeslices share no link during the sweeps, so running groups of them for
    several half-sweeps at a time changes nothing but the order of independent
    work: same first half-sweep below tolerance, and G bit-identical to the same
    number of unblocked half-sweeps."""
    ns, nt = 8, 8
    U0 = gfc.synth_config(ns, nt, 54, 0.5)
    orc.reunitarize(U0)
    p = gfc.default_params(tolerance=1e-15, sweeps_to_reunitarization=100000)
    o = gfc.options(precision=gfc.PREC_FP64_FAST, stop_rule=gfc.STOP_EVERY)
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        lat.save_links()
        rc0, r0 = lat.fix(p, o)
        lat.restore_links()
        lat.set_blocking(2 | 4, 3, 4)          # groups of 3 slices (ragged last group), 4 half-sweeps
        rc1, r1 = lat.fix(p, o)
        G1 = lat.download_gt()
        assert r1.first_below_tol == r0.first_below_tol
        assert rc1 % 4 == 0 and rc1 >= r0.first_below_tol + 1 and r1.final_residue <= 1e-15
        lat.restore_links()
        lat.set_identity_gt()
        lat.halfsweeps(0, rc1, 1.95, 2, gfc.PREC_FP64_FAST)
        lat.reunitarize_gt()
        assert orc.sha(lat.download_gt()) == orc.sha(G1)
        # mixed precision with blocking in both phases still reaches the tolerance
        lat.restore_links()
        rc2, r2 = lat.fix(p, gfc.options(precision=gfc.PREC_MIXED, stop_rule=gfc.STOP_EVERY))
        assert rc2 > 0 and r2.final_residue <= 1e-15


@pytest.mark.parametrize("precision", [gfc.PREC_FP64_FAST, gfc.PREC_MIXED, gfc.PREC_FP64_FULL,
                                       gfc.PREC_FP64_EXACT])
def test_sparse_e2_measurement_stops_at_the_same_half_sweep(precision):
    """Measuring e2 only on one pair of half-sweeps per chunk while the tolerance is
    far must not change the stop: same first half-sweep below tolerance, same G."""
    ns, nt = 8, 12
    U0 = gfc.synth_config(ns, nt, 57, 0.5)
    out = {}
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        lat.reunitarize()
        lat.save_links()
        for dense in (1, 0):
            lat.restore_links()
            rc, rep = lat.fix(gfc.default_params(tolerance=1e-15),
                              gfc.options(precision=precision, stop_rule=gfc.STOP_EVERY, dense_check=dense))
            out[dense] = (rc, rep.first_below_tol, rep.sweeps_fp32, orc.sha(lat.download_gt()))
            assert rep.final_residue <= 1e-15
    assert out[0] == out[1]


@pytest.mark.parametrize("warm", [0, 1])
def test_mixed_refresh_out_of_sweeps_leaves_a_consistent_state(warm):
    """A mixed fix with FP32 rebuilds that runs out of half-sweeps in the FP32 phase
    returns GFC_FIX_NOT_CONVERGED with the FP64 fields at the last rebuild: G in SU(3)
    and the links equal to G U G^dagger of the links it started from."""
    ns, nt = 6, 8
    U0 = gfc.synth_config(ns, nt, 61, 0.6)
    orc.reunitarize(U0)
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        if warm:
            lat.set_identity_gt()
        rc, rep = lat.fix(gfc.default_params(tolerance=1e-15, max_sweeps_to_fix=100),
                          gfc.options(precision=gfc.PREC_MIXED, stop_rule=gfc.STOP_EVERY, switch_e2=1e-12,
                                      fp32_refresh=32, warm_start=warm))
        G = lat.download_gt()
        U = lat.download_links()
    assert rc == gfc.FIX_NOT_CONVERGED
    assert su3_error(G) < 1e-13
    ident = np.zeros((9, 2))
    ident[[0, 4, 8], 0] = 1.0
    assert np.abs(G.reshape(-1, 9, 2) - ident).max() > 1e-3   # the rebuilds moved G
    U1 = U0.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(U1, U, atol=1e-12)


@pytest.mark.parametrize("refresh,switch", [(64, 1e-11), (128, 1e-11), (16, 1e-10)])
def test_mixed_with_fp32_refresh(refresh, switch):
    """The mixed path with the FP32 links rebuilt from the FP64 start (as G U0 G^dagger
    with the FP32 G folded into an FP64 G) every `refresh` half-sweeps: the result is
    the fix the FP64 oracle gives (e2 below the tolerance, the same gauge functional,
    G in SU(3), links G U0 G^dagger, plaquettes unchanged)."""
    ns, nt, tol = 8, 8, 1e-15
    U0 = gfc.synth_config(ns, nt, 58, 0.5)
    orc.reunitarize(U0)
    k_ref, Uref, Gref = first_below(ns, nt, U0, tol)
    with gfc.Lattice(ns, nt, mixed=True) as lat:
        lat.upload_links(U0, 8, False)
        ps0, pt0 = lat.plaquette()
        rc, rep = lat.fix(gfc.default_params(tolerance=tol),
                          gfc.options(precision=gfc.PREC_MIXED, stop_rule=gfc.STOP_EVERY, switch_e2=switch,
                                      fp32_refresh=refresh))
        ps1, pt1 = lat.plaquette()
        G = lat.download_gt()
        U = lat.download_links()
        e2, _ = lat.e2_theta()
    assert rc > 0 and 0 < rep.sweeps_fp32 < rc
    assert e2 <= tol and rep.final_residue <= tol
    assert su3_error(G) < 1e-13
    assert abs(ps1 - ps0) < 1e-13 and abs(pt1 - pt0) < 1e-13
    U1 = U0.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(U1, U, atol=1e-12)
    assert rep.functional == pytest.approx(orc.functional(Uref, ns, nt), rel=1e-10)

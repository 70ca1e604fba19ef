"""The batch engine: many lattices, per-timeslice retirement, graph-replayed rounds.

Properties checked (the batch does not round like the reference, and retires each
timeslice on its own e2, so parity is stated through what the result must be):
every lattice ends with e2 below the tolerance, G in SU(3), links equal to
G U0 G^dagger, plaquettes unchanged to 1e-13, the same gauge functional as a
single-lattice fix; and a lattice gives bit-identical results alone or admitted
into a batch that is already running others.
"""
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


def params():
    return gfc.default_params(tolerance=TOL)


def test_device_generator_matches_host():
    ns, nt = 6, 4
    with gfc.Batch(max_sites=10 ** 5, max_slots=2, max_nt=8) as b:
        s = b.add(ns, nt)
        b.synth(s, 81, 0.6)
        b.activate(s, gfc.PREC_FP64_FAST)
        b.finalize(s)                # makes the slot readable; links unchanged (no round ran)
        Ud = b.download_links(s)
    Uh = gfc.synth_config(ns, nt, 81, 0.6)
    orc.reunitarize(Uh)
    np.testing.assert_allclose(Ud, Uh, atol=1e-13)


# launch shapes (minimum resident CTAs per SM of the FP32 and FP64 sweeps): the
# default 128-thread CTAs, and one-warp CTAs that sweep a 128-site work item 32
# sites at a time (the lattices below have 16, 108 and 256 sites per timeslice and
# parity: ragged pieces and items)
SHAPES = [None, (12, 12), (8, 11)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("precision", [gfc.PREC_MIXED, gfc.PREC_FP64_FAST])
def test_uneven_batch_fixes_every_lattice(precision, shape):
    geoms = [(4, 8, 71, 0.4), (6, 6, 72, 0.7), (8, 12, 73, 0.5)]
    U0 = {}
    with gfc.Batch(max_sites=10 ** 6, max_slots=8, max_nt=16) as b:
        if shape:
            b.set_shape(shape[0], shape[1], 8)
        slots = []
        for ns, nt, seed, scale in geoms:
            s = b.add(ns, nt)
            U = gfc.synth_config(ns, nt, seed, scale)
            b.upload(s, U, 8, False)
            orc.reunitarize(U)
            U0[s] = U
            slots.append(s)
        plaq0 = {}
        for s in slots:
            b.activate(s, precision)
        rounds, reps = b.fix_all(params(), gfc.options(precision=precision))
        assert rounds > 0
        for s, (ns, nt, seed, scale) in zip(slots, geoms):
            r = reps[s]
            assert r.status > 0, r.status
            assert r.e2 <= TOL
            G = b.download_gt(s)
            U = b.download_links(s)
            assert su3_error(G) < 1e-13
            U1 = U0[s].copy()
            orc.apply_gt(U1, G, ns, nt)
            np.testing.assert_allclose(U1, U, atol=1e-12)
            for w in (0, 1):
                assert orc.plaquette(U, ns, nt, w) == pytest.approx(orc.plaquette(U0[s], ns, nt, w), abs=1e-13)
            # same Coulomb gauge as a single-lattice FP64 fix
            with gfc.Lattice(ns, nt) as lat:
                lat.upload_links(U0[s], 8, False)
                rc, rep1 = lat.fix(params(), gfc.options(precision=gfc.PREC_FP64_FAST, stop_rule=gfc.STOP_EVERY))
            assert r.functional == pytest.approx(rep1.functional, rel=1e-10)
            sw = b.slice_sweeps(s)
            assert sw.min() > 0 and sw.max() == r.sweeps
        assert b.status() == 0


@pytest.mark.parametrize("shape", [None, (12, 12)])
def test_fp32_rebuilds(shape):
    """options.fp32_refresh in the batch: FP32 timeslices rebuilt from FP64 every 16
    of their own half-sweeps, a later switch; every lattice still ends in the Coulomb
    gauge of a single-lattice FP64 fix, with links G U0 G^dagger."""
    geoms = [(4, 8, 171, 0.4), (6, 6, 172, 0.7), (8, 12, 173, 0.5)]
    o = gfc.options(precision=gfc.PREC_MIXED, switch_e2=1e-10, fp32_refresh=16)
    with gfc.Batch(max_sites=10 ** 6, max_slots=8, max_nt=16) as b:
        if shape:
            b.set_shape(shape[0], shape[1], 8)
        U0, slots = {}, []
        for ns, nt, seed, scale in geoms:
            s = b.add(ns, nt)
            U = gfc.synth_config(ns, nt, seed, scale)
            b.upload(s, U, 8, False)
            orc.reunitarize(U)
            U0[s] = U
            slots.append(s)
            b.activate(s, gfc.PREC_MIXED)
        rounds, reps = b.fix_all(params(), o)
        for s, (ns, nt, seed, scale) in zip(slots, geoms):
            r = reps[s]
            assert r.status > 0 and r.e2 <= TOL
            G, U = b.download_gt(s), b.download_links(s)
            assert su3_error(G) < 1e-13
            U1 = U0[s].copy()
            orc.apply_gt(U1, G, ns, nt)
            np.testing.assert_allclose(U1, U, atol=1e-12)
            with gfc.Lattice(ns, nt) as lat:
                lat.upload_links(U0[s], 8, False)
                rc, rep1 = lat.fix(params(), gfc.options(precision=gfc.PREC_FP64_FAST, stop_rule=gfc.STOP_EVERY))
            assert r.functional == pytest.approx(rep1.functional, rel=1e-10)
            assert b.slice_sweeps(s).max() > 16   # rebuilds ran
        assert b.status() == 0


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("refresh", [0, 16])
def test_same_result_alone_and_in_the_mix(shape, refresh):
    """Continuous batching: a lattice admitted while others are running gets exactly
    the result it gets alone (also with FP32 rebuilds every 16 own half-sweeps)."""
    ns, nt = 6, 8
    U = gfc.synth_config(ns, nt, 91, 0.5)
    other = gfc.synth_config(8, 8, 92, 0.6)
    p = params()
    o = gfc.options(precision=gfc.PREC_MIXED, **({"switch_e2": 1e-10, "fp32_refresh": refresh} if refresh else {}))
    with gfc.Batch(max_sites=10 ** 6, max_slots=4, max_nt=16) as b:
        if shape:
            b.set_shape(shape[0], shape[1], 8)
        s = b.add(ns, nt)
        b.upload(s, U, 8, False)
        b.activate(s, gfc.PREC_MIXED)
        b.fix_all(p, o)
        G_alone = b.download_gt(s)
        sw_alone = b.slice_sweeps(s)
    with gfc.Batch(max_sites=10 ** 6, max_slots=4, max_nt=16) as b:
        if shape:
            b.set_shape(shape[0], shape[1], 8)
        s_other = b.add(8, 8)
        b.upload(s_other, other, 8, False)
        b.activate(s_other, gfc.PREC_MIXED)
        b.round(p, o)
        b.round(p, o)
        s = b.add(ns, nt)
        b.upload(s, U, 8, False)
        b.activate(s, gfc.PREC_MIXED)
        active, rounds = 1, 0
        while active and rounds < 1000:
            active = b.round(p, o)
            rounds += 1
        assert active == 0
        b.finalize(s)
        G_mix = b.download_gt(s)
        assert np.array_equal(b.slice_sweeps(s), sw_alone)
    assert G_mix.tobytes() == G_alone.tobytes()


def test_batch_admission_limits():
    with gfc.Batch(max_sites=5000, max_slots=2, max_nt=8) as b:
        with pytest.raises(gfc.GFCError):
            b.add(0, 4)                  # empty lattice
        with pytest.raises(gfc.GFCError):
            b.add(4, 16)                 # nt above max_nt
        s = b.add(8, 8)                  # 4096 sites
        with pytest.raises(gfc.GFCError):
            b.add(6, 8)                  # 1728 more: over max_sites
        b.remove(s)
        b.add(6, 8)


def test_batch_autotune_then_fix():
    with gfc.Batch(max_sites=10 ** 6, max_slots=4, max_nt=16) as b:
        times = b.autotune(8, 12)
        assert all(t > 0 for v in times.values() for t in v)
        shape = b.shape()
        assert shape["minb32"] in (2, 3, 4, 8, 11, 12) and shape["round_sweeps"] in (4, 8, 16)
        assert shape["minb64"] in (2, 3, 4, 8, 11, 12)
        with pytest.raises(gfc.GFCError):
            s = b.add(6, 8)
            b.upload(s, gfc.synth_config(6, 8, 5, 0.5), 8, False)
            b.activate(s, gfc.PREC_MIXED)
            b.autotune(8, 12)          # refused while a slot is being fixed
        rounds, reps = b.fix_all(params(), gfc.options(precision=gfc.PREC_MIXED))
        assert reps[s].status > 0 and reps[s].e2 <= TOL


@pytest.mark.parametrize("stage", [0, 1])
def test_staging_gives_a_valid_fix(stage):
    ns, nt = 6, 8
    U = gfc.synth_config(ns, nt, 95, 0.6)
    with gfc.Batch(max_sites=10 ** 5, max_slots=2, max_nt=8) as b:
        b.set_staging(stage)
        s = b.add(ns, nt)
        b.upload(s, U, 8, False)
        orc.reunitarize(U)
        b.activate(s, gfc.PREC_FP64_FAST)
        rounds, reps = b.fix_all(params(), gfc.options(precision=gfc.PREC_FP64_FAST))
        assert reps[s].e2 <= TOL
        G = b.download_gt(s)
        Uf = b.download_links(s)
    assert su3_error(G) < 1e-13
    U1 = U.copy()
    orc.apply_gt(U1, G, ns, nt)
    np.testing.assert_allclose(U1, Uf, atol=1e-12)


@pytest.mark.parametrize("elem_bytes,swap", [(4, True), (8, True), (4, False)])
def test_batch_upload_formats_match_single_lattice(elem_bytes, swap):
    """A slot loads file bytes (FP32 or FP64, big or native endian) exactly as the
    single-lattice context does: same links after the reunitarisation of activation."""
    ns, nt = 4, 6
    U = gfc.synth_config(ns, nt, 97, 0.5)
    raw = U.astype((">" if swap else "<") + ("f4" if elem_bytes == 4 else "f8"))
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(raw, elem_bytes, byteswap=swap)
        lat.reunitarize()
        U_single = lat.download_links()
    with gfc.Batch(max_sites=10 ** 4, max_slots=2, max_nt=8) as b:
        s = b.add(ns, nt)
        b.upload(s, raw, elem_bytes, swap)
        b.activate(s, gfc.PREC_FP64_FAST)
        b.finalize(s)                  # no round ran: the links as loaded (and reunitarised)
        U_batch = b.download_links(s)
    np.testing.assert_allclose(U_batch, U_single, atol=1e-14)


def test_held_slot_gives_the_same_result():
    """A slot kept out of some rounds (resident, frozen) ends with the G it gets alone."""
    ns, nt = 6, 6
    U = gfc.synth_config(ns, nt, 98, 0.6)
    p, o = params(), gfc.options(precision=gfc.PREC_MIXED)
    with gfc.Batch(max_sites=10 ** 5, max_slots=2, max_nt=8) as b:
        s = b.add(ns, nt)
        b.upload(s, U, 8, False)
        b.activate(s, gfc.PREC_MIXED)
        b.fix_all(p, o)
        G_alone = b.download_gt(s)
    with gfc.Batch(max_sites=10 ** 5, max_slots=4, max_nt=8) as b:
        other = b.add(4, 8)
        b.upload(other, gfc.synth_config(4, 8, 99, 0.5), 8, False)
        b.activate(other, gfc.PREC_MIXED)
        s = b.add(ns, nt)
        b.upload(s, U, 8, False)
        b.activate(s, gfc.PREC_MIXED)
        for r in range(12):                      # hold it now and then, in FP32 and FP64 phases
            b.hold(s, r % 3 == 1 or 5 <= r <= 7)
            b.round(p, o)
        b.hold(s, False)
        active, rounds = 1, 0
        while active and rounds < 1000:
            active = b.round(p, o)
            rounds += 1
        assert active == 0
        b.finalize(s)
        assert b.download_gt(s).tobytes() == G_alone.tobytes()


@pytest.mark.parametrize("precision", [gfc.PREC_MIXED, gfc.PREC_FP64_FAST])
def test_odd_ns_slots(precision):
    """Lattices of odd ns (3, 5 and 7) beside an even one: each is fixed (e2 below the
    tolerance, G in SU(3), links G U0 G^dagger, plaquettes unchanged) to the oracle's
    gauge functional, and an odd-ns lattice gets the same G alone and in the mix.
    Odd ns runs in FP64 by boundary levels, whatever the precision asked for."""
    geoms = [(3, 4, 141, 0.5), (5, 4, 142, 0.6), (7, 6, 143, 0.4), (6, 4, 144, 0.5)]
    U0 = {}
    with gfc.Batch(max_sites=10 ** 5, max_slots=6, max_nt=8) as b:
        slots = []
        for ns, nt, seed, scale in geoms:
            s = b.add(ns, nt)
            U = gfc.synth_config(ns, nt, seed, scale)
            b.upload(s, U, 8, False)
            orc.reunitarize(U)
            U0[s] = U
            slots.append(s)
        for s in slots:
            b.activate(s, precision)
        rounds, reps = b.fix_all(params(), gfc.options(precision=precision))
        G5_mix = b.download_gt(slots[1])
        for s, (ns, nt, seed, scale) in zip(slots, geoms):
            r = reps[s]
            assert r.status > 0 and r.e2 <= TOL, (ns, nt, r.status, r.e2)
            G = b.download_gt(s)
            U = b.download_links(s)
            assert su3_error(G) < 1e-13
            U1 = U0[s].copy()
            orc.apply_gt(U1, G, ns, nt)
            np.testing.assert_allclose(U1, U, atol=1e-12)
            for w in (0, 1):
                assert orc.plaquette(U, ns, nt, w) == pytest.approx(orc.plaquette(U0[s], ns, nt, w), abs=1e-13)
            # the oracle's gauge functional at its e2 <= tol (reference schedule, deeper)
            Uo, Go = U0[s].copy(), np.zeros(ns ** 3 * nt * 18)
            orc.fix(Uo, Go, ns, nt, tol=TOL)
            assert r.functional == pytest.approx(orc.functional(Uo, ns, nt), rel=1e-10)
        assert b.status() == 0
    with gfc.Batch(max_sites=10 ** 5, max_slots=2, max_nt=8) as b:
        s = b.add(5, 4)
        b.upload(s, gfc.synth_config(5, 4, 142, 0.6), 8, False)
        b.activate(s, precision)
        b.fix_all(params(), gfc.options(precision=precision))
        assert b.download_gt(s).tobytes() == G5_mix.tobytes()

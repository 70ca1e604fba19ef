"""Observables and the on-GPU load/store pipeline (byte swap, FP32 <-> FP64,
reference AoS <-> device layout), checked against the oracle and numpy."""
import numpy as np
import pytest

import gfc
import oracle_ref as orc
from gauge_util import global_rotation_residual

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ns,nt,seed", [(4, 8, 21), (6, 3, 22), (5, 4, 23), (8, 8, 24)])
def test_observables_match_oracle(ns, nt, seed):
    U = gfc.synth_config(ns, nt, seed, 0.6)
    orc.reunitarize(U)
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        e2, th = lat.e2_theta()
        F = lat.functional()
        ps, pt = lat.plaquette()
        sl = lat.e2_slices()
    e2o, slo = orc.e2(U, ns, nt, slices=True)
    assert e2 == pytest.approx(e2o, rel=1e-13)
    assert th == pytest.approx(orc.theta(U, ns, nt), rel=1e-13)
    assert th == pytest.approx(e2 / 6, rel=1e-13)
    assert F == pytest.approx(orc.functional(U, ns, nt), rel=1e-13)
    assert ps == pytest.approx(orc.plaquette(U, ns, nt, 0), rel=1e-13)
    assert pt == pytest.approx(orc.plaquette(U, ns, nt, 1), rel=1e-13)
    np.testing.assert_allclose(sl, slo, rtol=1e-12)


@pytest.mark.parametrize("ns,nt", [(4, 6), (3, 5)])
def test_link_roundtrip_all_formats(ns, nt):
    U = gfc.synth_config(ns, nt, 31, 0.5)
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        assert np.array_equal(lat.download_links(8, False), U)
        assert lat.download_links(8, True).tobytes() == U.astype(">f8").tobytes()
        assert np.array_equal(lat.download_links(4, False), U.astype(np.float32))
        assert lat.download_links(4, True).tobytes() == U.astype(">f4").tobytes()
        lat.upload_links(np.frombuffer(U.astype(">f8").tobytes(), np.uint8), 8, True)
        assert np.array_equal(lat.download_links(8, False), U)
        lat.upload_links(np.frombuffer(U.astype(">f4").tobytes(), np.uint8), 4, True)
        assert np.array_equal(lat.download_links(8, False), U.astype(np.float32).astype(np.float64))
        for site, mu in [(0, 0), (7, 3), (ns ** 3 * nt - 1, 1)]:
            np.testing.assert_array_equal(lat.get_link(site, mu),
                                          U.astype(np.float32).astype(np.float64)[(site * 4 + mu) * 18:][:18])


def test_gt_roundtrip_and_identity():
    ns, nt = 4, 4
    V = ns ** 3 * nt
    G = np.random.default_rng(1).standard_normal(V * 18)
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_gt(G, 8, False)
        assert np.array_equal(lat.download_gt(8, False), G)
        assert lat.download_gt(4, True).tobytes() == G.astype(">f4").tobytes()
        lat.upload_gt(np.frombuffer(G.astype(">f8").tobytes(), np.uint8), 8, True)
        assert np.array_equal(lat.download_gt(), G)
        lat.set_identity_gt()
        I = lat.download_gt().reshape(V, 9, 2)
    assert np.all(I[:, [0, 4, 8], 0] == 1) and np.count_nonzero(I) == 3 * V


def test_reunitarize_matches_oracle_bitwise():
    ns, nt = 4, 4
    U = gfc.synth_config(ns, nt, 41, 0.8)
    U += 1e-6 * np.random.default_rng(2).standard_normal(U.size)   # off the group
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        lat.reunitarize()
        Ug = lat.download_links()
        assert lat.status() == 0
    orc.reunitarize(U)
    assert Ug.tobytes() == U.tobytes()


def test_projection_failure_reported():
    """A null first row cannot be projected (normalize3Vec returns -1); the status
    word reports it like reunitarizeField's -1 (fields.c:144-187)."""
    ns, nt = 2, 2
    U = gfc.synth_config(ns, nt, 42, 0.5)
    U[0:6] = 0.0     # row 0 of the first link
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        lat.reunitarize()
        assert lat.status() & 1
        assert lat.status() == 0     # cleared by the read


def _mats(G):
    M = G.reshape(-1, 9, 2)
    return (M[..., 0] + 1j * M[..., 1]).reshape(-1, 3, 3)


def _a_transformation(ns, nt, seed):
    """An SU(3) field: G after a few half-sweeps of an unconverged fix."""
    U = gfc.synth_config(ns, nt, seed, 0.5)
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        rc, _ = lat.fix(gfc.default_params(max_sweeps_to_fix=7))
        assert rc == gfc.FIX_NOT_CONVERGED
        return lat.download_gt()


def test_apply_gt_matches_oracle_bitwise():
    ns, nt = 4, 6
    U = gfc.synth_config(ns, nt, 131, 0.5)
    orc.reunitarize(U)
    G = _a_transformation(ns, nt, 132)
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(U, 8, False)
        lat.upload_gt(G, 8, False)
        lat.apply_gt()
        Ug = lat.download_links()
    Uo = U.copy()
    orc.apply_gt(Uo, G, ns, nt)
    assert orc.sha(Ug) == orc.sha(Uo)


@pytest.mark.parametrize("precision,stop,refresh", [(gfc.PREC_FP64_EXACT, gfc.STOP_REFERENCE, 0),
                                                    (gfc.PREC_FP64_FAST, gfc.STOP_EVERY, 0),
                                                    (gfc.PREC_MIXED, gfc.STOP_EVERY, 0),
                                                    (gfc.PREC_MIXED, gfc.STOP_EVERY, 16)])
def test_warm_start(precision, stop, refresh):
    """Fixing from a saved transformation G0: the links fixed are G0 U G0^dagger and
    the G returned is the whole transformation (the oracle: applyGaugeTransformationU,
    then the fix, then the product); also with the mixed path's FP32 rebuilds, which
    compose G0 with each piece of the FP32 phase."""
    ns, nt = 4, 8
    U0 = gfc.synth_config(ns, nt, 133, 0.5)
    orc.reunitarize(U0)
    G0 = _a_transformation(ns, nt, 134)
    U1 = U0.copy()
    orc.apply_gt(U1, G0, ns, nt)
    Gf = np.zeros_like(G0)
    rc_o = orc.fix(U1, Gf, ns, nt, tol=1e-15)[0]
    with gfc.Lattice(ns, nt, mixed=precision == gfc.PREC_MIXED) as lat:
        lat.upload_links(U0, 8, False)
        lat.upload_gt(G0, 8, False)
        extra = {"fp32_refresh": refresh, "switch_e2": 1e-10} if refresh else {}
        rc, rep = lat.fix(gfc.default_params(tolerance=1e-15),
                          gfc.options(precision=precision, stop_rule=stop, warm_start=1, **extra))
        G = lat.download_gt()
        U = lat.download_links()
    assert rep.final_residue <= 1e-15
    if refresh:
        assert rep.sweeps_fp32 > refresh   # rebuilds ran
    # the fast paths stop at the first half-sweep below the tolerance (the oracle on
    # the reference schedule later), so their G agrees to what e2 ~ 1e-15 pins down;
    # the FP32 phase of the mixed path also drifts along the residual gauge freedom
    # (a rotation constant on each timeslice), which is removed before comparing
    G_expect = (_mats(Gf) @ _mats(G0)).reshape(-1, 9)
    G_expect = np.stack([G_expect.real, G_expect.imag], -1).reshape(-1)
    if precision == gfc.PREC_MIXED:
        res, drift = global_rotation_residual(G, G_expect, np.arange(ns ** 3 * nt) // ns ** 3)
        print(f"mixed warm start: |G - h(t) G_ref| <= {res:.1e}, |h(t) - 1| <= {drift:.1e}")
        assert res <= 1e-6
    else:
        atol = 1e-12 if precision == gfc.PREC_FP64_EXACT else 1e-6
        np.testing.assert_allclose(_mats(G), _mats(Gf) @ _mats(G0), atol=atol)
    assert rep.functional == pytest.approx(orc.functional(U1, ns, nt), rel=1e-12)
    U2 = U0.copy()
    orc.apply_gt(U2, G, ns, nt)
    np.testing.assert_allclose(U, U2, atol=1e-12)
    if precision == gfc.PREC_FP64_EXACT:
        # the links evolve as in the reference from G0 U G0^dagger, bit for bit
        assert rc == rc_o
        assert orc.sha(U.reshape(-1, 4, 18)[:, 1:4, :]) == orc.sha(U1.reshape(-1, 4, 18)[:, 1:4, :])


@pytest.mark.parametrize("warm", [0, 1])
def test_mixed_needs_a_mixed_context(warm):
    """A context created without GFC_CTX_MIXED has no FP32 fields and no FP64 copy of
    the start: the mixed path is refused with a message, cold or warm."""
    with gfc.Lattice(4, 4) as lat:
        lat.upload_links(gfc.synth_config(4, 4, 135, 0.5), 8, False)
        with pytest.raises(gfc.GFCError, match="GFC_CTX_MIXED"):
            lat.fix(gfc.default_params(), gfc.options(precision=gfc.PREC_MIXED, warm_start=warm))


@pytest.mark.parametrize("elem_bytes,swap", [(8, True), (4, True), (8, False)])
def test_fused_upload_and_reunitarise(elem_bytes, swap):
    """Loading and reunitarising in one pass gives the links of the two separate steps,
    bit for bit."""
    ns, nt = 4, 6
    U = gfc.synth_config(ns, nt, 141, 0.6)
    raw = U.astype((">" if swap else "<") + ("f4" if elem_bytes == 4 else "f8"))
    with gfc.Lattice(ns, nt) as a, gfc.Lattice(ns, nt) as b:
        a.upload_links(raw, elem_bytes, swap)
        a.reunitarize()
        b.upload_links_reunit(raw, elem_bytes, swap)
        assert a.download_links().tobytes() == b.download_links().tobytes()


@pytest.mark.parametrize("elem_bytes,swap", [(8, False), (4, True)])
def test_async_gt_download_matches_the_synchronous_one(elem_bytes, swap):
    """G downloaded with the copy left in flight equals the synchronous download
    bytewise once the context is synchronised; two downloads in a row into two
    buffers, with a fix queued in between, each hold the G of their moment;
    pageable memory is refused."""
    ns, nt = 6, 5
    V = ns ** 3 * nt
    dt = np.float64 if elem_bytes == 8 else np.float32
    with gfc.Lattice(ns, nt) as lat:
        lat.upload_links(gfc.synth_config(ns, nt, 171, 0.5), 8, False)
        lat.set_identity_gt()
        lat.halfsweeps(0, 7, 1.95, 2)
        G1 = lat.download_gt(elem_bytes, swap)
        b1, b2 = gfc.PinnedBuffer(V * 18 * elem_bytes), gfc.PinnedBuffer(V * 18 * elem_bytes)
        lat.download_gt_async(b1.view(dt), elem_bytes, swap)
        lat.halfsweeps(7, 5, 1.95, 2)
        lat.download_gt_async(b2.view(dt), elem_bytes, swap)
        lat.sync()
        G2 = lat.download_gt(elem_bytes, swap)
        assert b1.view(dt).tobytes() == G1.tobytes()
        assert b2.view(dt).tobytes() == G2.tobytes()
        assert G1.tobytes() != G2.tobytes()
        with pytest.raises(gfc.GFCError):
            lat.download_gt_async(np.empty(V * 18, dtype=dt), elem_bytes, swap)
        b1.close()
        b2.close()


def test_device_code_is_sm100a():
    """The kernels the runtime loaded for this library are sm_100 machine code
    compiled from the compute_100 virtual architecture (cudaFuncGetAttributes through
    the C ABI); the library embeds nothing else (its build recipe names
    arch=compute_100a,code=sm_100a only)."""
    binary, ptx = gfc.device_code_version(0)
    assert (binary, ptx) == (100, 100)

"""Observables and the on-GPU load/store pipeline (byte swap, FP32 <-> FP64,
reference AoS <-> device layout), checked against the oracle and numpy."""
import numpy as np
import pytest

import gfc
import oracle_ref as orc

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

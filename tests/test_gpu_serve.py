"""The request server: admission by free capacity, continuous batching, release.

A request's G must be bit-identical to the same lattice fixed alone in a batch,
whatever else the server runs beside it and whenever it was admitted."""
import numpy as np
import pytest

import gfc

pytestmark = pytest.mark.gpu
TOL = 1e-15


def alone(ns, nt, seed, scale, precision, links=None):
    with gfc.Batch(max_sites=10 ** 6, max_slots=2, max_nt=16) as b:
        s = b.add(ns, nt)
        if links is None:
            b.synth(s, seed, scale)
        else:
            b.upload(s, links, 8, False)
        b.activate(s, precision)
        b.fix_all(gfc.default_params(tolerance=TOL), gfc.options(precision=precision))
        return b.download_gt(s)


def run_until_done(srv, ids, p, o, max_steps=5000):
    done = {}
    for _ in range(max_steps):
        srv.step(p, o)
        for rid in ids:
            if rid not in done and srv.poll(rid)[0] == gfc.REQ_DONE:
                done[rid] = srv.fetch(rid)
        if len(done) == len(ids):
            return done
    raise AssertionError("server did not finish")


def test_admission_first_fit_and_release():
    p, o = gfc.default_params(tolerance=TOL), gfc.options(precision=gfc.PREC_MIXED)
    reqs = [(8, 8, 101, 0.5), (8, 8, 102, 0.6), (6, 8, 103, 0.4)]   # 4096, 4096, 1728 sites
    with gfc.Server(max_sites=6000, max_slots=4, max_nt=16) as srv:
        ids = [srv.submit(ns, nt, seed=sd, scale=sc) for ns, nt, sd, sc in reqs]
        running, queued = srv.step(p, o)
        st = [srv.poll(r)[0] for r in ids]
        # the second 8^3x8 does not fit beside the first; the 6^3x8 behind it does
        assert st[1] == gfc.REQ_QUEUED and queued == 1
        assert st[0] in (gfc.REQ_RUNNING, gfc.REQ_DONE) and st[2] in (gfc.REQ_RUNNING, gfc.REQ_DONE)
        out = run_until_done(srv, ids, p, o)
        for rid in ids:
            state, t_admit, t_done, rep = srv.poll(rid)
            assert state == gfc.REQ_FETCHED
            assert 0 <= t_admit <= t_done
            assert rep.status > 0 and rep.e2 <= TOL
        assert srv.poll(ids[1])[1] >= srv.poll(ids[0])[2] - 0.01   # admitted after the first one finished
        with pytest.raises(gfc.GFCError):
            srv.submit(12, 8)                                       # 13824 sites > capacity
    for rid, (ns, nt, sd, sc) in zip(ids, reqs):
        assert out[rid].tobytes() == alone(ns, nt, sd, sc, gfc.PREC_MIXED).tobytes()


def test_uploaded_and_synthetic_requests_mix():
    p = gfc.default_params(tolerance=TOL)
    o = gfc.options(precision=gfc.PREC_FP64_FAST)
    U = gfc.synth_config(6, 6, 111, 0.7)
    with gfc.Server(max_sites=10 ** 5, max_slots=4, max_nt=16) as srv:
        a = srv.submit(6, 6, links=U, precision=gfc.PREC_FP64_FAST)
        b = srv.submit(4, 10, seed=112, scale=0.5, precision=gfc.PREC_FP64_FAST)
        out = run_until_done(srv, [a, b], p, o)
    assert out[a].tobytes() == alone(6, 6, 0, 0, gfc.PREC_FP64_FAST, links=U).tobytes()
    assert out[b].tobytes() == alone(4, 10, 112, 0.5, gfc.PREC_FP64_FAST).tobytes()


def test_smallest_first_policy():
    """With one request sweeping at a time, smallest first: the small request that
    arrived second finishes first; both results are those of the lattice alone."""
    p = gfc.default_params(tolerance=TOL)
    o = gfc.options(precision=gfc.PREC_MIXED)
    with gfc.Server(max_sites=10 ** 5, max_slots=4, max_nt=16) as srv:
        srv.set_policy(gfc.SERVE_SMALLEST_FIRST, 1)
        big = srv.submit(8, 8, seed=121, scale=0.5)
        small = srv.submit(4, 4, seed=122, scale=0.5)
        out = run_until_done(srv, [big, small], p, o)
        t_big, t_small = srv.poll(big)[2], srv.poll(small)[2]
    assert t_small < t_big
    assert out[big].tobytes() == alone(8, 8, 121, 0.5, gfc.PREC_MIXED).tobytes()
    assert out[small].tobytes() == alone(4, 4, 122, 0.5, gfc.PREC_MIXED).tobytes()


def test_larger_requests_admitted_while_others_run():
    """Requests of 16^3x16 and 12^3x12 submitted while a 16^3x8 is being swept, in
    both precisions: each G equals the lattice fixed alone, bit for bit."""
    p = gfc.default_params(tolerance=TOL)
    reqs = [(16, 8, 131, 0.6, gfc.PREC_MIXED), (16, 16, 132, 0.4, gfc.PREC_FP64_FAST),
            (12, 12, 133, 0.7, gfc.PREC_MIXED)]
    with gfc.Server(max_sites=2 * 10 ** 5, max_slots=4, max_nt=16) as srv:
        first = srv.submit(*reqs[0][:2], seed=reqs[0][2], scale=reqs[0][3], precision=reqs[0][4])
        for _ in range(3):
            srv.step(p, gfc.options(precision=gfc.PREC_MIXED))
        later = [srv.submit(ns, nt, seed=sd, scale=sc, precision=pr) for ns, nt, sd, sc, pr in reqs[1:]]
        ids = [first] + later
        out = run_until_done(srv, ids, p, gfc.options(precision=gfc.PREC_MIXED))
        for rid in ids:
            rep = srv.poll(rid)[3]
            assert rep.status > 0 and rep.e2 <= TOL
    for rid, (ns, nt, sd, sc, pr) in zip(ids, reqs):
        assert out[rid].tobytes() == alone(ns, nt, sd, sc, pr).tobytes()


def test_odd_ns_request():
    """A 5^3x4 request beside an 8^3x8 one: fixed in FP64 by boundary levels, the same
    G as the lattice alone in a batch."""
    p = gfc.default_params(tolerance=TOL)
    with gfc.Server(max_sites=10 ** 5, max_slots=4, max_nt=16) as srv:
        a = srv.submit(5, 4, seed=151, scale=0.5)
        b_ = srv.submit(8, 8, seed=152, scale=0.5)
        out = run_until_done(srv, [a, b_], p, gfc.options(precision=gfc.PREC_MIXED))
        assert srv.poll(a)[3].e2 <= TOL
    assert out[a].tobytes() == alone(5, 4, 151, 0.5, gfc.PREC_MIXED).tobytes()
    assert out[b_].tobytes() == alone(8, 8, 152, 0.5, gfc.PREC_MIXED).tobytes()

"""The request loop (cpsb_serve_*) on the GPU.

A mix of DWF solves of differing lattice, Ls, mass, tolerance, right-hand-side
count and inner precision is run once request by request and once submitted
all at once to a server with several slots.  Stated tolerance: each result is
bit-identical alone and in the mix (a request's arithmetic does not depend on
what else runs; the launch shapes the autotuner chose are cached per operator
shape), and every solve meets its FP64 true residual.  Admission under a tight
HBM budget splits requests into single right-hand-side items, never reserves
more than the budget, and gives the single-RHS InvCg result.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAUGES = [((4, 4, 4, 4), 0.2, 301), ((4, 4, 4, 8), 0.2, 302), ((8, 8, 8, 8), 0.15, 303)]
# (gauge, ls, mass, stop_rsd, nrhs, precision)
REQUESTS = [
    (0, 4, 0.05, 1e-10, 1, "F16"),
    (1, 8, 0.01, 1e-8, 2, "F32"),
    (2, 8, 0.1, 1e-12, 3, "F32"),
    (0, 6, 0.003, 1e-10, 2, "F64"),
    (1, 4, 0.02, 1e-10, 1, "F16"),
    (2, 4, 0.05, 1e-10, 4, "F16"),
    (0, 12, 0.01, 1e-12, 1, "F32"),
    (1, 8, 0.05, 1e-8, 3, "F64"),
]


@pytest.fixture(scope="module")
def setup():
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    cb.init(0)
    gauges = [cb.Gauge(fields.random_gauge(d, eps, seed), d) for d, eps, seed in GAUGES]
    reqs = []
    for k, (gi, ls, mass, tol, nrhs, prec) in enumerate(REQUESTS):
        op = cb.DiracOp(gauges[gi], "dwf", mass=mass, ls=ls, m5=1.8)
        n = op.n // 24
        srcs = [fields.random_source(n, 1000 + 17 * k + i) for i in range(nrhs)]
        reqs.append((op, srcs, tol, getattr(cb, prec)))
    return cb, gauges, reqs


def true_rsd(op, x, b):
    ax, _ = op.MatPcDagMatPc(x)
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


def test_alone_equals_mix(setup):
    cb, _, reqs = setup
    alone = []
    srv = cb.Server(slots=1)
    for op, srcs, tol, prec in reqs:
        rid = srv.submit(op, srcs, stop_rsd=tol, precision=prec)
        alone.append(srv.wait(rid))
    srv.close()
    srv = cb.Server(slots=4)
    ids = [srv.submit(op, srcs, stop_rsd=tol, precision=prec) for op, srcs, tol, prec in reqs]
    mix = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2, st          # the mix really overlapped
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (op, srcs, tol, prec), (xa, ra, _), (xm, rm, _) in zip(reqs, alone, mix):
        for i, b in enumerate(srcs):
            assert np.array_equal(xa[i], xm[i])
            assert ra[i].iters == rm[i].iters
            assert rm[i].status == 0 and rm[i].true_rsd <= tol
            assert true_rsd(op, xm[i], b) <= 1.5 * tol


def test_admission_budget_splits_requests(setup):
    cb, _, reqs = setup
    op, srcs, tol, prec = reqs[5]           # 8^4, Ls 4, four right-hand sides, 16-bit inner
    n = op.n // 24
    one_rhs = n * (192 * 6 + 52 * 5 + 96) + (8 << 20)  # footprint of one RHS (serve.cu)
    srv = cb.Server(slots=4, hbm_bytes=one_rhs + (1 << 20))
    rid = srv.submit(op, srcs, stop_rsd=tol, precision=prec)
    xs, rs, _ = srv.wait(rid)
    st = srv.stats()
    srv.close()
    assert st["peak_running"] == 1 and st["peak_reserved_bytes"] <= st["budget_bytes"]
    for i, b in enumerate(srcs):
        x1, r1 = op.InvCg(b, stop_rsd=tol, precision=prec)
        assert np.array_equal(xs[i], x1) and rs[i].iters == r1.iters
        assert true_rsd(op, xs[i], b) <= 1.5 * tol


def test_request_larger_than_budget_is_refused(setup):
    cb, _, reqs = setup
    op, srcs, tol, prec = reqs[0]
    srv = cb.Server(slots=2, hbm_bytes=1 << 20)
    with pytest.raises(cb.CpsbError) as e:
        srv.submit(op, srcs, stop_rsd=tol, precision=prec)
    assert e.value.code == -3
    srv.close()


def test_multishift_requests_overlap_and_match(setup):
    """RHMC-style batch: the multishift solves of several pseudofermions
    submitted at once equal the same solves run one at a time (cpsb_minvcg),
    bit for bit, for the FP64 and the FP32-Krylov-plus-refinement forms."""
    cb, gauges, _ = setup
    from cps_public_b200 import fields
    op = cb.DiracOp(gauges[1], "dwf", mass=0.05, ls=8, m5=1.8)
    shifts = [0.001, 0.01, 0.1, 1.0]
    srcs = [fields.random_source(op.n // 24, 700 + i) for i in range(4)]
    for prec in (cb.F64, cb.F32):
        alone = [op.MInvCG(s, shifts, [1e-10] * 4, precision=prec) for s in srcs]
        srv = cb.Server(slots=4)
        ids = [srv.submit_minvcg(op, s, shifts, [1e-10] * 4, precision=prec) for s in srcs]
        got = [srv.wait_minvcg(i) for i in ids]
        st = srv.stats()
        srv.close()
        assert st["completed"] == 4 and st["peak_running"] >= 2
        for (xa, ra, rsa), (xm, rm, rsm, _) in zip(alone, got):
            assert rm.status == 0 and ra.iters == rm.iters
            np.testing.assert_array_equal(rsa, rsm)
            for k in range(len(shifts)):
                np.testing.assert_array_equal(xa[k], xm[k])


def test_zmobius_request_owns_coefficients(setup):
    """A zMobius request copies its complex b_s, c_s at submission: clearing the
    caller's arrays afterwards does not change the solve, which equals InvCg."""
    cb, gauges, _ = setup
    from cps_public_b200 import fields
    ls = 4
    zb = [1.5 + 0.1j * (s - 1.5) for s in range(ls)]
    zc = [0.5 - 0.05j * s for s in range(ls)]
    op = cb.DiracOp(gauges[0], "zmobius", mass=0.05, ls=ls, m5=1.8, bs=zb, cs=zc)
    src = fields.random_source(op.n // 24, 4242)
    x_ref, r_ref = op.InvCg(src, stop_rsd=1e-10)
    srv = cb.Server(slots=2)
    rid = srv.submit(op, [src], stop_rsd=1e-10, precision=cb.F64)
    op._zb[:] = 0.0
    op._zc[:] = 0.0
    xs, res, _ = srv.wait(rid)
    srv.close()
    assert res[0].status == 0 and res[0].iters == r_ref.iters
    np.testing.assert_array_equal(xs[0], x_ref)


def test_gauge_free_refused_while_requests_are_in_flight():
    """cpsb_gauge_free returns CPSB_ERR_BUSY while a request on the field is
    queued or running (its kernels read the links), and frees it afterwards."""
    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields
    cb.init(0)
    lib = _lib.load()
    dims, ls = (8, 8, 8, 16), 8
    g = cb.Gauge(fields.random_gauge(dims, 0.2, 311), dims)
    op = cb.DiracOp(g, "dwf", mass=0.01, ls=ls, m5=1.8)
    srcs = [fields.random_source(op.n // 24, 312 + i) for i in range(2)]
    srv = cb.Server(slots=1)
    rid = srv.submit(op, srcs, stop_rsd=1e-12, precision=cb.F64)
    assert lib.cpsb_gauge_free(g.h) == -7          # CPSB_ERR_BUSY: the request holds the field
    assert b"request" in lib.cpsb_last_error()
    xs, res, _ = srv.wait(rid)
    srv.close()
    assert all(r.status == 0 for r in res)
    assert lib.cpsb_gauge_free(g.h) == 0
    g.h = None

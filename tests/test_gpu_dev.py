"""The device-pointer entry points (cpsb_*_dev: fields already in HBM, the
caller's stream) against their host-pointer twins through the C ABI, on the
same inputs.  Both pack the same FP64 values with the same kernels, so FP64
results agree to rounding (1e-14 for the operator; the same iteration count and
1e-12 for solves) and mixed-precision solves to 1e-9."""
import ctypes as C

import numpy as np
import pytest

from tests.golden_util import rel

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 4)


def make(action):
    import torch

    import cps_public_b200 as cb
    from cps_public_b200 import fields
    cb.init(0)
    g = cb.Gauge(fields.random_gauge(DIMS, 0.2, 21), DIMS)
    op = cb.DiracOp(g, action, mass=0.1, ls=4)
    stream = torch.cuda.Stream()
    return cb, torch, g, op, stream


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).to("cuda:0")


@pytest.mark.parametrize("action", ["dwf", "mobius"])
def test_mdagm_dev_matches_host(action):
    cb, torch, g, op, stream = make(action)
    from cps_public_b200 import _lib, fields
    x = fields.random_source(op.n // 24, 22)
    x_d = to_dev(torch, x)
    out_d = torch.empty_like(x_d)
    dot = C.c_double()
    torch.cuda.synchronize()
    _lib.check(_lib.load().cpsb_mdagm_dev(g.h, C.byref(op.p), C.c_void_p(out_d.data_ptr()),
                                          C.c_void_p(x_d.data_ptr()), C.byref(dot),
                                          C.c_void_p(stream.cuda_stream)), "cpsb_mdagm_dev")
    out_h, dot_h = op.MatPcDagMatPc(x)
    assert rel(out_d.cpu().numpy(), out_h) < 1e-14
    assert abs(dot.value - dot_h) <= 1e-14 * dot_h


@pytest.mark.parametrize("prec", ["F64", "F16"])
@pytest.mark.parametrize("action", ["dwf", "mobius"])
def test_invcg_dev_and_multi_dev_match_host(action, prec):
    cb, torch, g, op, stream = make(action)
    from cps_public_b200 import _lib, fields
    P = getattr(cb, prec)
    lib = _lib.load()
    srcs = [fields.random_source(op.n // 24, 30 + i) for i in range(3)]
    a = cb.CgArg(1e-10, 5000, P, 0.1, 0)
    # one right-hand side
    b_d = to_dev(torch, srcs[0])
    x_d = torch.zeros_like(b_d)
    r = cb.SolveResult()
    torch.cuda.synchronize()
    rc = lib.cpsb_invcg_dev(g.h, C.byref(op.p), C.byref(a), C.c_void_p(x_d.data_ptr()),
                            C.c_void_p(b_d.data_ptr()), C.byref(r), C.c_void_p(stream.cuda_stream))
    _lib.check(rc, "cpsb_invcg_dev")
    x_h, r_h = op.InvCg(srcs[0], stop_rsd=1e-10, precision=P)
    tol = 1e-12 if P == cb.F64 else 1e-9
    assert r.status == 0 and r.true_rsd <= 1e-10 and r_h.true_rsd <= 1e-10
    assert rel(x_d.cpu().numpy(), x_h) < tol
    if P == cb.F64:
        assert r.iters == r_h.iters
    # three right-hand sides stacked in one device array
    bm_d = to_dev(torch, np.stack(srcs))
    xm_d = torch.zeros_like(bm_d)
    res = (cb.SolveResult * 3)()
    torch.cuda.synchronize()
    rc = lib.cpsb_invcg_multi_dev(g.h, C.byref(op.p), C.byref(a), 3, C.c_void_p(xm_d.data_ptr()),
                                  C.c_void_p(bm_d.data_ptr()), res, C.c_void_p(stream.cuda_stream))
    _lib.check(rc, "cpsb_invcg_multi_dev")
    xs_h, rs_h = op.InvCgMulti(srcs, stop_rsd=1e-10, precision=P)
    xm = xm_d.cpu().numpy()
    for i in range(3):
        assert res[i].true_rsd <= 1e-10
        assert rel(xm[i], xs_h[i]) < tol
        if P == cb.F64:
            assert res[i].iters == rs_h[i].iters


def test_minvcg_dev_matches_host():
    cb, torch, g, op, stream = make("dwf")
    from cps_public_b200 import _lib, fields
    src = fields.random_source(op.n // 24, 40)
    shifts = np.array([1e-3, 0.05, 0.4, 2.0])
    ns = len(shifts)
    b_d = to_dev(torch, src)
    x_d = torch.zeros((ns, op.n), dtype=torch.float64, device="cuda:0")
    xptr = (C.c_void_p * ns)(*[C.c_void_p(x_d[k].data_ptr()) for k in range(ns)])
    rs = np.full(ns, 1e-10)
    al = np.ones(ns)
    a = cb.CgArg(1e-10, 5000, cb.F64, 0.1, 0)
    r = cb.SolveResult()
    torch.cuda.synchronize()
    rc = _lib.load().cpsb_minvcg_dev(g.h, C.byref(op.p), C.byref(a), xptr, C.c_void_p(b_d.data_ptr()),
                                     _lib.ptr(shifts), ns, _lib.ptr(rs), cb.MULTI, _lib.ptr(al), C.byref(r),
                                     C.c_void_p(stream.cuda_stream))
    _lib.check(rc, "cpsb_minvcg_dev")
    xs_h, r_h, rs_h = op.MInvCG(src, list(shifts), [1e-10] * ns)
    assert r.iters == r_h.iters
    xs = x_d.cpu().numpy()
    for k in range(ns):
        assert rel(xs[k], xs_h[k]) < 1e-12
    np.testing.assert_allclose(rs, rs_h, rtol=1e-6)

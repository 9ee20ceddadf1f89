"""Edge cases of the solver entry points, as CPS defines them: a zero source
is solved by x = 0 (CPS divides by |src|^2; inv_cg.C returns at once), a solve
cut off by max_num_iter reports CPSB_NOT_CONVERGED with its FP64 true residual
(CPS only warns, inv_cg.C:392-396), bad arguments are refused with
CPSB_ERR_ARG, and the initial guess is honoured (a converged guess takes one
iteration, CPS's itr+1 count)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def op():
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    cb.init(0)
    dims = (4, 4, 4, 8)
    g = cb.Gauge(fields.random_gauge(dims, 0.2, 55), dims)
    return cb, cb.DiracOp(g, "dwf", mass=0.05, ls=4)


@pytest.mark.parametrize("prec", ["F64", "F32", "F16"])
def test_zero_source(op, prec):
    cb, o = op
    x, r = o.InvCg(np.zeros(o.n), precision=getattr(cb, prec))
    assert r.status == 0 and not np.any(x)


@pytest.mark.parametrize("prec", ["F64", "F32", "F16"])
def test_max_iterations_reported(op, prec):
    cb, o = op
    from cps_public_b200 import fields
    b = fields.random_source(o.n // 24, 56)
    x, r = o.InvCg(b, stop_rsd=1e-12, max_num_iter=4, precision=getattr(cb, prec))
    assert r.status == 1 and r.rc == 1
    ax, _ = o.MatPcDagMatPc(x)
    true = np.linalg.norm(b - ax) / np.linalg.norm(b)
    assert abs(r.true_rsd - true) < 1e-6 * max(true, 1e-30) + 1e-12


def test_converged_guess_takes_one_iteration(op):
    cb, o = op
    from cps_public_b200 import fields
    b = fields.random_source(o.n // 24, 57)
    # The first solve stops on the iterated residual, so its true residual may
    # end a little above its target: solve it ten times tighter.
    x, r = o.InvCg(b, stop_rsd=1e-11)
    assert r.true_rsd <= 1e-10
    x2, r2 = o.InvCg(b, stop_rsd=1e-10, guess=x)
    assert r2.iters == 1 and r2.true_rsd <= 1e-10


def test_bad_arguments_refused(op):
    cb, o = op
    from cps_public_b200 import _lib
    import ctypes as C
    p = cb.DiracParams.from_buffer_copy(o.p)
    p.ls = 1  # DWF needs ls >= 2
    out = np.zeros(o.n)
    rc = _lib.load().cpsb_mdagm(o.gauge.h, C.byref(p), _lib.ptr(out), _lib.ptr(np.zeros(o.n)), None)
    assert rc == -1
    a = cb.CgArg(-1.0, 10, 0, 0.1, 0)  # negative stop_rsd
    res = cb.SolveResult()
    rc = _lib.load().cpsb_invcg(o.gauge.h, C.byref(o.p), C.byref(a), _lib.ptr(out), _lib.ptr(np.ones(o.n)),
                                C.byref(res))
    assert rc == -1

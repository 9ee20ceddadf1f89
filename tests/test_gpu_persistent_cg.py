"""The persistent FP64 CG loop (one cooperative kernel runs every iteration of a
small-lattice solve) against the launch-per-step loop of the same recurrence.

Both run DiracOp::InvCg's recurrence (inv_cg.C:293-364); they differ only in
the number of blocks whose partial sums make up each dot product, so their
iteration counts agree within one and their solutions within 1e-9 relative
(the bound the FP64 solver keeps against CPS itself).  CPSB_PERSISTENT_CG
selects the loop: 0 launch-per-step, 1 (default) persistent for Wilson fields
of at most 2^14 entries, 2 persistent for any action and size.  Fields of at
most 2^14 entries run eight lanes per entry with the direction update folded
into the next iteration's hops; larger ones one thread per entry with a
separate direction-update phase.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests.golden_util import load, rel

pytestmark = pytest.mark.gpu


def _launches(lib):
    n = C.c_ulonglong(0)
    assert lib.cpsb_kernel_launches(C.byref(n)) == 0
    return n.value


def _solve(op, srcs, mode):
    old = os.environ.get("CPSB_PERSISTENT_CG")
    os.environ["CPSB_PERSISTENT_CG"] = str(mode)
    try:
        from cps_public_b200 import _lib
        lib = _lib.load()
        n0 = _launches(lib)
        xs, rs = op.InvCgMulti(srcs, stop_rsd=1e-10, max_num_iter=5000)
        return xs, rs, _launches(lib) - n0
    finally:
        if old is None:
            del os.environ["CPSB_PERSISTENT_CG"]
        else:
            os.environ["CPSB_PERSISTENT_CG"] = old


def _compare(op, srcs, mode=1):
    xa, ra, na = _solve(op, srcs, 0)
    xb, rb, nb = _solve(op, srcs, mode)
    for q, (x0, r0, x1, r1) in enumerate(zip(xa, ra, xb, rb)):
        assert r1.status == 0 and r1.true_rsd <= 1e-10, (q, r1.as_dict())
        assert abs(r1.iters - r0.iters) <= 1, (q, r0.iters, r1.iters)
        if np.linalg.norm(x0) == 0:
            assert np.linalg.norm(x1) == 0
        else:
            assert rel(x1, x0) < 1e-9, (q, rel(x1, x0))
    # the whole iteration loop is one launch: the set-up and the true residuals
    # are a handful of kernels per right-hand side, against several per
    # iteration step by step
    assert nb <= 16 + 4 * len(srcs) and 10 * nb < na, (na, nb)
    return ra, rb


def test_persistent_wilson_8x8x8x8_config_case():
    """The reference's CPU-runnable case (Wilson 8^4, mass 0.1, 1e-10): the
    persistent loop matches CPS's iteration count and solution as well."""
    import cps_public_b200 as cb
    rec, u, src = load("wilson_8x8x8x8_cg")
    cb.init(0)
    g = cb.Gauge(u, (8, 8, 8, 8))
    op = cb.DiracOp(g, "wilson", mass=0.1)
    _compare(op, [src])
    xs, rs, _ = _solve(op, [src], 1)
    assert abs(rs[0].iters - int(rec["cg_iters"])) <= 1
    assert rel(xs[0], rec["cg_sol"]) < 1e-9


def test_persistent_dwf_multi_rhs_with_zero_source():
    """DWF 4^3 x 8 x Ls 8, four right-hand sides of different difficulty (one a
    zero source, halted before the first iteration); right-hand sides halt at
    different iterations inside the one launch."""
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    cb.init(0)
    dims, ls = (4, 4, 4, 8), 8
    g = cb.Gauge(fields.random_gauge(dims, 0.2, 71), dims)
    n = int(np.prod(dims)) // 2 * ls
    srcs = [fields.random_source(n, 72), np.zeros(n * 24), fields.random_source(n, 73) * 1e-3,
            fields.random_source(n, 74)]
    for mass in (0.05, 0.3):
        op = cb.DiracOp(g, "dwf", mass=mass, ls=ls)
        ra, rb = _compare(op, srcs, mode=2)  # the direction-parallel form with the 5th-direction hop
        assert rb[1].iters == ra[1].iters


def test_persistent_forced_at_larger_size():
    """Mode 2 on DWF 8^4 x Ls 16 with 8 right-hand sides (262144 entries, above
    the automatic limit): the one-thread-per-entry form, blocks striding over
    several work units per phase."""
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    cb.init(0)
    dims, ls = (8, 8, 8, 8), 16
    g = cb.Gauge(fields.random_gauge(dims, 0.2, 81), dims)
    op = cb.DiracOp(g, "dwf", mass=0.1, ls=ls)
    n = int(np.prod(dims)) // 2 * ls
    srcs = [fields.random_source(n, 82 + q) for q in range(8)]
    _compare(op, srcs, mode=2)

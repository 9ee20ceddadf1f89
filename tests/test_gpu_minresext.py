"""DiracOp::MinResExt on the device (cpsb_minresext) against the compiled
reference's fixtures.  The device sums dot products in a different order than
CPS's sequential loops, so agreement is to 1e-11 relative (the Gram-Schmidt
and the small elimination amplify rounding by the conditioning of the previous
solutions).  Property: when phi = A (v0 + 0.5 v1), the guess reproduces that
combination and its residual vanishes."""
import os

import numpy as np
import pytest

from tests.golden_util import rel, sha

pytestmark = pytest.mark.gpu

CASES = [("wilson_4x4x4x4", "wilson"), ("dwf_4x4x4x4_ls4", "dwf"), ("mobius_4x4x4x4_ls4", "mobius")]
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def device_op(rec, u, action):
    import cps_public_b200 as cb
    cb.init(0)
    g = cb.Gauge(u, tuple(int(d) for d in rec["dims"]))
    kw = dict(mass=float(rec["mass"]), ls=int(rec["ls"]))
    for k in ("m5", "b", "c"):
        if k in rec:
            kw[k] = float(rec[k])
    return cb.DiracOp(g, action, **kw)


@pytest.mark.parametrize("name,action", CASES)
def test_minresext_vs_reference(name, action):
    from cps_public_b200 import fields
    from tests.golden.make_golden import minresext_inputs
    rec = dict(np.load(os.path.join(GOLDEN, f"minresext_{name}.npz")))
    u = fields.random_gauge(tuple(int(d) for d in rec["dims"]), float(rec["eps"]), int(rec["seed"]))
    assert sha(u) == str(rec["gauge_sha"])
    op = device_op(rec, u, action)
    phi, prev = minresext_inputs(rec)
    psi, v, vm, res = op.MinResExt(phi, prev)
    assert rel(psi, rec["psi"]) < 1e-11
    for i in range(len(v)):
        assert abs(np.linalg.norm(v[i]) - 1.0) < 1e-13


@pytest.mark.parametrize("name,action", CASES)
def test_minresext_recovers_exact_combination(name, action):
    from cps_public_b200 import fields
    rec = dict(np.load(os.path.join(GOLDEN, f"minresext_{name}.npz")))
    u = fields.random_gauge(tuple(int(d) for d in rec["dims"]), float(rec["eps"]), int(rec["seed"]))
    op = device_op(rec, u, action)
    n = op.n // 24
    x0, x1, x2 = (fields.random_source(n, 900 + i) for i in range(3))
    target = x0 + 0.5 * x1
    phi, _ = op.MatPcDagMatPc(target)
    psi, _, _, res = op.MinResExt(phi, [x0, x1, x2])
    assert res < 1e-10
    assert rel(psi, target) < 1e-8

"""The drop-in, run from CPS: CPS's own Lattice entry points with the B200 bridge linked in.

oracle/_ref/cpsref_b200 is CPS built as INTEGRATION.md tells a maintainer to
(oracle/build_dropin.py: the bridge source, and f_dwf_base.C / f_mobius.C /
f_wilson.C with the USE_B200 branches inserted, compiled with -DUSE_B200 and
linked with libcpsb200.so).  oracle/_ref/cpsref is the same CPS without them.
Both run the same harness request -- GwilsonFdwf / GwilsonFmobius /
GwilsonFwilson with the fields of the golden fixtures -- through
Lattice::FmatEvlInv, Lattice::FmatEvlMInv and Lattice::FmatInv, and the
results are compared:

* with the bridge's inner precision set to FP64: iteration counts within 1
  and solutions within 1e-9 relative of the CPU run (the bound the other
  FP64 parity tests use), the reported true residuals below the tolerance
  (MInvCG's per-shift iterated residuals within 2%: a shift that freezes one
  iteration apart reports the next iterate's residual);
* with the bridge's defaults (16-bit inner CG for FmatEvlInv / FmatInv, FP32
  Krylov vectors for FmatEvlMInv): every FP64 true residual below the
  tolerance and the solutions within 3e-8 of the CPU run (the spread a 1e-10
  residual leaves on these lattices);
* the B200 run launched the library's kernels (its harness reports the
  count), so the solve did go through the bridge.
"""
import numpy as np
import pytest

from tests.golden_util import load, rel

pytestmark = pytest.mark.gpu

CASES = [("wilson_4x4x4x4", "wilson"), ("dwf_4x4x4x4_ls4", "dwf"), ("mobius_4x4x4x4_ls4", "mobius"),
         ("cg_dwf_8x8x8x8_ls16", "dwf")]
F64, F32, F16 = 0, 1, 2


def _inputs(name, action):
    from oracle import refrun
    if not (refrun.available() and refrun.available(refrun.CPSREF_B200)):
        pytest.skip("compiled reference builds not present (oracle/build_ref.sh, oracle/build_dropin.py)")
    rec, u, src = load(name)
    dims = tuple(int(d) for d in rec["dims"])
    kw = dict(ls=int(rec.get("ls", 1)), mass=float(rec["mass"]))
    for k in ("m5", "b", "c"):
        if k in rec:
            kw[k] = float(rec[k])
    return refrun, dims, u, src, kw


@pytest.mark.parametrize("name,action", CASES)
def test_fmat_evl_inv_from_cps(name, action):
    refrun, dims, u, src, kw = _inputs(name, action)
    z = np.zeros_like(src)
    it_c, rp_c, x_c = refrun.run(refrun.OP_FMATEVLINV, action, dims, u, [src, z], **kw)
    it_b, rp_b, x_b = refrun.run(refrun.OP_FMATEVLINV, action, dims, u, [src, z], **kw,
                                 binary=refrun.CPSREF_B200, bridge_prec=(F64, F32))
    assert rp_b[44] > 0, "the B200 build launched no kernels"
    assert rp_c[44] == 0
    assert abs(it_b - it_c) <= 1, (it_b, it_c)
    assert rel(x_b, x_c) < 1e-9
    assert rp_b[0] <= 1e-10 and rp_c[0] <= 1e-10
    it_h, rp_h, x_h = refrun.run(refrun.OP_FMATEVLINV, action, dims, u, [src, z], **kw,
                                 binary=refrun.CPSREF_B200)
    assert rp_h[44] > 0
    assert rp_h[0] <= 1e-10, rp_h[0]
    assert rel(x_h, x_c) < 3e-8


@pytest.mark.parametrize("name,action", CASES[:3])
def test_fmat_evl_minv_from_cps(name, action):
    refrun, dims, u, src, kw = _inputs(name, action)
    shifts = [0.0, 0.01, 0.1, 0.5]
    rsd, alpha = np.full(4, 1e-10), np.ones(4)
    it_c, rp_c, x_c = refrun.run(refrun.OP_MINVCG, action, dims, u, [src], **kw, shifts=shifts, extra=[rsd, alpha])
    for prec, tol in ((F64, 1e-9), (F32, 1e-7)):
        it_b, rp_b, x_b = refrun.run(refrun.OP_MINVCG, action, dims, u, [src], **kw, shifts=shifts,
                                     extra=[rsd, alpha], binary=refrun.CPSREF_B200, bridge_prec=(F16, prec))
        assert rp_b[44] > 0, "the B200 build launched no kernels"
        if prec == F64:
            assert abs(it_b - it_c) <= 1, (it_b, it_c)
            # each shift reports its iterated residual at the iteration it froze;
            # reductions summed in another order can move that iteration by one
            np.testing.assert_allclose(rp_b[:4], rp_c[:4], rtol=2e-2)
        else:
            assert np.all(rp_b[:4] <= 1e-10 * 1.01), rp_b[:4]
        n = len(src)
        for s in range(4):
            assert rel(x_b[s * n:(s + 1) * n], x_c[s * n:(s + 1) * n]) < tol, (prec, s)


@pytest.mark.parametrize("name,action", CASES[:3])
def test_fmat_inv_from_cps(name, action):
    from cps_public_b200 import fields
    refrun, dims, u, src, kw = _inputs(name, action)
    full = fields.random_source(2 * len(src) // 24, 91)
    guess = np.zeros_like(full)
    it_c, rp_c, x_c = refrun.run(refrun.OP_FMATINV, action, dims, u, [full, guess], **kw)
    it_b, rp_b, x_b = refrun.run(refrun.OP_FMATINV, action, dims, u, [full, guess], **kw,
                                 binary=refrun.CPSREF_B200, bridge_prec=(F64, F32))
    assert rp_b[44] > 0, "the B200 build launched no kernels"
    assert abs(it_b - it_c) <= 1, (it_b, it_c)
    assert rel(x_b, x_c) < 1e-9
    it_h, rp_h, x_h = refrun.run(refrun.OP_FMATINV, action, dims, u, [full, guess], **kw,
                                 binary=refrun.CPSREF_B200)
    assert rp_h[44] > 0
    assert rel(x_h, x_c) < 3e-8

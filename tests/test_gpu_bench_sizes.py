"""Parity at the benchmark's own sizes, through the C ABI, against the C oracle.

Every other parity test runs at 8^4 x Ls 16 or smaller; these run the
operators on the lattices the performance numbers are quoted on, where index
arithmetic and the launch shapes chosen by the autotuner differ:

* DWF 16^3x32, Ls 16, m_f 0.01, M5 1.8 with the benchmark's own fields (links
  reunitarise(exp(i 0.2 H)) seed 2024, Gaussian sources seeds 2025...): the
  FP64 Dslash for both checkerboards and daggers and MatPcDagMatPc with its
  fused |MatPc in|^2, to 1e-13 relative (the dot, a sum of 2.5e7 squares in a
  different order than CPS's, to 1e-12); the FP32 and 16-bit Dslash on 12
  right-hand sides in one launch (the multi-RHS hop of the headline solve),
  each right-hand side to 2e-6 (FP32) and 5e-4 (16-bit) relative;
* Mobius SYM2, 24^3x64, Ls 16, b 1.5, c 0.5, m_f 0.005 (links with eps 0.15):
  MatPcDagMatPc on a 12-right-hand-side FP64 field (85 M sites, 2.0e9 reals,
  16 GB: byte offsets past 2^32), right-hand sides 0 and 11 checked against the
  oracle to 1e-13, their dots to 1e-12.

The oracle evaluations run concurrently in threads (its ctypes calls release
the interpreter lock and allocate their own scratch).
"""
import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (16, 16, 16, 32)
LS = 16
MF = 0.01
M5 = 1.8
NRHS = 12
TOL_HOP = {1: 2e-6, 2: 5e-4}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def dwf():
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    from oracle import oracle
    cb.init(0)
    u = fields.random_gauge(DIMS, 0.2, 2024)              # bench.py's links
    n5 = int(np.prod(DIMS)) // 2 * LS
    srcs = [fields.random_source(n5, 2025 + i) for i in range(NRHS)]   # bench.py's sources
    g = cb.Gauge(u, DIMS)
    op = cb.DiracOp(g, "dwf", mass=MF, ls=LS, m5=M5)
    ref = oracle.Op("dwf", DIMS, u, ls=LS, mass=MF, m5=M5)
    yield cb, g, op, ref, srcs
    g.free()


def test_dwf_bench_lattice_fp64_dslash_and_mdagm(dwf):
    cb, g, op, ref, srcs = dwf
    src = srcs[0]
    jobs = [(cb_, dag) for cb_ in (0, 1) for dag in (0, 1)]
    with ThreadPoolExecutor(max_workers=5) as ex:
        fut = {j: ex.submit(ref.dslash, src, *j) for j in jobs}
        fmd = ex.submit(ref.mdagm, src)
        got = {j: op.Dslash(src, *j) for j in jobs}
        out, dot = op.MatPcDagMatPc(src)
        for j in jobs:
            err = _rel(got[j], fut[j].result())
            assert err < 1e-13, (j, err)
        rout, rdot = fmd.result()
    assert _rel(out, rout) < 1e-13
    # the fused |MatPc in|^2 sums 2.5e7 squares in another order than CPS: 1e-12
    assert abs(dot - rdot) <= 1e-12 * abs(rdot)
    # and against the compiled reference's own outputs at this size (digest fixture)
    import os

    from tests.golden.make_golden import solution_digest
    from tests.golden_util import GOLDEN
    rec = dict(np.load(os.path.join(GOLDEN, "bench_dwf_16x16x16x32_ls16.npz")))
    assert int(rec["src_seed"]) == 2025 and int(rec["seed"]) == 2024
    nsites = op.n // 24
    for got_v, key in ((got[(1, 0)], "dslash_digest"), (out, "mdagm_digest")):
        dg, rd = solution_digest(got_v, nsites), rec[key]
        scale = np.linalg.norm(got_v) * np.sqrt(nsites * 24)   # |x| |v| of the seeded digest vectors
        assert abs(dg[0] - rd[0]) <= 1e-13 * rd[0]
        assert np.all(np.abs(dg[1:] - rd[1:]) <= 1e-13 * scale), (key, dg, rd)
    assert abs(dot - float(rec["mdagm_dot"])) <= 1e-12 * abs(rdot)


@pytest.mark.parametrize("prec", [1, 2], ids=["f32", "f16"])
def test_dwf_bench_lattice_multi_rhs_hop(dwf, prec):
    import torch
    from cps_public_b200 import _lib
    cb, g, op, ref, srcs = dwf
    lib = _lib.load()
    n = op.n
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.concatenate(srcs)).to(dev)
    y = torch.empty_like(x)
    with ThreadPoolExecutor(max_workers=NRHS) as ex:
        fut = [ex.submit(ref.dslash, s, 1, 0) for s in srcs]
        rc = lib.cpsb_dslash_multi_dev(g.h, C.byref(op.p), prec, NRHS, C.c_void_p(y.data_ptr()),
                                       C.c_void_p(x.data_ptr()), 1, 0, None)
        assert rc == 0
        got = y.cpu().numpy().reshape(NRHS, n)
        errs = [_rel(got[q], fut[q].result()) for q in range(NRHS)]
    assert max(errs) < TOL_HOP[prec], errs


def test_mobius_config2_lattice_twelve_rhs_mdagm():
    import torch

    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields
    from oracle import oracle
    cb.init(0)
    lib = _lib.load()
    dims, ls, mf = (24, 24, 24, 64), 16, 0.005
    u = fields.random_gauge(dims, 0.15, 2026)
    n5 = int(np.prod(dims)) // 2 * ls
    n = n5 * 24
    s0, s11 = fields.random_source(n5, 2027), fields.random_source(n5, 2028)
    ref = oracle.Op("mobius", dims, u, ls=ls, mass=mf, m5=M5, b=1.5, c=0.5, pc_type=2)
    g = cb.Gauge(u, dims)
    op = cb.DiracOp(g, "mobius", mass=mf, ls=ls, m5=M5, b=1.5, c=0.5, pc_type=2)
    assert op.n == n and NRHS * n * 8 > 2**32   # byte offsets of the field pass 2^32
    dev = torch.device("cuda", 0)
    with ThreadPoolExecutor(max_workers=2) as ex:
        f0, f11 = ex.submit(ref.mdagm, s0), ex.submit(ref.mdagm, s11)
        x = torch.zeros(NRHS * n, dtype=torch.float64, device=dev)
        x[:n].copy_(torch.from_numpy(s0))
        x[11 * n:].copy_(torch.from_numpy(s11))
        y = torch.empty_like(x)
        dots = (C.c_double * NRHS)()
        rc = lib.cpsb_mdagm_multi_dev(g.h, C.byref(op.p), 0, NRHS, C.c_void_p(y.data_ptr()),
                                      C.c_void_p(x.data_ptr()), dots, None)
        assert rc == 0
        del x
        got0 = y[:n].cpu().numpy()
        got11 = y[11 * n:].cpu().numpy()
        assert float(torch.count_nonzero(y[n:11 * n])) == 0.0   # zero right-hand sides stay zero
        del y
        (r0, d0), (r11, d11) = f0.result(), f11.result()
    g.free()
    assert _rel(got0, r0) < 1e-13
    assert _rel(got11, r11) < 1e-13
    assert abs(dots[0] - d0) <= 1e-12 * d0 and abs(dots[11] - d11) <= 1e-12 * d11   # 1.7e8-term sums
    assert all(dots[q] == 0.0 for q in range(1, 11))

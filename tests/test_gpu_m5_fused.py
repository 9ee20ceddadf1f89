"""The Mobius hop with the M5 sweeps fused into its epilogue (hop_m5.cuh).

Mobius SYM2 MatPc runs M5^-1 after its first hop and MatPcDag runs M5^-dag
after both of its hops (zmobius_m-sym2.h, zmobius_mdag-sym2.h); the operator
fuses each such pair into one kernel.  Checked here, through the C ABI, for
every Ls the kernels support, on a 4x4x4x6 antiperiodic lattice (192
checkerboard sites: the tiles of Ls 20, 24 and 32 -- 6, 5 and 4 columns --
end inside the lattice):

* FP64 MatPc, MatPcDag and MatPcDagMatPc with the fused norm against the C
  oracle to 1e-13 relative, and against the two-kernel form (fusion switched
  off with CPSB_M5_FUSE=0) to 1e-14;
* FP32 and 16-bit MatPcDagMatPc against the oracle to 4 x (2e-6, 5e-4), the
  per-hop tolerances of the other reduced-precision tests over the four hops;
* 12 right-hand sides in one launch at 8x8x4x6, Ls 16, FP32 and 16-bit, with
  the launch shape of the unfused hops pinned (CPSB_TUNE_FORCE): each
  right-hand side bit-identical to the same operator on that right-hand side
  alone, its |M x|^2 to 1e-12 (the grid, and so the order of the partial sums,
  depends on the number of right-hand sides), and a right-hand side of zeros
  stays zero.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {1: 2e-6, 2: 5e-4}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("ls", [4, 8, 12, 16, 20, 24, 32])
def test_fused_mobius_operator_matches_oracle_and_unfused(ls, monkeypatch):
    import cps_public_b200 as cb
    from cps_public_b200 import fields
    from oracle import oracle
    cb.init(0)
    dims = (4, 4, 4, 6)
    u = fields.random_gauge(dims, 0.25, 7)
    n5 = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(n5, 8)
    kw = dict(mass=0.05, ls=ls, m5=1.8, b=1.5, c=0.5, pc_type=2)
    ref = oracle.Op("mobius", dims, u, bc_t=1, **kw)
    g = cb.Gauge(u, dims, bc_t=1)
    got = {}
    for fuse in ("1", "0"):
        monkeypatch.setenv("CPSB_M5_FUSE", fuse)
        op = cb.DiracOp(g, "mobius", **kw)
        got[fuse] = (op.MatPc(src), op.MatPcDag(src), op.MatPcDagMatPc(src), op.MatPcDagMatPcPrec(src, 1),
                     op.MatPcDagMatPcPrec(src, 2))
    g.free()
    m, md, (mm, dot), (m32, d32), (m16, d16) = got["1"]
    rm, rmd = ref.matpc(src, 0), ref.matpc(src, 1)
    rmm, rdot = ref.mdagm(src)
    assert _rel(m, rm) < 1e-13 and _rel(md, rmd) < 1e-13 and _rel(mm, rmm) < 1e-13
    assert abs(dot - rdot) <= 1e-13 * rdot
    u_m, u_md, (u_mm, u_dot) = got["0"][:3]
    assert _rel(m, u_m) < 1e-14 and _rel(md, u_md) < 1e-14 and _rel(mm, u_mm) < 1e-14
    assert abs(dot - u_dot) <= 1e-14 * u_dot
    assert _rel(m32, rmm) < 4 * TOL[1] and abs(d32 - rdot) < 4 * TOL[1] * rdot
    assert _rel(m16, rmm) < 4 * TOL[2] and abs(d16 - rdot) < 4 * TOL[2] * rdot


def _multi_child(prec):
    import json
    import torch
    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields
    cb.init(0)
    lib = _lib.load()
    dims, ls, nrhs = (8, 8, 4, 6), 16, 12
    u = fields.random_gauge(dims, 0.25, 17)
    n5 = int(np.prod(dims)) // 2 * ls
    n = n5 * 24
    g = cb.Gauge(u, dims, bc_t=1)
    op = cb.DiracOp(g, "mobius", mass=0.02, ls=ls, m5=1.8, b=1.5, c=0.5, pc_type=2)
    dev = torch.device("cuda", 0)
    srcs = [fields.random_source(n5, 100 + q) for q in range(nrhs)]
    srcs[5] = np.zeros(n)
    x = torch.from_numpy(np.concatenate(srcs)).to(dev)
    y = torch.empty_like(x)
    dots = (C.c_double * nrhs)()
    rc = lib.cpsb_mdagm_multi_dev(g.h, C.byref(op.p), prec, nrhs, C.c_void_p(y.data_ptr()),
                                  C.c_void_p(x.data_ptr()), dots, None)
    torch.cuda.synchronize()
    multi = y.cpu().numpy().reshape(nrhs, n)
    res = {"rc": rc, "zero": bool(not multi[5].any() and dots[5] == 0.0), "same": [], "dot": []}
    for q in (0, 11):
        one, d1 = op.MatPcDagMatPcPrec(srcs[q], prec)
        res["same"].append(bool(np.array_equal(multi[q], one)))
        res["dot"].append(abs(dots[q] - d1) / d1)
    g.free()
    print(json.dumps(res))


@pytest.mark.parametrize("prec", [1, 2])
def test_fused_mobius_multi_rhs_equals_single(prec):
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CPSB_TUNE_FORCE="0")   # the same launch shape for 1 and 12 right-hand sides
    p = subprocess.run([sys.executable, "-c", f"import tests.test_gpu_m5_fused as t; t._multi_child({prec})"],
                       cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    assert res["rc"] == 0 and res["zero"], res
    assert all(res["same"]), res
    assert all(d <= 1e-12 for d in res["dot"]), res

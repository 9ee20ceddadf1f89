"""The allocation-free entry point cpsb_redot_noalloc against the existing one.

Some callers cannot allocate device memory -- a solver or HMC loop that runs
inside an HBM arena it reserved up front and may not grow, or code that must
not synchronise the device through cudaFree -- so the library offers one
reduction whose scratch is a static device array.  These tests compute
|MatPc in|^2 with it and compare with the |MatPc in|^2 that cpsb_mdagm reports,
twice in a row (the second call reuses the scratch the first one left
behind).  They run last (file name) and work alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_dots(lib, x, n, nvec, res):
    import torch
    res.zero_()
    rc = lib.cpsb_redot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), n, nvec,
                                C.c_void_p(res.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0
    return res.cpu().numpy()


def test_redot_noalloc_matches_mdagm_dot():
    import torch

    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields

    cb.init(0)
    lib = _lib.load()
    dims, ls = (4, 4, 4, 8), 8
    u = fields.random_gauge(dims, 0.2, 41)
    src = fields.random_source(int(np.prod(dims)) // 2 * ls, 42)
    g = cb.Gauge(u, dims)
    op = cb.DiracOp(g, "dwf", mass=0.05, ls=ls)
    _, dot_ref = op.MatPcDagMatPc(src)          # existing entry point: |MatPc src|^2
    mv = op.MatPc(src)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.concatenate([mv, src])).to(dev)
    res = torch.zeros(2, dtype=torch.float64, device=dev)
    n = mv.size
    for _ in range(2):
        got = _noalloc_dots(lib, x, n, 2, res)
        assert abs(got[0] - dot_ref) <= 1e-13 * dot_ref
        assert abs(got[1] - float(np.dot(src, src))) <= 1e-13 * float(np.dot(src, src))
    assert lib.cpsb_redot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), n, 17,
                                  C.c_void_p(res.data_ptr()), None) == -1


def test_redot_noalloc_sixteen_long_vectors():
    """nvec = 16 (the limit) with n = 393216 doubles per vector, more than the
    592 blocks x 256 threads of one pass, so every block strides over the
    vector and all 16 x 592 partial slots of the scratch are used."""
    import torch

    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields

    cb.init(0)
    lib = _lib.load()
    dims, ls, nvec = (8, 8, 8, 8), 8, 16
    u = fields.random_gauge(dims, 0.2, 43)
    g = cb.Gauge(u, dims)
    op = cb.DiracOp(g, "dwf", mass=0.05, ls=ls)
    n5 = int(np.prod(dims)) // 2 * ls
    mvs, dots = [], []
    for v in range(nvec):
        src = fields.random_source(n5, 100 + v)
        _, d = op.MatPcDagMatPc(src)            # existing entry point: |MatPc src|^2
        dots.append(d)
        mvs.append(op.MatPc(src))
    n = mvs[0].size
    assert n > 592 * 256
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.concatenate(mvs)).to(dev)
    res = torch.zeros(nvec, dtype=torch.float64, device=dev)
    for _ in range(2):
        got = _noalloc_dots(lib, x, n, nvec, res)
        for v in range(nvec):
            assert abs(got[v] - dots[v]) <= 1e-13 * dots[v], (v, got[v], dots[v])

"""The allocation-free entry point cpsb_redot_noalloc against the existing one.

Some callers cannot allocate device memory -- a stream that is recording a
CUDA graph, a solver living inside a fixed HBM arena -- so the library offers
one reduction whose scratch is a static device array.  This test computes
|MatPc in|^2 with it and compares with the |MatPc in|^2 that cpsb_mdagm
reports, twice in a row (the second call reuses the scratch the first one left
behind).  It runs last (file name) and works alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
        res.zero_()
        rc = lib.cpsb_redot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), n, 2,
                                    C.c_void_p(res.data_ptr()), None)
        torch.cuda.synchronize()
        assert rc == 0
        got = res.cpu().numpy()
        assert abs(got[0] - dot_ref) <= 1e-13 * dot_ref
        assert abs(got[1] - float(np.dot(src, src))) <= 1e-13 * float(np.dot(src, src))
    assert lib.cpsb_redot_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), n, 17,
                                  C.c_void_p(res.data_ptr()), None) == -1

"""Dslash bandwidth benchmark: python -m cps_public_b200.dslash_bench [--prec f16,f32,f64]

Times the 5-D Shamir DWF hop (one checkerboard, dag 0) on the 16^3x32, Ls=16
workload with CUDA events over many launches and reports algorithmic GB/s
(spinor in + out + links per application) against the measured HBM copy peak.

--op mdagm times MatPcDagMatPc instead (cpsb_mdagm_multi_dev on nrhs device
vectors, CUDA events over --reps applications), e.g. the Mobius operator with
its fused hop + M5 kernels:
  python -m cps_public_b200.dslash_bench --op mdagm --action mobius --prec f16 --nrhs 12

--op cg runs one InvCg on nrhs seeded sources, stopped after --reps
iterations (a short launch sequence of every CG kernel, for a profiler), e.g.
the 16-bit mixed solve's hop with the fused CG update:
  python -m cps_public_b200.dslash_bench --op cg --dims 16,16,16,16 --prec f16 --nrhs 12 --reps 12
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os

import numpy as np

from . import DiracOp, F16, F32, F64, Gauge, _lib, fields, init

PRECS = {"f16": F16, "f32": F32, "f64": F64}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--prec", default="f16,f32,f64")
    ap.add_argument("--dims", default="16,16,16,32")
    ap.add_argument("--ls", type=int, default=16)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--action", default="dwf")
    ap.add_argument("--op", default="hop", choices=["hop", "mdagm", "cg"])
    a = ap.parse_args()
    dims = tuple(int(x) for x in a.dims.split(","))
    init(0)
    g = Gauge(fields.random_gauge(dims, 0.2, 7), dims)
    op = DiracOp(g, a.action, mass=0.01, ls=a.ls, m5=1.8)
    peak = 6650.0
    try:
        peak = float(json.load(open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                 "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        pass
    lib = _lib.load()
    if a.op == "cg":
        srcs = [fields.random_source(op.n // 24, 100 + q) for q in range(a.nrhs)]
        for name in a.prec.split(","):
            _, rs = op.InvCgMulti(srcs, stop_rsd=1e-10, max_num_iter=a.reps, precision=PRECS[name])
            print(json.dumps({"op": "cg", "action": a.action, "prec": name, "dims": dims, "ls": a.ls,
                              "nrhs": a.nrhs, "iters": [r.iters for r in rs], "status": [r.status for r in rs]}))
        return
    if a.op == "mdagm":
        import torch
        dev = torch.device("cuda", 0)
        src = fields.random_source(op.n // 24, 11)
        x = torch.from_numpy(np.tile(src, a.nrhs)).to(dev)
        y = torch.empty_like(x)
        for name in a.prec.split(","):
            def apply():
                _lib.check(lib.cpsb_mdagm_multi_dev(g.h, C.byref(op.p), PRECS[name], a.nrhs, C.c_void_p(y.data_ptr()),
                                                    C.c_void_p(x.data_ptr()), None, None), "cpsb_mdagm_multi_dev")
            for _ in range(3):
                apply()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(a.reps):
                apply()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / a.reps
            print(json.dumps({"op": "mdagm", "action": a.action, "prec": name, "dims": dims, "ls": a.ls,
                              "nrhs": a.nrhs, "ms_per_application": ms,
                              "note": "includes packing the FP64 CPS-order vectors in and out"}))
        return
    for name in a.prec.split(","):
        ms, by = C.c_double(), C.c_double()
        _lib.check(lib.cpsb_bench_dslash(g.h, C.byref(op.p), PRECS[name], a.nrhs, a.reps, C.byref(ms),
                                         C.byref(by)), "cpsb_bench_dslash")
        gbs = by.value / (ms.value * 1e-3) / 1e9
        print(json.dumps({"prec": name, "dims": dims, "ls": a.ls, "nrhs": a.nrhs, "ms": ms.value,
                          "bytes": by.value, "gbs": gbs, "frac_of_peak": gbs / peak}))


if __name__ == "__main__":
    main()

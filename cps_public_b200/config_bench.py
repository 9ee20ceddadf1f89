"""Benchmarks of the multi-RHS Mobius and the multishift workloads:

  python -m cps_public_b200.config_bench mobius12
      Mobius DWF (b = 1.5, c = 0.5, SYM2 preconditioning) on 24^3x64, Ls = 16,
      M5 = 1.8, m_f = 0.005, links reunitarise(exp(i 0.15 H)) seeded: the 12
      spin-colour point sources at one seeded odd site (4-D source embedded on
      s = 0 / Ls-1 by chirality) solved in one batched mixed-precision CG
      (16-bit and FP32 storage inner, FP64 reliable updates) to FP64 true
      residual 1e-10, against the plain FP64 CG on one of the sources.

  python -m cps_public_b200.config_bench multishift
      Shamir DWF on 24^3x64, Ls = 12, m_f = 0.01, links as above: MInvCG with 12
      shifts log-spaced in [1e-4, 10], per-shift tolerance 1e-10, Gaussian source;
      FP32 Krylov vectors with per-shift mixed-precision refinement to the FP64
      true residual, against the FP64 MInvCG.

  python -m cps_public_b200.config_bench multishift_batch [--nvec 2]
      The same multishift system for nvec pseudofermion sources at once (the
      RHMC batch): cpsb_minvcg_multi (FP32 Krylov + refinement, and FP64)
      against nvec one-source cpsb_minvcg calls in sequence, and, through the
      host-pointer entry points, against nvec concurrent requests of the
      serving loop (cpsb_serve_submit_minvcg on nvec slots).

Each prints one JSON line: solves/s (right-hand sides or shift systems per
second) with sources and solutions resident in device memory (the *_dev entry
points; torch provides the device buffers), the same through the host-pointer
entry points ("e2e", host copies included), iteration counts and the worst
FP64 true residual.  bench.py calls mobius12_run / multishift_run with
arms=... and e2e=False to add these workloads to its line.
"""
from __future__ import annotations

import argparse
import json
import time

import ctypes as C

import numpy as np

from . import F16, F32, F64, MULTI, CgArg, DiracOp, Gauge, SolveResult, _lib, fields, init

DIMS = (24, 24, 24, 64)


def mobius12(a):
    print(json.dumps(mobius12_run(a.stop)))


def mobius12_run(stop=1e-10, arms=("f16", "f32", "f64"), e2e=True):
    """Runs the Mobius 12-point-source workload; arms: inner precisions of the
    12-RHS mixed solves ("f16", "f32") and "f64" (the plain FP64 CG on one
    source).  Returns the result dict."""
    init(0)
    u = fields.random_gauge(DIMS, 0.15, 2401)
    rng = np.random.default_rng(2402)
    while True:  # a seeded site of the solve checkerboard (odd 4-D parity)
        site = tuple(int(rng.integers(d)) for d in DIMS)
        if sum(site) % 2 == 1:
            break
    srcs = [fields.point_source(DIMS, 16, site, sp, c, cb=1, five_d_parity=False) for sp in range(4) for c in range(3)]
    import torch
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    nr = len(srcs)
    b_d = torch.from_numpy(np.stack(srcs)).to(dev)
    x_d = torch.zeros_like(b_d)
    res = (SolveResult * nr)()

    def arm(nrhs, prec):
        # Each arm loads its own gauge and frees it afterwards, which drops its
        # cached solvers: the 12-RHS workspaces of all arms would not fit together.
        g = Gauge(u, DIMS)
        op = DiracOp(g, "mobius", mass=0.005, ls=16, m5=1.8, b=1.5, c=0.5)

        def solve_dev(maxit):
            x_d.zero_()
            torch.cuda.synchronize()
            arg = CgArg(stop, maxit, prec, 0.1, 0)
            t0 = time.perf_counter()
            rc = lib.cpsb_invcg_multi_dev(g.h, C.byref(op.p), C.byref(arg), nrhs, C.c_void_p(x_d.data_ptr()),
                                          C.c_void_p(b_d.data_ptr()), res, None)
            dt = time.perf_counter() - t0
            _lib.check(rc, "cpsb_invcg_multi_dev")
            return dt, [res[i].as_dict() for i in range(nrhs)]

        solve_dev(40)  # warm-up: tunes every launch shape and captures the iteration graphs
        dt, rr = solve_dev(100000)
        x0 = x_d[0].cpu().numpy()
        g.free()
        return dt, rr, x0

    def mixed_rec(t, rr):
        return {"solves_per_s": nr / t, "seconds": t, "iters": max(r["iters"] for r in rr),
                "max_true_rsd": max(r["true_rsd"] for r in rr),
                "reliable_updates": max(r["reliable_updates"] for r in rr)}

    out = {"workload": "mobius_multi_rhs_24x24x24x64_ls16", "rhs": nr, "site": site, "stop_true_rsd": stop}
    x_mixed0 = {}
    if "f64" in arms:
        t_f64, r_f64, x64 = arm(1, F64)
        out["f64_x1"] = {"solves_per_s": 1.0 / t_f64, "seconds": t_f64, "iters": r_f64[0]["iters"],
                         "true_rsd": r_f64[0]["true_rsd"]}
    for name, prec in (("f16", F16), ("f32", F32)):
        if name not in arms:
            continue
        t, rr, x0 = arm(nr, prec)
        x_mixed0[name] = x0
        out[f"mixed_{name}_x12"] = mixed_rec(t, rr)
        if "f64" in arms:
            out[f"mixed_{name}_vs_fp64"] = (nr / t) * t_f64
            out[f"rhs0_mixed_{name}_vs_fp64_rel_diff"] = float(np.linalg.norm(x0 - x64) / np.linalg.norm(x64))
    del b_d, x_d
    torch.cuda.empty_cache()
    if e2e:
        g = Gauge(u, DIMS)
        op = DiracOp(g, "mobius", mass=0.005, ls=16, m5=1.8, b=1.5, c=0.5)
        t0 = time.perf_counter()
        xs, rs = op.InvCgMulti(srcs, stop_rsd=stop, max_num_iter=100000, precision=F16)
        t_e2e = time.perf_counter() - t0
        out["e2e_mixed_f16_x12"] = {"solves_per_s": nr / t_e2e, "seconds": t_e2e,
                                    "max_true_rsd": max(r.true_rsd for r in rs),
                                    "path": "cpsb_invcg_multi (host vectors, copies included)"}
        g.free()
    return out


def multishift(a):
    print(json.dumps(multishift_run(a.stop)))


def multishift_run(stop=1e-10, e2e=True):
    """Runs the 12-shift multishift workload, FP32 Krylov + refinement and FP64;
    returns the result dict."""
    init(0)
    u = fields.random_gauge(DIMS, 0.15, 2403)
    g = Gauge(u, DIMS)
    op = DiracOp(g, "dwf", mass=0.01, ls=12, m5=1.8)
    src = fields.random_source(op.n // 24, 2404)
    shifts = list(np.logspace(-4, 1, 12))
    rsd = [stop] * 12
    import torch
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    ns = len(shifts)
    b_d = torch.from_numpy(src).to(dev)
    x_d = torch.zeros((ns, op.n), dtype=torch.float64, device=dev)
    xptr = (C.c_void_p * ns)(*[C.c_void_p(x_d[k].data_ptr()) for k in range(ns)])
    sh = np.array(shifts)
    al = np.ones(ns)

    def minv_dev(prec, maxit):
        rs_ = np.array(rsd, np.float64)
        arg = CgArg(stop, maxit, prec, 0.1, 0)
        r = SolveResult()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.cpsb_minvcg_dev(g.h, C.byref(op.p), C.byref(arg), xptr, C.c_void_p(b_d.data_ptr()),
                                 _lib.ptr(sh), ns, _lib.ptr(rs_), MULTI, _lib.ptr(al), C.byref(r), None)
        dt = time.perf_counter() - t0
        _lib.check(rc, "cpsb_minvcg_dev")
        return dt, r, rs_

    minv_dev(F32, 30)   # warm-up / tuning
    minv_dev(F64, 30)
    res = {}
    for name, prec in (("f32_krylov_refined", F32), ("f64", F64)):
        dt, r, rs_ = minv_dev(prec, 100000)
        worst = 0.0
        for k in (0, 5, 11):  # FP64 true residual of the smallest, a middle and the largest shift
            xk = x_d[k].cpu().numpy()
            ax, _ = op.MatPcDagMatPc(xk)
            worst = max(worst, float(np.linalg.norm(src - ax - shifts[k] * xk) / np.linalg.norm(src)))
        res[name] = {"seconds": dt, "shift_systems_per_s": ns / dt, "iters": r.iters,
                     "max_reported_rsd": float(np.max(rs_)), "checked_true_rsd": worst}
    del b_d, x_d
    torch.cuda.empty_cache()
    out = {"workload": "dwf_multishift_24x24x24x64_ls12", "shifts": shifts, **res,
           "mixed_vs_fp64": res["f64"]["seconds"] / res["f32_krylov_refined"]["seconds"]}
    if e2e:
        t0 = time.perf_counter()
        op.MInvCG(src, shifts, rsd, ms_type=MULTI, max_num_iter=100000, precision=F32)
        t_e2e = time.perf_counter() - t0
        out["e2e_f32_krylov_refined"] = {"seconds": t_e2e, "shift_systems_per_s": ns / t_e2e,
                                         "path": "cpsb_minvcg (host vectors, copies included)"}
    g.free()
    return out


def multishift_batch(a):
    print(json.dumps(multishift_batch_run(a.stop, a.nvec)))


def multishift_batch_run(stop=1e-10, nvec=2, e2e=True):
    """Runs the 12-shift multishift workload on nvec sources at once and one at a
    time; returns the result dict."""
    init(0)
    u = fields.random_gauge(DIMS, 0.15, 2403)
    g = Gauge(u, DIMS)
    op = DiracOp(g, "dwf", mass=0.01, ls=12, m5=1.8)
    srcs = [fields.random_source(op.n // 24, 2404 + q) for q in range(nvec)]
    shifts = list(np.logspace(-4, 1, 12))
    ns = len(shifts)
    import torch
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    b_d = torch.from_numpy(np.stack(srcs)).to(dev)
    x_d = torch.zeros((nvec, ns, op.n), dtype=torch.float64, device=dev)
    xptr = (C.c_void_p * (nvec * ns))(*[C.c_void_p(x_d[q, s].data_ptr()) for q in range(nvec) for s in range(ns)])
    sh = np.array(shifts)
    al = np.ones(ns)

    def batched(prec, maxit):
        rs_ = np.full((nvec, ns), stop)
        arg = CgArg(stop, maxit, prec, 0.1, 0)
        res = (SolveResult * nvec)()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.cpsb_minvcg_multi_dev(g.h, C.byref(op.p), C.byref(arg), nvec, xptr, C.c_void_p(b_d.data_ptr()),
                                       _lib.ptr(sh), ns, _lib.ptr(rs_), MULTI, _lib.ptr(al), res, None)
        dt = time.perf_counter() - t0
        _lib.check(rc, "cpsb_minvcg_multi_dev")
        return dt, list(res), rs_

    def one_at_a_time(prec, maxit):
        t0 = time.perf_counter()
        iters = []
        for q in range(nvec):
            rs_ = np.full(ns, stop)
            arg = CgArg(stop, maxit, prec, 0.1, 0)
            r = SolveResult()
            xq = (C.c_void_p * ns)(*[C.c_void_p(x_d[q, s].data_ptr()) for s in range(ns)])
            rc = lib.cpsb_minvcg_dev(g.h, C.byref(op.p), C.byref(arg), xq,
                                     C.c_void_p(b_d[q].data_ptr()), _lib.ptr(sh), ns, _lib.ptr(rs_), MULTI,
                                     _lib.ptr(al), C.byref(r), None)
            _lib.check(rc, "cpsb_minvcg_dev")
            iters.append(r.iters)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, iters

    def worst_true(q_list):
        worst = 0.0
        for q in q_list:
            for k in (0, 11):
                xk = x_d[q, k].cpu().numpy()
                ax, _ = op.MatPcDagMatPc(xk)
                worst = max(worst, float(np.linalg.norm(srcs[q] - ax - shifts[k] * xk) / np.linalg.norm(srcs[q])))
        return worst

    batched(F32, 30)   # warm-up / tuning
    batched(F64, 30)
    one_at_a_time(F32, 30)
    out = {"workload": f"dwf_multishift_24x24x24x64_ls12_x{nvec}_sources", "nvec": nvec, "shifts": shifts}
    for name, prec in (("f32_krylov_refined", F32), ("f64", F64)):
        dt, res, rs_ = batched(prec, 100000)
        out["batched_" + name] = {"seconds": dt, "shift_systems_per_s": nvec * ns / dt,
                                  "iters": [r.iters for r in res], "max_reported_rsd": float(np.max(rs_)),
                                  "checked_true_rsd": worst_true(range(nvec))}
        dt1, iters1 = one_at_a_time(prec, 100000)
        out["one_at_a_time_" + name] = {"seconds": dt1, "shift_systems_per_s": nvec * ns / dt1, "iters": iters1}
        out["batched_speedup_" + name] = dt1 / dt
    out["batched_mixed_vs_batched_f64"] = out["batched_f64"]["seconds"] / out["batched_f32_krylov_refined"]["seconds"]
    del b_d, x_d
    torch.cuda.empty_cache()
    if e2e:
        # host-pointer paths, copies included: the batched call against nvec
        # concurrent requests of the serving loop
        t0 = time.perf_counter()
        op.MInvCGMulti(srcs, shifts, [stop] * ns, max_num_iter=100000, precision=F32)
        t_b = time.perf_counter() - t0
        from . import Server
        srv = Server(slots=nvec)
        t0 = time.perf_counter()
        rids = [srv.submit_minvcg(op, s_, shifts, [stop] * ns, max_num_iter=100000, precision=F32) for s_ in srcs]
        for rid in rids:
            srv.wait_minvcg(rid)
        t_c = time.perf_counter() - t0
        srv.close()
        out["e2e_batched_f32_krylov_refined"] = {"seconds": t_b, "path": "cpsb_minvcg_multi (host vectors)"}
        out["e2e_concurrent_requests_f32_krylov_refined"] = {
            "seconds": t_c, "path": f"{nvec} cpsb_serve_submit_minvcg requests on {nvec} slots (host vectors)"}
        out["batched_vs_concurrent_requests"] = t_c / t_b
    g.free()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["mobius12", "multishift", "multishift_batch"])
    ap.add_argument("--stop", type=float, default=1e-10)
    ap.add_argument("--nvec", type=int, default=2)
    a = ap.parse_args()
    {"mobius12": mobius12, "multishift": multishift, "multishift_batch": multishift_batch}[a.workload](a)


if __name__ == "__main__":
    main()

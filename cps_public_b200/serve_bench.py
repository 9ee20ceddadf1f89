"""Serving benchmark: python -m cps_public_b200.serve_bench [--requests N] [--rate R] [--slots S]

A Poisson stream of DWF solve requests against 8 resident seeded gauge fields
(lattices 8^4, 16^3x32, 24^3x64 in turn), each request drawn uniformly: a gauge
field, Ls in {8, 12, 16, 24}, m_f log-uniform in [1e-3, 1e-1], stop_rsd in
{1e-8, 1e-10, 1e-12} and 1-12 Gaussian right-hand sides.  Requests are
submitted at their arrival times to the request loop (cpsb_serve_*), which
admits them by free HBM and runs them concurrently; the line printed reports
p50/p99 latency (submission to completion), requests/s and right-hand-side
solves/s over the run, and the true residual of every solve.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import F16, F32, F64, DiracOp, Gauge, Server, fields, init

LATTICES = [((8, 8, 8, 8), 0.3), ((16, 16, 16, 32), 0.2), ((24, 24, 24, 64), 0.15)]
PRECS = {"f16": F16, "f32": F32, "f64": F64}


def make_requests(n, rate, seed):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for k in range(n):
        reqs.append(dict(arrival=float(t[k]), gauge=int(rng.integers(8)), ls=int(rng.choice([8, 12, 16, 24])),
                         mass=float(10 ** rng.uniform(-3, -1)), tol=float(rng.choice([1e-8, 1e-10, 1e-12])),
                         nrhs=int(rng.integers(1, 13)), seed=int(rng.integers(1 << 30))))
    return reqs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=16)
    ap.add_argument("--rate", type=float, default=20.0, help="mean arrivals per second")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--precision", default="f32", choices=list(PRECS))
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--hbm-fraction", type=float, default=0.85)
    a = ap.parse_args()
    print(json.dumps(run(a.requests, a.rate, a.slots, a.precision, a.seed, a.hbm_fraction)))


def make_gauges():
    """The 8 resident seeded gauge fields (8^4, 16^3x32, 24^3x64 in turn)."""
    init(0)
    gauges = []
    for i in range(8):
        dims, eps = LATTICES[i % 3]
        gauges.append(Gauge(fields.random_gauge(dims, eps, 5000 + i), dims))
    return gauges


def run(requests=16, rate=20.0, slots=4, precision="f32", seed=4, hbm_fraction=0.85, gauges=None,
        one_at_a_time=False):
    """Serves `requests` Poisson arrivals at `rate` per second and returns the
    result dict.  one_at_a_time: each request is submitted only after the
    previous one has completed (latency = service time, no queueing)."""
    gauges = gauges if gauges is not None else make_gauges()
    a = argparse.Namespace(requests=requests, rate=rate, slots=slots, precision=precision, seed=seed,
                           hbm_fraction=hbm_fraction)
    reqs = make_requests(a.requests, a.rate, a.seed)
    # Right-hand sides: per (gauge, Ls) one Gaussian base vector 11 sites longer
    # than a solve's vector; right-hand side i is the window starting at site i
    # (distinct sources without a copy each).
    ops, srcs, bases = [], [], {}
    for r in reqs:
        op = DiracOp(gauges[r["gauge"]], "dwf", mass=r["mass"], ls=r["ls"], m5=1.8)
        ops.append(op)
        key = (r["gauge"], r["ls"])
        if key not in bases:
            bases[key] = fields.random_source(op.n // 24 + 11, 7000 + 31 * r["gauge"] + r["ls"])
        srcs.append([bases[key][24 * i:24 * i + op.n] for i in range(r["nrhs"])])
    srv = Server(slots=a.slots, hbm_fraction=a.hbm_fraction)
    t0 = time.perf_counter()
    ids, done = [], {}
    for r, op, s in zip(reqs, ops, srcs):
        dt = r["arrival"] - (time.perf_counter() - t0)
        if dt > 0 and not one_at_a_time:
            time.sleep(dt)
        rid = srv.submit(op, s, stop_rsd=r["tol"], precision=PRECS[a.precision])
        ids.append(rid)
        if one_at_a_time:
            done[rid] = srv.wait(rid)
    per = []
    worst = 0.0
    for r, op, s, rid in zip(reqs, ops, srcs, ids):
        xs, res, lat = done[rid] if rid in done else srv.wait(rid)
        del xs
        tr = max(float(q.true_rsd) / r["tol"] for q in res)
        worst = max(worst, tr)
        per.append(dict(lattice="x".join(map(str, gauges[r["gauge"]].dims)), ls=r["ls"], mass=round(r["mass"], 5),
                        tol=r["tol"], nrhs=r["nrhs"], iters=max(q.iters for q in res), latency_ms=round(lat, 1),
                        status=max(q.status for q in res)))
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    out = {"metric": "dwf_serving", "requests": a.requests,
           "offered_rate_per_s": None if one_at_a_time else a.rate, "one_at_a_time": one_at_a_time,
           "slots": a.slots,
           "precision": a.precision, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
           "requests_per_s": st["requests_per_s"], "rhs_solves_per_s": st["rhs_per_s"],
           "completed": st["completed"], "failed": st["failed"], "peak_running": st["peak_running"],
           "hbm_budget_gb": st["budget_bytes"] / 1e9, "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9,
           "wall_s": wall, "max_true_rsd_over_tol": worst, "per_request": per}
    return out


if __name__ == "__main__":
    main()

"""Benchmark: Shamir DWF even-odd CG solves/s at true residual 1e-10, mixed vs FP64.

Workload (the reference's headline DWF configuration): 16^3 x 32 lattice,
Ls = 16, M5 = 1.8, m_f = 0.01, links reunitarise(exp(i 0.2 H)) seeded,
Gaussian source on the odd checkerboard, stop_rsd 1e-10 on the FP64 true
residual.  A step is one full solve (MatPcDagMatPc x = b from x = 0) of the
arm's right-hand sides.

Arms:
  (default)        this library.  The headline `value` is the 16-bit-storage
                   mixed-precision CG solving 12 right-hand sides in one batched
                   solve (solves/s counts right-hand sides, each to FP64 true
                   residual 1e-10); FP32-mixed x12, single-RHS 16-bit and FP32
                   mixed, and the plain FP64 CG on one right-hand side are timed
                   beside it.  `value` uses device-resident inputs
                   (cpsb_invcg_multi_dev); `e2e` goes through the host-pointer C
                   ABI (cpsb_invcg_multi) with the H2D copies of guesses and sources
                   and the D2H copy of the solutions in every step.
  --impl reference the CPS noarch CPU code (oracle/_ref/cpsref, compiled from the
                   reference sources) on all host cores: each step runs one
                   MatPcDagMatPc per core in parallel processes, and solves/s is
                   extrapolated with the FP64 CG iteration count of this workload.

Multi-GPU (--gpus N under torchrun): independent replicas, one per GPU, no
data-path collective; value = solves on all ranks / max elapsed over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (16, 16, 16, 32)
LS = 16
M5 = 1.8
MF = 0.01
EPS = 0.2
STOP = 1e-10
SEED = 2024
METRIC = "dwf_cg_solves_per_s"
UNIT = "solves/s"
# FP64 CG iterations (CPS counting, itr+1) of this workload, measured on B200 by
# the FP64 solver, which runs CPS's recurrence (its iteration counts match the
# compiled reference within one on every golden case).  The CPU arm uses it to
# turn one timed MatPcDagMatPc into solves/s.
FP64_ITERS = 348
WORKLOAD = {"workload": "shamir_dwf_eo_cg_16x16x16x32_ls16", "lattice": "16^3x32", "ls": LS, "m5": M5, "mf": MF,
            "link_eps": EPS, "stop_true_rsd": STOP, "source": "gaussian odd checkerboard", "reliable_delta": 0.1,
            "l2": "inputs larger than L2 (201 MB FP64 / 52 MB FP16 per vector, 75 MB FP64 links)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other BASELINE workloads (Wilson 8^4, Mobius x12, multishift, serving)")
    return ap.parse_args()


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank number over all ranks (identity without a
    process group): every multi-GPU time in this file is the slowest rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput of independent replicas: all ranks' units over the
    slowest rank's time."""
    return world * units_per_rank / max_seconds


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 8:
                continue
            for n, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the FP16 Dslash from the committed ncu summary."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "dslash_dram_traffic_dwf_16x16x16x32_ls16.json")))
        return d
    except Exception:
        return None


def make_inputs(nsrc):
    from cps_public_b200 import fields
    u = fields.random_gauge(DIMS, EPS, SEED)
    n5 = int(np.prod(DIMS)) // 2 * LS
    srcs = [fields.random_source(n5, SEED + 1 + i) for i in range(nsrc)]
    return u, srcs


# Solver arms: (name, inner precision, right-hand sides per solve).  The
# headline is the 16-bit-storage mixed-precision CG on NRHS right-hand sides in
# one batched solve (every RHS to FP64 true residual 1e-10); the plain FP64 CG
# on one right-hand side is its reference point (mixed_vs_fp64).
NRHS = 12
HEADLINE = "f16_mixed_x12"


def arms(cb):
    return [("f16_mixed_x12", cb.F16, NRHS), ("f32_mixed_x12", cb.F32, NRHS), ("f16_mixed", cb.F16, 1),
            ("f32_mixed", cb.F32, 1), ("f64", cb.F64, 1)]


def run_ours(args):
    import ctypes as C

    import torch
    import cps_public_b200 as cb
    from cps_public_b200 import _lib
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    cb.init(local)
    lib = _lib.load()
    npool = NRHS + 4
    u, srcs = make_inputs(npool)
    g = cb.Gauge(u, DIMS)
    op = cb.DiracOp(g, "dwf", mass=MF, ls=LS, m5=M5)
    n = op.n
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    pool = torch.stack([torch.from_numpy(s) for s in srcs]).to(dev)      # npool x n, device resident
    b_dev = torch.empty((NRHS, n), dtype=torch.float64, device=dev)
    x_dev = torch.zeros((NRHS, n), dtype=torch.float64, device=dev)
    res = (cb.SolveResult * NRHS)()

    def batch(k, nrhs):
        # step k solves pool rows k, k+1, ... (mod npool): inputs differ from step to step
        idx = torch.tensor([(k + i) % npool for i in range(nrhs)], device=dev)
        torch.index_select(pool, 0, idx, out=b_dev[:nrhs])

    def solve_on_device(nrhs, prec):
        x_dev[:nrhs].zero_()
        a = cb.CgArg(STOP, 100000, prec, 0.1, 0)
        rc = lib.cpsb_invcg_multi_dev(g.h, C.byref(op.p), C.byref(a), nrhs, C.c_void_p(x_dev.data_ptr()),
                                      C.c_void_p(b_dev.data_ptr()), res, C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"solve failed rc={rc} ({lib.cpsb_last_error().decode()}) {res[0].as_dict()}")
        return [res[i].as_dict() for i in range(nrhs)]

    out = {}
    sampler = ClockSampler(local)
    launches0 = C.c_ulonglong()
    launches1 = C.c_ulonglong()
    clocks = None
    for name, prec, nrhs in arms(cb):
        for w in range(args.warmup):
            batch(w, nrhs)
            solve_on_device(nrhs, prec)
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        head = name == HEADLINE
        if head:
            sampler.start()
            lib.cpsb_kernel_launches(C.byref(launches0))
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        infos = []
        torch.cuda.synchronize()
        # NVTX range "timed_<arm>": lets a profiler select one arm's timed solves
        # (ncu --nvtx --nvtx-include "timed_f16_mixed_x12/").
        torch.cuda.nvtx.range_push("timed_" + name)
        for k in range(args.steps):
            batch(args.warmup + k, nrhs)
            ev[k][0].record(stream)
            infos += solve_on_device(nrhs, prec)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if head:
            lib.cpsb_kernel_launches(C.byref(launches1))
            clocks = sampler.stop()
        lat = [ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)]
        total_ms = max_over_ranks(ev[0][0].elapsed_time(ev[-1][1]), dev)
        out[name] = {"solves_per_s": rate(nrhs * args.steps, world, total_ms / 1000.0), "rhs_per_solve": nrhs,
                     "ms_per_step": total_ms / args.steps,
                     "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "iters": int(statistics.median(i["iters"] for i in infos)),
                     "max_true_rsd": max(i["true_rsd"] for i in infos),
                     "reliable_updates": int(statistics.median(i["reliable_updates"] for i in infos))}
        assert out[name]["max_true_rsd"] <= STOP, (name, out[name])
    head_prec = dict((a[0], a[1]) for a in arms(cb))[HEADLINE]
    # e2e: host buffers through the public host-pointer entry point (cpsb_invcg_multi):
    # every step copies the NRHS guesses and sources in and the NRHS solutions out.
    e2e_lat = []
    for k in range(args.warmup + args.steps):
        bs = [srcs[(k + i) % npool] for i in range(NRHS)]
        t0 = time.perf_counter()
        xs, rs = op.InvCgMulti(bs, stop_rsd=STOP, max_num_iter=100000, precision=head_prec)
        if k >= args.warmup:
            e2e_lat.append(time.perf_counter() - t0)
        assert max(r.true_rsd for r in rs) <= STOP
    e2e_total = max_over_ranks(sum(e2e_lat), dev)
    # Dslash roofline: the 16-bit 5-D hop on NRHS right-hand sides, the dominant
    # kernel of the headline solve, timed with CUDA events on its stream.
    dsl = {}
    peak, peak_kind = peak_hbm()
    for pname, prec, nr in (("f16_x12", cb.F16, NRHS), ("f16", cb.F16, 1), ("f32", cb.F32, 1), ("f64", cb.F64, 1)):
        ms, by = C.c_double(), C.c_double()
        lib.cpsb_bench_dslash(g.h, C.byref(op.p), prec, nr, 50 if nr == 1 else 10, C.byref(ms), C.byref(by))
        gbs = by.value / (ms.value * 1e-3) / 1e9
        dsl[pname] = {"ms": ms.value, "bytes": by.value, "gbs": gbs, "frac": gbs / peak}
    traffic = ncu_traffic()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    head = out[HEADLINE]
    line = {
        "metric": METRIC, "value": head["solves_per_s"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16-storage/f32-math, f64 reliable updates",
        "data": "synthetic (seeded reunitarised exp(i*0.2*H) links, Gaussian sources)",
        "config": dict(WORKLOAD, rhs_per_solve=NRHS), "parallelism": f"replicas x{world}",
        "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"],
        "variants": out,
        "mixed_vs_fp64": head["solves_per_s"] / out["f64"]["solves_per_s"],
        "e2e": {"value": rate(NRHS * args.steps, world, e2e_total), "unit": UNIT,
                "h2d_bytes_per_step": 2 * NRHS * n * 8, "d2h_bytes_per_step": NRHS * n * 8,
                "path": "cpsb_invcg_multi (host pointers, pinned staging)"},
        "roofline": {"bound": "hbm", "achieved": dsl["f16_x12"]["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": dsl["f16_x12"]["frac"], "peak_kind": peak_kind,
                     "traffic": (traffic or {}).get("f16_x12_bytes_per_launch"),
                     "kernel": f"16-bit 5-D Shamir hop, one checkerboard, {NRHS} right-hand sides",
                     "algorithmic_bytes": dsl["f16_x12"]["bytes"]},
        "dslash_gbs": {k: v["gbs"] for k, v in dsl.items()},
        "dslash_frac": {k: v["frac"] for k, v in dsl.items()},
        "gpu_launches": int(launches1.value - launches0.value),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(u, srcs[0], out["f64"]["iters"])
    if world == 1 and not args.no_configs:
        # The other workloads of the reference's benchmark set, each with its own
        # small, stated number of timed runs (not --steps); the headline's
        # workspaces are released first.
        g.free()
        del pool, b_dev, x_dev
        torch.cuda.empty_cache()
        line["configs"] = run_configs(args.no_cpu_baseline)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line, default=_plain))


def config0_wilson(with_cpu=True):
    """Plain Wilson even-odd CG, FP64, 8^4 periodic, mass 0.1, stop 1e-10 (links
    eps 0.3, Gaussian odd-checkerboard source): 3 warm-up and 20 timed solves
    through the device-pointer entry point; the compiled reference's own solve of
    the same system on one host core beside it."""
    import ctypes as C

    import torch
    import cps_public_b200 as cb
    from cps_public_b200 import _lib, fields
    dims = (8, 8, 8, 8)
    u = fields.random_gauge(dims, 0.3, 2020)
    src = fields.random_source(int(np.prod(dims)) // 2, 2021)
    g = cb.Gauge(u, dims)
    op = cb.DiracOp(g, "wilson", mass=0.1)
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    b = torch.from_numpy(src).to(dev)
    x = torch.zeros_like(b)
    res = cb.SolveResult()
    st = torch.cuda.current_stream(dev)
    lat = []
    for k in range(23):
        x.zero_()
        a = cb.CgArg(STOP, 5000, cb.F64, 0.0, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc = lib.cpsb_invcg_dev(g.h, C.byref(op.p), C.byref(a), C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()),
                                C.byref(res), C.c_void_p(st.cuda_stream))
        e1.record(st)
        torch.cuda.synchronize()
        assert rc == 0 and res.true_rsd <= STOP
        if k >= 3:
            lat.append(e0.elapsed_time(e1))
    g.free()
    out = {"workload": "wilson_eo_cg_fp64_8x8x8x8", "mass": 0.1, "stop_true_rsd": STOP, "timed_solves": len(lat),
           "solves_per_s": 1000.0 * len(lat) / sum(lat), "p50_ms": float(np.percentile(lat, 50)),
           "p99_ms": float(np.percentile(lat, 99)), "iters": res.iters, "true_rsd": res.true_rsd}
    if with_cpu:
        from oracle import refrun
        if refrun.available():
            t0 = time.perf_counter()
            it, rp, _ = refrun.run(refrun.OP_INVCG, "wilson", dims, u, [src, np.zeros_like(src)], mass=0.1,
                                   stop_rsd=STOP, max_iter=5000, threads=1)
            out["cpu_reference"] = {"seconds_per_solve": float(rp[10]), "solves_per_s": 1.0 / float(rp[10]),
                                    "iters": it, "cores": 1,
                                    "sample": "one CPS noarch InvCg solve (compiled reference), its own timing"}
    return out


def run_configs(no_cpu=False):
    """BASELINE's other configurations, each with a stated small sample."""
    from cps_public_b200 import config_bench, serve_bench
    cfg = {}
    t0 = time.perf_counter()
    cfg["config0"] = config0_wilson(with_cpu=not no_cpu)
    cfg["config2"] = dict(config_bench.mobius12_run(STOP, arms=("f16", "f64"), e2e=False),
                          sample="one timed 12-RHS 16-bit mixed solve and one FP64 solve, each after a 40-iteration "
                                 "warm-up")
    cfg["config3"] = dict(config_bench.multishift_run(STOP, e2e=False),
                          sample="one timed multishift solve per arm after a 30-iteration warm-up")
    gauges = serve_bench.make_gauges()
    sat = serve_bench.run(requests=12, rate=20.0, slots=4, precision="f32", seed=4, gauges=gauges)
    light = serve_bench.run(requests=6, rate=0.2, slots=4, precision="f32", seed=6, gauges=gauges)
    alone = serve_bench.run(requests=4, rate=20.0, slots=4, precision="f32", seed=5, gauges=gauges,
                            one_at_a_time=True)
    for d in (sat, light, alone):
        d.pop("per_request", None)
    cfg["config4"] = {"poisson_20_per_s": sat, "poisson_0.2_per_s": light, "one_at_a_time": alone,
                      "sample": "12 Poisson arrivals at 20/s (saturated: one GPU serves ~0.3-0.6 requests/s of this "
                                "mix), 6 Poisson arrivals at 0.2/s (below capacity), and 4 requests submitted one at "
                                "a time (latency = service time, no queueing)"}
    del gauges
    cfg["seconds"] = time.perf_counter() - t0
    return cfg


def _ref_mdagm_seconds(u, src, nproc, threads_per_proc=1):
    """Runs nproc concurrent reference processes, each timing one MatPcDagMatPc;
    returns (per-process in-harness seconds, overlap report).  The report holds
    the union of the processes' timed windows and the span common to all of
    them (steady clock): a step counts as concurrent only if that span is
    positive, i.e. every process was inside its MatPcDagMatPc at one instant."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import refrun

    def one(_):
        _, rp, _ = refrun.run(refrun.OP_BENCH, "dwf", DIMS, u, [src], ls=LS, mass=MF, m5=M5, reps=1,
                              threads=threads_per_proc)
        return rp[10], rp[11], rp[12]

    with ThreadPoolExecutor(max_workers=nproc) as ex:
        res = list(ex.map(one, range(nproc)))
    ts = [r[0] for r in res]
    starts, ends = [r[1] for r in res], [r[2] for r in res]
    overlap = {"union_s": max(ends) - min(starts), "common_s": max(0.0, min(ends) - max(starts)),
               "all_overlap": bool(min(ends) > max(starts))}
    return ts, overlap


def cpu_baseline(u, src, iters):
    from oracle import refrun
    cores = os.cpu_count() or 1
    if refrun.available():
        ts, ov = _ref_mdagm_seconds(u, src, cores)
        per = max(ts)
        rate = cores / (per * iters)
        return {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"{cores} concurrent CPS noarch processes, one MatPcDagMatPc each at 16^3x32x16 "
                          f"(slowest {per:.2f} s; windows {'all overlapping' if ov['all_overlap'] else 'NOT all overlapping'}"
                          f", common span {ov['common_s']:.2f} s of union {ov['union_s']:.2f} s); solves/s "
                          f"extrapolated with {iters} CG iterations",
                "mdagm_s": per, "windows": ov}
    from oracle import oracle
    op = oracle.Op("dwf", DIMS, u, ls=LS, mass=MF, m5=M5)
    t0 = time.perf_counter()
    op.mdagm(src)
    per = time.perf_counter() - t0
    return {"value": 1.0 / (per * iters), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one MatPcDagMatPc of the C oracle ({per:.2f} s); extrapolated with {iters} iterations"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from oracle import refrun
    iters = FP64_ITERS
    u, srcs = make_inputs(1)
    cores = os.cpu_count() or 1
    if not refrun.available():
        kind = "port"
    else:
        kind = "reference"
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable": "FP64 iteration count of the workload not recorded"}))
        return
    times, overlaps = [], []
    for k in range(args.warmup + args.steps):
        if kind == "reference":
            # the step ends when the slowest concurrent process has applied its
            # MatPcDagMatPc; process start-up and field input are not CPS's path
            ts, ov = _ref_mdagm_seconds(u, srcs[0], cores)
            wall = max(ts)
        else:
            from oracle import oracle
            op = oracle.Op("dwf", DIMS, u, ls=LS, mass=MF, m5=M5)
            t0 = time.perf_counter()
            op.mdagm(srcs[0])
            wall = time.perf_counter() - t0
            ov = None
        if k >= args.warmup:
            times.append(wall)
            overlaps.append(ov)
    nper = cores if kind == "reference" else 1
    step = statistics.mean(times)
    rate = nper / (step * iters)
    conc = ""
    if kind == "reference":
        n_ok = sum(1 for o in overlaps if o["all_overlap"])
        conc = (f"; in {n_ok} of {len(overlaps)} steps every process's timed window overlapped all others "
                f"(median common span {statistics.median(o['common_s'] for o in overlaps):.2f} s of "
                f"{statistics.median(o['union_s'] for o in overlaps):.2f} s)")
    # A step is the measured one: nper concurrent MatPcDagMatPc applications
    # (ms_per_step, what the timed region holds).  One CPS solve of this
    # workload takes hours, so solves/s is extrapolated from the step with the
    # FP64 CG iteration count; the per-solve time is reported beside it.
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step * 1000, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, rhs_per_solve=NRHS), "parallelism": f"cpu x{nper} processes",
            "impl": "reference",
            "step": f"{nper} concurrent MatPcDagMatPc applications (one per process)",
            "extrapolated_ms_per_solve": step * 1000 * iters / nper,
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": nper, "kind": kind,
                             "sample": f"per step: {nper} concurrent MatPcDagMatPc at 16^3x32x16 "
                                       f"({step:.2f} s, the slowest process's own timing); extrapolated with "
                                       f"{iters} CG iterations; CPS "
                                       f"solves the {NRHS} right-hand sides one after another, so the "
                                       f"per-right-hand-side rate is the solve rate{conc}"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=_plain))


def _plain(o):
    """JSON form of numpy scalars and arrays in a result line."""
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError(f"not JSON serializable: {type(o).__name__}")


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

// solver.cu -- conjugate-gradient drivers on MatPcDagMatPc.
//
// Plain FP64 CG restates DiracOp::InvCgShift (cps_pp/src/util/dirac_op/d_op_base/
// comsrc/inv_cg.C:84-447): the same recurrence, stopping test |r|^2 <=
// stop_rsd^2 |src|^2 on the iterated residual, at most max_num_iter-1
// iterations, the true residual computed once at the end, and itr+1 returned.
//
// Mixed precision runs the same recurrence in FP32 or FP16 storage (FP32
// arithmetic, FP64 reductions) and replaces the residual by the FP64 true
// residual b - A x whenever the iterated residual has dropped by
// reliable_delta since the last replacement, or claims convergence; the
// solution is accumulated in FP64 at each replacement, and the solve only ends
// when the FP64 true residual meets the tolerance.
//
// Iterations are launched in batches captured as one CUDA graph: every scalar
// lives in device memory (CgState) and a halting RHS turns the rest of the batch
// into early exits.  The batch is the body of a device-side loop
// (graph_loop.cu), so one graph launch runs batches until a right-hand side
// needs the host (convergence, a reliable update, the iteration limit), and
// the host reads the state only then.
#include <math.h>
#include <string.h>

#include <chrono>

#include "host.h"

namespace cpsb {

CgSolver::CgSolver(Gauge *g, const cpsb_dirac_params &pp, int sl, int nr) : G(g), p(pp), sloppy(sl), nrhs(nr) {
  // The FP64 operator serves the FP64 recurrence (all right-hand sides at once)
  // or, for mixed precision, only the true residuals, which it forms one
  // right-hand side at a time so that its temporaries are one vector each.
  op64.reset(new Operator(G, p, P64, sl == P64 ? nr : 1));
  geom = op64->geom;
  geom.nrhs = nr;
  geom.nsites = op64->geom.nsites / op64->geom.nrhs * nr;
  const long n = geom.nsites;
  x64.create(P64, n);
  b64.create(P64, n);
  r64.create(P64, n);
  if (sloppy != P64) {
    opS.reset(new Operator(G, p, sloppy, nrhs));
    G->ptr(sloppy);  // build the reduced-precision links now, never inside a graph capture
    rS.create(sloppy, n);
    pS.create(sloppy, n);
    ApS.create(sloppy, n);
    // the iterates' sum since the last reliable update, in FP32 for FP32 and
    // 16-bit solves: a 16-bit sum's rounding noise, amplified by the condition
    // number in the true residual, stalls ill-conditioned solves (DWF m_f 0.01)
    xS.create(P32, n);
  } else {
    rS.create(P64, n);  // r, p, Ap of the FP64 recurrence
    pS.create(P64, n);
    ApS.create(P64, n);
    pcg_partial.alloc(sizeof(double) * PCG_PARTIAL_SLOTS);
    pcg_bar.alloc(4 * sizeof(unsigned));
  }
  state.alloc(sizeof(CgState));
  CK(cudaMallocHost((void **)&hstate, sizeof(CgState)));
  loop.alloc(sizeof(LoopCtl));
  CK(cudaMallocHost((void **)&hloop, 2 * sizeof(LoopCtl)));
  CK(cudaMallocHost((void **)&hscal, sizeof(double) * MAX_RHS));
  p.zmobius_b = p.zmobius_c = nullptr;  // the operators hold copies of the zMobius coefficients
  scal.alloc(sizeof(double) * MAX_RHS * 8);
}

CgSolver::~CgSolver() {
  if (graph) cudaGraphExecDestroy(graph);
  if (hstate) cudaFreeHost(hstate);
  if (hloop) cudaFreeHost(hloop);
  if (hscal) cudaFreeHost(hscal);
}

static Scal2 sc2(int n, double a, double b) {
  Scal2 s;
  for (int i = 0; i < MAX_RHS; i++) {
    s.a[i] = a;
    s.b[i] = b;
  }
  (void)n;
  return s;
}

// One batch of k iterations of the (sloppy or FP64) recurrence.
void CgSolver::launch_batch(int k, cudaStream_t st) {
  CgState *S = (CgState *)state.p;
  Operator &op = opS ? *opS : *op64;
  const int px = opS ? xS.prec : P64;
  Field &xx = opS ? xS : x64;
  Reduce rd = red_d.r(S->d);
  Reduce rr = red_r.r(nullptr);
  Reduce rp = red_p.r(nullptr);
  const bool fused = op.can_fuse_cg_r();
  for (int j = 0; j < k; j++) {
    if (fused) {
      // the residual update rides on the last hop of MatPcDagMatPc (A p stays in registers)
      // and so does x += alpha p: the x/p kernel then updates p alone
      const SpinorPtr xp = xx.ptr();
      op.mdagm_cg_r(ApS.ptr(), pS.ptr(), &rd, S->halt, S, rS.ptr(), &rr, shift != 0.0, &xp, st);
    } else {
      op.mdagm(ApS, pS, &rd, S->halt, st);
      CK(launch_cg_r_update(op.prec, op.geom, rS.ptr(), ApS.ptr(), pS.ptr(), S, rr, st));
    }
    CK(launch_cg_xp_update(px, op.prec, op.geom, fused ? SpinorPtr{} : xx.ptr(), pS.ptr(), rS.ptr(), S, rp, st));
  }
}

void CgSolver::run_batches(int batch, cudaStream_t st, const bool *done, bool any) {
  // the captured iterations depend on whether the solve is shifted (the fused
  // residual update then also reads p)
  const bool shifted = shift != 0.0;
  if (!graph || graph_batch != batch || graph_shifted != shifted) {
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    // One uncaptured application tunes the sloppy operator's launch shapes.
    {
      CgState *S = (CgState *)state.p;
      Operator &op = opS ? *opS : *op64;
      Reduce rd = red_d.r(S->d);
      op.mdagm(ApS, pS, &rd, S->halt, st);
    }
    size_t nn = 0;
    graph_loop = graph_loops_enabled() &&
                 build_loop_graph(st, [&](cudaGraphConditionalHandle h) {
                   launch_batch(batch, st);
                   CK(launch_cg_loop_cond(h, (const CgState *)state.p, (LoopCtl *)loop.p, nrhs, any ? 1 : 0, st));
                 }, &graph, &nn);
    if (!graph_loop) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      set_capturing(true);
      try {
        launch_batch(batch, st);
      } catch (...) {
        set_capturing(false);
        cudaStreamEndCapture(st, &g);
        throw;
      }
      set_capturing(false);
      CK(cudaStreamEndCapture(st, &g));
      CK(cudaGraphGetNodes(g, nullptr, &nn));
      CK(cudaGraphInstantiate(&graph, g, 0));
      cudaGraphDestroy(g);
    }
    graph_nodes = nn;
    graph_batch = batch;
    graph_shifted = shifted;
  }
  for (;;) {
    if (graph_loop) {
      // batches that can still do work, plus one: every launch ends
      LoopCtl &c = hloop[0];
      c.count = 0;
      c.cap = (unsigned)((hstate->max_iter + batch - 1) / batch + 2);
      for (int q = 0; q < MAX_RHS; q++) c.done[q] = q < nrhs && done[q] ? 1 : 0;
      CK(cudaMemcpyAsync(loop.p, &c, sizeof(LoopCtl), cudaMemcpyHostToDevice, st));
    }
    CK(cudaGraphLaunch(graph, st));
    CK(cudaMemcpyAsync(hstate, state.p, sizeof(CgState), cudaMemcpyDeviceToHost, st));
    if (graph_loop) CK(cudaMemcpyAsync(&hloop[1], loop.p, sizeof(LoopCtl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    count_launch(graph_nodes * (graph_loop ? hloop[1].count : 1));
    bool all = true, one = false;
    for (int q = 0; q < nrhs; q++) {
      all = all && hstate->halt_done[q];
      one = one || (hstate->halt_done[q] && !done[q]);
    }
    if (all || (any && one)) return;
  }
}

bool CgSolver::run_persistent(cudaStream_t st) {
  const int mode = persistent_cg_mode();
  if (opS || shift != 0.0 || mode == 0 || !op64->can_fuse_cg_r()) return false;
  // automatic: Wilson fields small enough for the direction-parallel form (for
  // DWF, whose columns of slices share each link, the graph loop is faster)
  if (mode == 1 && (geom.nsites > PCG_AUTO_SITES || p.action != CPSB_WILSON)) return false;
  Operator &op = *op64;
  DslashArgs A;
  memset(&A, 0, sizeof(A));
  A.g = op.geom;
  A.U = G->ptr(P64);
  A.five_d = p.action == CPSB_DWF;
  A.hop5 = p.action == CPSB_DWF;
  A.hop5_fact = 2.0 * p.a5_inv;
  A.hop5_wall = -2.0 * p.mass * p.a5_inv;
  A.bc_t_sign = 1.0;  // FP64 links carry the boundary sign
  const cudaError_t e =
      launch_persistent_cg(A, -op.kappa * op.kappa, op.t1.ptr(), op.t2.ptr(), rS.ptr(), pS.ptr(), x64.ptr(),
                           (CgState *)state.p, (double *)pcg_partial.p, PCG_PARTIAL_SLOTS, (unsigned *)pcg_bar.p, st);
  if (e == cudaErrorNotSupported) {
    cudaGetLastError();
    return false;
  }
  CK(e);
  unsigned flags[4];
  CK(cudaMemcpyAsync(hstate, state.p, sizeof(CgState), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(flags, pcg_bar.p, sizeof(flags), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (flags[2]) throw Error{CPSB_ERR_CUDA, "persistent CG: a grid barrier wait ran out"};
  return true;
}

// rr_out[q] = |b - (A + shift) x64|^2 (FP64), leaves r64 = b - (A + shift) x64,
// for every right-hand side q not masked by skip_h (host) / skip_d (the same
// mask on the device); masked entries of rr_out and r64 are left as they were.
void CgSolver::true_residual(double *rr_out, const double *bnorm, cudaStream_t st, const int *skip_h,
                             const int *skip_d) {
  (void)bnorm;
  double *dres = (double *)scal.p;
  // r = b - (A + shift) x, formed in place in r (no separate A x vector)
  if (op64->nrhs == nrhs) {
    op64->mdagm(r64, x64, nullptr, skip_d, st);
  } else {
    const long n1 = op64->nsites();
    for (int q = 0; q < nrhs; q++)
      if (!(skip_h && skip_h[q])) op64->mdagm(r64.view(q * n1), x64.view(q * n1), nullptr, nullptr, st);
  }
  Reduce rm = red_misc.r(dres);
  if (shift != 0.0) {
    Reduce none;
    memset(&none, 0, sizeof(none));
    CK(launch_axpby(P64, r64.ptr(), P64, r64.ptr(), P64, x64.ptr(), geom, sc2(nrhs, 1.0, shift), skip_d,
                    none, 0, st));
  }
  CK(launch_axpby(P64, r64.ptr(), P64, b64.ptr(), P64, r64.ptr(), geom, sc2(nrhs, 1.0, -1.0), skip_d, rm, 1,
                  st));
  double rr[MAX_RHS];
  CK(cudaMemcpyAsync(rr, dres, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int q = 0; q < nrhs; q++)
    if (!(skip_h && skip_h[q])) rr_out[q] = rr[q];
}

int CgSolver::solve(const cpsb_cg_arg &a, cpsb_solve_result *res, cudaStream_t st, double sigma,
                    const double *stop_q) {
  auto stop = [&](int q) { return stop_q ? stop_q[q] : a.stop_rsd; };
  auto t0 = std::chrono::steady_clock::now();
  shift = sigma;
  const Geom &gg = geom;
  double bnorm[MAX_RHS], rr[MAX_RHS];
  double *dres = (double *)scal.p;
  // |b|^2, read back by the synchronisation that ends the true residual
  {
    Reduce rm = red_misc.r(dres + 7 * MAX_RHS);
    CK(launch_redot(P64, gg, b64.ptr(), b64.ptr(), rm, st));
    CK(cudaMemcpyAsync(hscal, dres + 7 * MAX_RHS, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
  }
  // r = b - A x
  true_residual(rr, bnorm, st);
  for (int q = 0; q < nrhs; q++) bnorm[q] = hscal[q];
  CgState hs;
  memset(&hs, 0, sizeof(hs));
  const double delta = sloppy == P64 ? 0.0 : (a.reliable_delta > 0 ? a.reliable_delta : 0.1);
  hs.delta = delta;
  hs.shift = shift;
  hs.max_iter = a.max_num_iter;
  hs.nrhs = nrhs;
  int nupd[MAX_RHS] = {0};
  bool done[MAX_RHS];
  for (int q = 0; q < nrhs; q++) {
    hs.rr[q] = rr[q];
    hs.pp[q] = rr[q];  // p = r
    hs.stp[q] = bnorm[q] * stop(q) * stop(q);
    hs.maxr[q] = sqrt(rr[q]);
    done[q] = (rr[q] <= hs.stp[q]) || (a.max_num_iter - 1 <= 0);
    hs.halt[q] = hs.halt_done[q] = done[q] ? 1 : 0;
    hs.reason[q] = done[q] ? HALT_CONVERGED : HALT_NONE;
    if (bnorm[q] == 0.0) {  // CPS divides by |src|^2; a zero source is solved by x = 0
      done[q] = true;
      hs.halt[q] = hs.halt_done[q] = 1;
    }
  }
  // p = r (sloppy copy of r), xS = 0
  if (opS) {
    CK(launch_convert(sloppy, rS.ptr(), P64, r64.ptr(), gg.nsites, st));
    CK(cudaMemsetAsync(xS.data.p, 0, xS.data.bytes, st));
    if (xS.norm.p) CK(cudaMemsetAsync(xS.norm.p, 0, xS.norm.bytes, st));  // quantum 0: every value 0
  } else {
    CK(cudaMemcpyAsync(rS.data.p, r64.data.p, r64.data.bytes, cudaMemcpyDeviceToDevice, st));
  }
  CK(cudaMemcpyAsync(pS.data.p, rS.data.p, rS.data.bytes, cudaMemcpyDeviceToDevice, st));
  if (pS.norm.p) CK(cudaMemcpyAsync(pS.norm.p, rS.norm.p, rS.norm.bytes, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(state.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st));
  // The host mirror starts from this solve's state: a right-hand side that has
  // converged before the first iteration reports it (CPS: itr + 1 = 1), not
  // the state the previous solve left behind.
  *hstate = hs;

  // Iterations per graph launch.  The host looks at the state between
  // launches, so a right-hand side that pauses for a reliable update idles
  // until its launch ends; with many right-hand sides an iteration is long
  // (milliseconds) and a host round trip every couple of iterations costs
  // little, so the batch shrinks as the right-hand sides grow.
  int batch = a.batch > 0 ? a.batch : (nrhs >= 8 ? 2 : nrhs >= 2 ? 4 : 16);
  // With the device-side loop a batch ends in a (cheap) condition check, not
  // a host round trip: short batches leave less idle work after a right-hand
  // side halts.
  if (a.batch <= 0 && graph_loops_enabled()) batch = nrhs >= 8 ? 1 : nrhs >= 2 ? 2 : 4;
  int status = CPSB_OK;
  for (;;) {
    bool all = true;
    for (int q = 0; q < nrhs; q++) all = all && done[q];
    if (all) break;
    if (!run_persistent(st)) run_batches(batch, st, done, opS != nullptr);
    CgState h = *hstate;
    if (!opS) {
      for (int q = 0; q < nrhs; q++) done[q] = true;
      break;
    }
    // Reliable update for every RHS that paused: x += xS, xS = 0, r = b - A x
    // in FP64.  RHS still iterating are masked out of every update.
    int *dskip = (int *)((double *)scal.p + MAX_RHS * 4);
    int skip_h[MAX_RHS];
    for (int q = 0; q < nrhs; q++) skip_h[q] = (done[q] || !h.halt_done[q]) ? 1 : 0;
    CK(cudaMemcpyAsync(dskip, skip_h, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, st));
    Reduce none;
    memset(&none, 0, sizeof(none));
    CK(launch_axpby(P64, x64.ptr(), P64, x64.ptr(), xS.prec, xS.ptr(), gg, sc2(nrhs, 1.0, 1.0), dskip, none, 0, st));
    CK(launch_axpby(xS.prec, xS.ptr(), xS.prec, xS.ptr(), xS.prec, SpinorPtr{}, gg, sc2(nrhs, 0.0, 0.0), dskip, none, 0,
                    st));
    // only the right-hand sides that paused need their FP64 residual
    true_residual(rr, bnorm, st, skip_h, dskip);
    Scal2 beta = sc2(nrhs, 1.0, 0.0);
    for (int q = 0; q < nrhs; q++) {
      if (skip_h[q]) continue;
      nupd[q]++;
      const int reason = h.reason[q];
      if (rr[q] <= h.stp[q]) {
        done[q] = true;
        h.reason[q] = HALT_CONVERGED;
        continue;
      }
      if (reason == HALT_MAXITER || reason == HALT_BREAKDOWN) {
        done[q] = true;
        continue;
      }
      // continue: r_s = r (true), p = r + beta p with beta = rr_true / rr_prev
      beta.b[q] = rr[q] / h.rr_prev[q];
      h.rr[q] = rr[q];
      h.maxr[q] = sqrt(rr[q]);
      h.halt[q] = h.halt_done[q] = 0;
      h.reason[q] = HALT_NONE;
    }
    // Refresh r and p only for the RHS that paused and now resume.
    int refresh_skip[MAX_RHS];
    for (int q = 0; q < nrhs; q++) {
      const bool resumed = !skip_h[q] && !done[q];
      refresh_skip[q] = resumed ? 0 : 1;
      if (done[q]) h.halt[q] = h.halt_done[q] = 1;
    }
    CK(cudaMemcpyAsync(dskip, refresh_skip, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, st));
    CK(launch_axpby(sloppy, rS.ptr(), P64, r64.ptr(), P64, SpinorPtr{}, gg, sc2(nrhs, 1.0, 0.0), dskip, none, 0, st));
    {
      Reduce rpp = red_misc.r((double *)scal.p + MAX_RHS);
      CK(launch_axpby(sloppy, pS.ptr(), sloppy, rS.ptr(), sloppy, pS.ptr(), gg, beta, dskip, rpp, 1, st));
      double pp_h[MAX_RHS];
      CK(cudaMemcpyAsync(pp_h, (double *)scal.p + MAX_RHS, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      for (int q = 0; q < nrhs; q++)
        if (!refresh_skip[q]) h.pp[q] = pp_h[q];
    }
    // The device was idle since the state was read, so h is current for the RHS
    // that kept running and updated for the others.
    CK(cudaMemcpyAsync(state.p, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    *hstate = h;
  }
  // Final FP64 true residual (inv_cg.C:401-417).
  CgState h = *hstate;
  if (!opS) true_residual(rr, bnorm, st);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int q = 0; q < nrhs; q++) {
    res[q].iters = h.iters[q] + 1;
    res[q].true_rsd = bnorm[q] > 0 ? sqrt(rr[q] / bnorm[q]) : 0.0;
    res[q].iter_rsd = bnorm[q] > 0 ? sqrt(h.rr[q] / bnorm[q]) : 0.0;
    res[q].reliable_updates = nupd[q];
    res[q].seconds = secs;
    int stq = CPSB_OK;
    if (h.reason[q] == HALT_BREAKDOWN) stq = CPSB_ERR_BREAKDOWN;
    else if (!(rr[q] <= bnorm[q] * stop(q) * stop(q)) && h.reason[q] != HALT_CONVERGED) stq = CPSB_NOT_CONVERGED;
    else if (opS && !(rr[q] <= bnorm[q] * stop(q) * stop(q))) stq = CPSB_NOT_CONVERGED;
    res[q].status = stq;
    if (stq == CPSB_ERR_BREAKDOWN) status = stq;
    else if (stq == CPSB_NOT_CONVERGED && status == CPSB_OK) status = stq;
  }
  return status;
}

// One cached solver per (gauge, parameters, precision, nrhs).
struct SolverKey {
  Gauge *G;
  int action, ls, sloppy, nrhs, pc;
  double mass, m5, a5, b, c;
  double zb[128], zc[128];  // zMobius b_s, c_s (re, im) by value
  bool operator<(const SolverKey &o) const {
    return memcmp(this, &o, sizeof(SolverKey)) < 0;
  }
};
static std::map<SolverKey, std::unique_ptr<CgSolver>> &solvers() {
  static std::map<SolverKey, std::unique_ptr<CgSolver>> m;
  return m;
}
static std::mutex solvers_mu;

CgSolver *get_solver(Gauge *G, const cpsb_dirac_params &p, int sloppy, int nrhs) {
  SolverKey k;
  memset(&k, 0, sizeof(k));
  k.G = G;
  k.action = p.action;
  k.ls = p.action == CPSB_WILSON ? 1 : p.ls;
  k.sloppy = sloppy;
  k.nrhs = nrhs;
  k.pc = p.pc_type;
  k.mass = p.mass;
  k.m5 = p.m5;
  k.a5 = p.a5_inv;
  k.b = p.mobius_b;
  k.c = p.mobius_c;
  if (p.action == CPSB_ZMOBIUS)
    for (int i = 0; i < 2 * k.ls && i < 128; i++) {
      k.zb[i] = p.zmobius_b[i];
      k.zc[i] = p.zmobius_c[i];
    }
  std::lock_guard<std::mutex> lk(solvers_mu);
  auto &m = solvers();
  auto it = m.find(k);
  if (it != m.end()) return it->second.get();
  CgSolver *s = new CgSolver(G, p, sloppy, nrhs);
  m[k].reset(s);
  return s;
}

// Removes the cached solvers of G (cpsb_gauge_free).  Each one is destroyed only
// after its busy lock could be taken, so a solve still running on another host
// thread finishes first; no lock is held while waiting.  The cache keeps one
// solver per distinct (parameters, precision, nrhs) until its gauge is freed.
void drop_solvers(Gauge *G) {
  std::vector<std::unique_ptr<CgSolver>> gone;
  {
    std::lock_guard<std::mutex> lk(solvers_mu);
    auto &m = solvers();
    for (auto it = m.begin(); it != m.end();) {
      if (it->first.G == G) {
        gone.push_back(std::move(it->second));
        it = m.erase(it);
      } else {
        ++it;
      }
    }
  }
  for (auto &s : gone) {
    std::lock_guard<std::mutex> wait_for_solve(s->busy);
  }
}

}  // namespace cpsb

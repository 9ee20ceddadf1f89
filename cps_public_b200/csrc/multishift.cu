// multishift.cu -- multishift CG on MatPcDagMatPc (DiracOp::MInvCG).
//
// Restates cps_pp/src/util/dirac_op/d_op_base/noarch/minvcg.C:47-353 for the
// MULTI and SINGLE solve types: shift[0] is the base system, the other shifts
// follow through the z / bs recurrences, a shift stops being updated once
// c*z_s^2 < RsdCG_s^2 |chi|^2, and the reported residual is the iterated
// absolute one, sqrt(c z_s^2).  One iteration is three launch groups --
// MatPcDagMatPc on p_0 (its fused norm gives |M p_0|^2), the residual update
// whose last block advances every scalar recurrence, and one pass that updates
// all solutions and search directions while reading r once -- captured as a
// CUDA graph and replayed in batches.
//
// Several source vectors with the same shifts (the pseudofermions of an RHMC
// force or action evaluation, alg_action_rational.C:259-359) are solved
// together: every vector keeps its own scalar recurrences (MsBatch), the
// MatPcDagMatPc on p_0 is one multi-right-hand-side launch for all of them (one
// link read serves every vector), and the update kernels run one grid row per
// vector.  A vector whose shifts have all converged drops out of every launch
// through the operator's skip mask.
//
// With a reduced Krylov precision the vectors are FP32 (or 16-bit storage)
// and every shift is then refined by mixed-precision CG on (A + shift) to its
// own tolerance, checked with the FP64 true residual (all vectors of a shift
// in one multi-right-hand-side solve).
#include <math.h>
#include <string.h>

#include <chrono>

#include "host.h"
#include "ms_state.h"

namespace cpsb {

struct ShiftPtrs {
  SpinorPtr v[MAX_SHIFT];
};

// The scalar step of one vector after its residual update, with cnew = |r|^2
// and d = <p_0, (A + shift_0) p_0>: the initial step (minvcg.C:148-196) or
// iteration k (:224-254, 283-301) with the per-shift convergence checks, then
// the scalars of the next direction update (:206-222).
__device__ void ms_advance(MsState *S, double cnew, double d) {
  const int ns = S->nshift;
  const double cp = S->c;
  S->cp = cp;
  if (!(d != 0.0) || !isfinite(cnew)) {
    S->breakdown = 1;
    S->done = 1;
  } else if (S->k == 0) {
    const double b0 = -cp / d;
    S->b = b0;
    S->z[0][0] = 1.0;
    S->z[1][0] = 1.0;
    S->bs[0] = b0;
    S->iz = 1;
    for (int s = 1; s < ns; s++) {
      S->z[0][s] = 1.0;
      S->z[1][s] = 1.0 / (1.0 - b0 * (S->mass[s] - S->mass[0]));
      S->bs[s] = b0 * S->z[1][s];
    }
    S->c = cnew;
    for (int s = 0; s < ns; s++) S->conv_prev[s] = 0;
    if (cnew < S->rsd_sq[0]) S->done = 1;
  } else {
    const double a = S->a;
    S->bp = S->b;
    const double bp = S->bp;
    const double b1 = -cp / d;
    S->b = b1;
    S->bs[0] = b1;
    const int iz = 1 - S->iz;
    S->iz = iz;
    for (int s = 1; s < ns; s++) {
      if (S->conv[s]) continue;
      const double ztmp = S->z[1 - iz][s] * S->z[iz][s] * bp /
                          (b1 * a * (S->z[iz][s] - S->z[1 - iz][s]) +
                           S->z[iz][s] * bp * (1 - b1 * (S->mass[s] - S->mass[0])));
      S->bs[s] = b1 * ztmp / S->z[1 - iz][s];
      S->z[iz][s] = ztmp;
    }
    S->c = cnew;
    for (int s = 0; s < ns; s++) S->conv_prev[s] = S->conv[s];
    for (int s = 0; s < ns; s++) {
      if (S->conv[s]) continue;
      const double css = cnew * S->z[iz][s] * S->z[iz][s];
      if (css < S->rsd_sq[s]) {
        S->conv[s] = 1;
        S->css[s] = css;
        S->conv_iter[s] = S->k;
      }
    }
    int all = S->conv[0];
    if (all)
      for (int s = 0; s < ns; s++)
        if (!S->conv[s]) all = 0;
    if (all || S->k >= S->max_iter) S->done = 1;
  }
  S->k += 1;
  const double an = S->c / S->cp;
  S->a = an;
  const int iz = S->iz;
  for (int s = 1; s < ns; s++) S->as[s] = an * (S->z[iz][s] * S->bs[s]) / (S->z[1 - iz][s] * S->b);
}

// r = r + b (Ap + shift0 p0), b = -c/d; |r|^2; the last block advances the
// scalars.  Grid row y is vector y (entries [y n, (y+1) n)); the rows of
// finished vectors do no work but take part in the reduction's ticket.
template <int P, int NT>
__global__ void __launch_bounds__(NT) ms_r_update_kernel(Geom g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p0, MsBatch *B,
                                                         Reduce red) {
  typedef typename PrecTraits<P>::real T;
  __shared__ double sh[NT / 32];
  const int q = blockIdx.y;
  const MsState *S = &B->s[q];
  const long n = (long)g.n4cb * g.ls;
  double acc = 0;
  if (!B->done_applied[q]) {
    const double m0 = S->mass[0];
    const double d = B->d_mm[q] + m0 * S->pp;
    const T b = (T)(-S->c / d), tm0 = (T)m0;
    for (long j = (long)blockIdx.x * NT + threadIdx.x; j < n; j += (long)gridDim.x * NT) {
      const long i = q * n + j;
      Spinor<T> rv = load_spinor<P>(r, i);
      const Spinor<T> av = load_spinor<P>(Ap, i);
      if (m0 != 0.0) {
        const Spinor<T> pv = load_spinor<P>(p0, i);
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) rv.c[s][c] = cscale(b, av.c[s][c] + cscale(tm0, pv.c[s][c])) + rv.c[s][c];
      } else {
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) rv.c[s][c] = cscale(b, av.c[s][c]) + rv.c[s][c];
      }
      store_spinor<P>(r, i, rv);
      acc += norm2(rounded<P>(rv));
    }
  }
  const double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[q * gridDim.x + blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int v = 0; v < (int)gridDim.y; v++) {
      const double cnew = ordered_sum<NT>(red.partial + v * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0 && !B->done_applied[v]) {
        MsState *Sv = &B->s[v];
        ms_advance(Sv, cnew, B->d_mm[v] + Sv->mass[0] * Sv->pp);
      }
      __syncthreads();
    }
  }
}

// psi_s += -bs_s p_s (shifts not frozen at the start of the iteration), then
// the next directions p_0 = a p_0 + r, p_s = z_s r + as_s p_s; r read once.
// Grid row y is vector y; its last block sets done_applied after the update
// of the final iteration.
template <int P, int PX, int NT>
__global__ void __launch_bounds__(NT) ms_xp_update_kernel(Geom g, SpinorPtr r, ShiftPtrs p, ShiftPtrs psi, MsBatch *B,
                                                          Reduce red) {
  typedef typename PrecTraits<P>::real T;
  typedef typename PrecTraits<PX>::real TX;
  __shared__ double sh[NT / 32];
  const int q = blockIdx.y;
  const MsState *S = &B->s[q];
  const long n = (long)g.n4cb * g.ls;
  double acc = 0;
  if (!B->done_applied[q]) {
    const int ns = S->nshift;
    const bool single = S->type == 1;
    const bool done = S->done != 0;
    const int iz = S->iz;
    for (long j = (long)blockIdx.x * NT + threadIdx.x; j < n; j += (long)gridDim.x * NT) {
      const long i = q * n + j;
      const Spinor<T> rv = load_spinor<P>(r, i);
      Spinor<TX> x0;
      if (single) x0 = load_spinor<PX>(psi.v[0], i);
      for (int s = 0; s < ns; s++) {
        const bool upd_x = !S->conv_prev[s];
        const bool upd_p = !done && !S->conv[s];
        if (!upd_x && !upd_p) continue;
        Spinor<T> pv = load_spinor<P>(p.v[s], i);
        if (upd_x) {
          const double f = single ? -S->bs[s] * S->alpha[s] : -S->bs[s];
          const TX tf = (TX)f;
          Spinor<TX> xv = single ? x0 : load_spinor<PX>(psi.v[s], i);
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
              xv.c[a][c].re = tf * (TX)pv.c[a][c].re + xv.c[a][c].re;
              xv.c[a][c].im = tf * (TX)pv.c[a][c].im + xv.c[a][c].im;
            }
          if (single) x0 = xv;
          else store_spinor<PX>(psi.v[s], i, xv);
        }
        if (upd_p) {
          if (s == 0) {
            const T a = (T)S->a;
#pragma unroll
            for (int a4 = 0; a4 < 4; a4++)
#pragma unroll
              for (int c = 0; c < 3; c++) pv.c[a4][c] = cscale(a, pv.c[a4][c]) + rv.c[a4][c];
          } else {
            const T z = (T)S->z[iz][s], as = (T)S->as[s];
#pragma unroll
            for (int a4 = 0; a4 < 4; a4++)
#pragma unroll
              for (int c = 0; c < 3; c++) pv.c[a4][c] = cscale(z, rv.c[a4][c]) + cscale(as, pv.c[a4][c]);
          }
          store_spinor<P>(p.v[s], i, pv);
          if (s == 0) acc += norm2(rounded<P>(pv));
        }
      }
      if (single) store_spinor<PX>(psi.v[0], i, x0);
    }
  }
  const double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[q * gridDim.x + blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int v = 0; v < (int)gridDim.y; v++) {
      const double pp = ordered_sum<NT>(red.partial + v * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0 && !B->done_applied[v]) {
        MsState *Sv = &B->s[v];
        if (!Sv->conv[0]) Sv->pp = pp;
        if (Sv->done) B->done_applied[v] = 1;
      }
      __syncthreads();
    }
  }
}

static int ms_blocks(long n) {
  long nb = (n + 255) / 256;
  if (nb > 148L * 8) nb = 148L * 8;
  return (int)(nb < 1 ? 1 : nb);
}

// g: the geometry of all vectors (g.nrhs of them, one grid row each).
cudaError_t launch_ms_r_update(int prec, const Geom &g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p0, MsBatch *B,
                               Reduce red, cudaStream_t st) {
  const dim3 grid(ms_blocks((long)g.n4cb * g.ls), g.nrhs);
  if (prec == P64) ms_r_update_kernel<P64, 256><<<grid, 256, 0, st>>>(g, r, Ap, p0, B, red);
  else if (prec == P32) ms_r_update_kernel<P32, 256><<<grid, 256, 0, st>>>(g, r, Ap, p0, B, red);
  else ms_r_update_kernel<P16, 256><<<grid, 256, 0, st>>>(g, r, Ap, p0, B, red);
  return launched();
}

cudaError_t launch_ms_xp_update(int prec, int px, const Geom &g, SpinorPtr r, const ShiftPtrs &p, const ShiftPtrs &psi,
                                MsBatch *B, Reduce red, cudaStream_t st) {
  const dim3 grid(ms_blocks((long)g.n4cb * g.ls), g.nrhs);
  if (prec == P64 && px == P64) ms_xp_update_kernel<P64, P64, 256><<<grid, 256, 0, st>>>(g, r, p, psi, B, red);
  else if (prec == P32 && px == P32) ms_xp_update_kernel<P32, P32, 256><<<grid, 256, 0, st>>>(g, r, p, psi, B, red);
  else if (prec == P16 && px == P32) ms_xp_update_kernel<P16, P32, 256><<<grid, 256, 0, st>>>(g, r, p, psi, B, red);
  else return cudaErrorInvalidValue;
  return launched();
}

}  // namespace cpsb

namespace cpsb {

namespace {
Scal2 scal_all(double a, double b) {
  Scal2 s;
  for (int i = 0; i < MAX_RHS; i++) {
    s.a[i] = a;
    s.b[i] = b;
  }
  return s;
}
}  // namespace

// nvec source vectors solved together.  chi: nvec x n FP64 (packed, vector q at
// entries [q n, (q+1) n)); x: outputs, FP64 fields of nvec x n, nshift of them
// for MULTI, one for SINGLE; rsd[q * nshift + s]: stop_rsd of shift s for
// vector q on entry, its reported residual on return; res[q]: the report of
// vector q (iters: CPS's iteration count of its Krylov phase plus, with
// refinement, the refinement iterations).
int multishift_multi(Gauge *G, const cpsb_dirac_params &p, const cpsb_cg_arg &a, int nvec, Field &chi,
                     std::vector<Field> &x, const double *shift, int nshift, double *rsd, int type,
                     const double *alpha, cpsb_solve_result *res, cudaStream_t st, CgSolver *refiner) {
  auto t0 = std::chrono::steady_clock::now();
  if (nshift < 1 || nshift > MAX_SHIFT) throw Error{CPSB_ERR_ARG, "nshift must be in [1, 32]"};
  if (nvec < 1 || nvec > MAX_RHS) throw Error{CPSB_ERR_ARG, "nvec must be in [1, 16]"};
  for (int s = 1; s < nshift; s++)
    if (shift[s] < shift[0]) throw Error{CPSB_ERR_ARG, "shift[0] must be the smallest shift (minvcg.C:141-165)"};
  if (refiner && refiner->nrhs != nvec) throw Error{CPSB_ERR_ARG, "refinement solver of the wrong width"};
  const int prec = a.precision;
  const bool refine = prec != P64;
  const int ktype = refine ? 0 : type;  // sloppy SINGLE runs as MULTI and combines after refinement
  Operator op(G, p, prec, nvec);
  const Geom &g = op.geom;
  const long n = g.nsites;       // all vectors
  const long n1 = n / nvec;      // one vector
  const int px = prec == P64 ? P64 : P32;
  Field r(prec, n), Ap(prec, n);
  std::vector<Field> pv(nshift);
  const int nx = ktype == 1 ? 1 : nshift;
  std::vector<Field> psi(nx);
  for (int s = 0; s < nshift; s++) pv[s].create(prec, n);
  for (int s = 0; s < nx; s++) {
    psi[s].create(px, n);
    CK(cudaMemsetAsync(psi[s].data.p, 0, psi[s].data.bytes, st));
  }
  RedSlot red_d, red_r, red_p, red_m;
  DevBuf dres(sizeof(double) * MAX_RHS);
  // |chi_q|^2 (FmatEvlMInv's NormSqGlbSum, f_dwf_base.C:248)
  double chi_norm[MAX_RHS];
  CK(launch_redot(P64, g, chi.ptr(), chi.ptr(), red_m.r((double *)dres.p), st));
  CK(cudaMemcpyAsync(chi_norm, dres.p, sizeof(double) * nvec, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(launch_convert(prec, r.ptr(), P64, chi.ptr(), n, st));
  for (int s = 0; s < nshift; s++) {
    CK(cudaMemcpyAsync(pv[s].data.p, r.data.p, r.data.bytes, cudaMemcpyDeviceToDevice, st));
    if (r.norm.p) CK(cudaMemcpyAsync(pv[s].norm.p, r.norm.p, r.norm.bytes, cudaMemcpyDeviceToDevice, st));
  }
  // Krylov tolerance: the requested one in FP64; with reduced precision the
  // shifts are refined afterwards, so the Krylov phase stops at a floor (FP32:
  // 1e-8 -- the iterated residual keeps falling there, and each shift's
  // refinement then starts closer: 655 iterations in total on the 24^3x64
  // Ls 12 twelve-shift workload against 825 with a 1e-6 floor).
  const double floor_rsd = prec == P64 ? 0.0 : (prec == P32 ? 1e-8 : 1e-4);
  MsBatch *hb = nullptr;
  CK(cudaMallocHost((void **)&hb, sizeof(MsBatch)));
  struct PinGuard {
    MsBatch *p;
    ~PinGuard() { cudaFreeHost(p); }
  } pin_guard{hb};
  memset(hb, 0, sizeof(MsBatch));
  hb->nvec = nvec;
  bool any = false;
  for (int q = 0; q < nvec; q++) {
    MsState &hs = hb->s[q];
    hs.c = chi_norm[q];
    hs.pp = chi_norm[q];
    hs.nshift = nshift;
    hs.type = ktype;
    hs.max_iter = a.max_num_iter;
    for (int s = 0; s < nshift; s++) {
      hs.mass[s] = shift[s];
      const double rq = rsd[q * nshift + s];
      const double rr = rq > floor_rsd ? rq : floor_rsd;
      hs.rsd_sq[s] = chi_norm[q] * (rr * rr);
      hs.alpha[s] = alpha ? alpha[s] : 1.0;
    }
    // a zero source (or no iterations) is done before the first iteration
    const bool idle = !(chi_norm[q] > 0) || a.max_num_iter <= 0;
    hb->done_applied[q] = idle ? 1 : 0;
    any |= !idle;
  }
  const MsBatch init = *hb;
  DevBuf state(sizeof(MsBatch));
  MsBatch *B = (MsBatch *)state.p;
  CK(cudaMemcpyAsync(state.p, &init, sizeof(MsBatch), cudaMemcpyHostToDevice, st));
  ShiftPtrs pp_, xx_;
  memset(&pp_, 0, sizeof(pp_));
  memset(&xx_, 0, sizeof(xx_));
  for (int s = 0; s < nshift; s++) pp_.v[s] = pv[s].ptr();
  for (int s = 0; s < nx; s++) xx_.v[s] = psi[s].ptr();
  if (any) {
    Reduce rd = red_d.r(B->d_mm), rr = red_r.r(nullptr), rp = red_p.r(nullptr);
    const int *skip = B->done_applied;
    op.mdagm(Ap, pv[0], &rd, skip, st);  // uncaptured application: tunes the launch shapes
    CK(cudaMemcpyAsync(state.p, &init, sizeof(MsBatch), cudaMemcpyHostToDevice, st));
    const int batch = a.batch > 0 ? a.batch : (graph_loops_enabled() ? 4 : 16);
    auto record = [&]() {
      for (int j = 0; j < batch; j++) {
        op.mdagm(Ap, pv[0], &rd, skip, st);
        CK(launch_ms_r_update(prec, g, r.ptr(), Ap.ptr(), pv[0].ptr(), B, rr, st));
        CK(launch_ms_xp_update(prec, px, g, r.ptr(), pp_, xx_, B, rp, st));
      }
    };
    // one graph launch runs batches on the device until every vector is done
    // (graph_loop.cu); else the host replays single batches
    DevBuf loopbuf(sizeof(LoopCtl));
    LoopCtl *hl = nullptr;
    CK(cudaMallocHost((void **)&hl, 2 * sizeof(LoopCtl)));
    struct LoopPin {
      LoopCtl *p;
      ~LoopPin() { cudaFreeHost(p); }
    } loop_pin{hl};
    cudaGraphExec_t exec = nullptr;
    size_t nn = 0;
    const bool as_loop = graph_loops_enabled() &&
                         build_loop_graph(st, [&](cudaGraphConditionalHandle h) {
                           record();
                           CK(launch_ms_loop_cond(h, B, (LoopCtl *)loopbuf.p, nvec, st));
                         }, &exec, &nn);
    if (!as_loop) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      set_capturing(true);
      try {
        record();
      } catch (...) {
        set_capturing(false);
        cudaStreamEndCapture(st, &graph);
        throw;
      }
      set_capturing(false);
      CK(cudaStreamEndCapture(st, &graph));
      CK(cudaGraphGetNodes(graph, nullptr, &nn));
      CK(cudaGraphInstantiate(&exec, graph, 0));
      cudaGraphDestroy(graph);
    }
    struct ExecGuard {
      cudaGraphExec_t e;
      ~ExecGuard() { cudaGraphExecDestroy(e); }
    } exec_guard{exec};
    for (;;) {
      if (as_loop) {
        hl[0].count = 0;
        hl[0].cap = (unsigned)((a.max_num_iter + batch - 1) / batch + 2);
        CK(cudaMemcpyAsync(loopbuf.p, &hl[0], sizeof(LoopCtl), cudaMemcpyHostToDevice, st));
      }
      CK(cudaGraphLaunch(exec, st));
      CK(cudaMemcpyAsync(hb, state.p, sizeof(MsBatch), cudaMemcpyDeviceToHost, st));
      if (as_loop) CK(cudaMemcpyAsync(&hl[1], loopbuf.p, sizeof(LoopCtl), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      count_launch(nn * (as_loop ? hl[1].count : 1));
      bool all = true;
      for (int q = 0; q < nvec; q++) all &= hb->done_applied[q] != 0;
      if (all) break;
    }
  }
  const MsBatch h = *hb;
  // Residuals as MInvCG reports them (minvcg.C:306-326); a vector that never
  // iterated reports its initial state (k = 0).
  std::vector<double> ms_rsd((size_t)nvec * nshift);
  int status[MAX_RHS], total_iters[MAX_RHS], nupd[MAX_RHS];
  for (int q = 0; q < nvec; q++) {
    const MsState &hq = h.s[q];
    for (int s = 0; s < nshift; s++)
      ms_rsd[q * nshift + s] = hq.conv[s] ? sqrt(hq.css[s]) : sqrt(hq.c * hq.z[hq.iz][s] * hq.z[hq.iz][s]);
    status[q] = hq.breakdown ? CPSB_ERR_BREAKDOWN : CPSB_OK;
    total_iters[q] = hq.k;
    nupd[q] = 0;
  }
  if (!refine) {
    for (int s = 0; s < nx; s++) CK(launch_convert(P64, x[s].ptr(), px, psi[s].ptr(), n, st));
    for (int q = 0; q < nvec; q++)
      for (int s = 0; s < nshift; s++) {
        rsd[q * nshift + s] = ms_rsd[q * nshift + s];
        if (!h.s[q].conv[s] && status[q] >= 0) status[q] = CPSB_NOT_CONVERGED;
      }
  } else {
    // Refine every shift with mixed-precision CG on (A + shift_s) to its own
    // tolerance, checked with the FP64 true residual: one solve over all
    // vectors per shift, each vector to its own stop_rsd.
    CgSolver *cg = refiner ? refiner : get_solver(G, p, prec, nvec);
    std::unique_lock<std::mutex> lk(cg->busy, std::defer_lock);
    if (!refiner) lk.lock();  // the cached solver may be shared between threads
    CK(launch_convert(P64, cg->b64.ptr(), P64, chi.ptr(), n, st));
    for (int s = 0; s < nshift; s++) {
      CK(launch_convert(P64, cg->x64.ptr(), px, psi[s].ptr(), n, st));
      double stop_q[MAX_RHS];
      for (int q = 0; q < nvec; q++) stop_q[q] = rsd[q * nshift + s];
      cpsb_solve_result rs[MAX_RHS];
      const int rc = cg->solve(a, rs, st, shift[s], stop_q);
      (void)rc;
      for (int q = 0; q < nvec; q++) {
        total_iters[q] += rs[q].iters - 1;
        nupd[q] += rs[q].reliable_updates;
        rsd[q * nshift + s] = rs[q].true_rsd;
        if (rs[q].status < 0) status[q] = rs[q].status;
        else if (rs[q].status == CPSB_NOT_CONVERGED && status[q] == CPSB_OK) status[q] = CPSB_NOT_CONVERGED;
      }
      if (type == 1) {
        Reduce none;
        memset(&none, 0, sizeof(none));
        const double al = alpha ? alpha[s] : 1.0;
        if (s == 0) CK(launch_axpby(P64, x[0].ptr(), P64, cg->x64.ptr(), P64, SpinorPtr{}, g, scal_all(al, 0.0),
                                    nullptr, none, 0, st));
        else CK(launch_axpby(P64, x[0].ptr(), P64, x[0].ptr(), P64, cg->x64.ptr(), g, scal_all(1.0, al), nullptr,
                             none, 0, st));
      } else {
        CK(cudaMemcpyAsync(x[s].data.p, cg->x64.data.p, x[s].data.bytes, cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  CK(cudaStreamSynchronize(st));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int worst = CPSB_OK;
  for (int q = 0; q < nvec; q++) {
    if (res) {
      cpsb_solve_result &o = res[q];
      o.iters = total_iters[q];
      o.true_rsd = 0;
      for (int s = 0; s < nshift; s++) o.true_rsd = rsd[q * nshift + s] > o.true_rsd ? rsd[q * nshift + s] : o.true_rsd;
      o.iter_rsd = ms_rsd[q * nshift];
      o.reliable_updates = nupd[q];
      o.seconds = secs;
      o.status = status[q];
    }
    if (status[q] < 0) worst = worst < 0 ? worst : status[q];
    else if (status[q] == CPSB_NOT_CONVERGED && worst == CPSB_OK) worst = CPSB_NOT_CONVERGED;
  }
  (void)n1;
  return worst;
}

int multishift(Gauge *G, const cpsb_dirac_params &p, const cpsb_cg_arg &a, Field &chi, std::vector<Field> &x,
               const double *shift, int nshift, double *rsd, int type, const double *alpha, cpsb_solve_result *res,
               cudaStream_t st, CgSolver *refiner) {
  return multishift_multi(G, p, a, 1, chi, x, shift, nshift, rsd, type, alpha, res, st, refiner);
}

}  // namespace cpsb

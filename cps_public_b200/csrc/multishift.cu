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
// With a reduced Krylov precision the vectors are FP32 (or 16-bit storage)
// and every shift is then refined by mixed-precision CG on (A + shift) to its
// own tolerance, checked with the FP64 true residual.
#include <math.h>
#include <string.h>

#include <chrono>

#include "host.h"
#include "ms_state.h"

namespace cpsb {

struct ShiftPtrs {
  SpinorPtr v[MAX_SHIFT];
};

// r = r + b (Ap + shift0 p0), b = -c/d; |r|^2; the last block advances the scalars.
template <int P, int NT>
__global__ void __launch_bounds__(NT) ms_r_update_kernel(Geom g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p0, MsState *S,
                                                         Reduce red) {
  typedef typename PrecTraits<P>::real T;
  __shared__ double sh[NT / 32];
  if (S->done_applied) return;
  const long n = g.nsites;
  const double m0 = S->mass[0];
  const double d = S->d_mm + m0 * S->pp;
  const double bnew = -S->c / d;
  const T b = (T)bnew, tm0 = (T)m0;
  double acc = 0;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) {
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
  const double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x)) {
    const double cnew = ordered_sum<NT>(red.partial, gridDim.x, sh);
    if (threadIdx.x == 0) {
      const int ns = S->nshift;
      const double cp = S->c;
      S->cp = cp;
      if (!(d != 0.0) || !isfinite(cnew)) {
        S->breakdown = 1;
        S->done = 1;
      } else if (S->k == 0) {
        // initial step (minvcg.C:148-196)
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
        // iteration k (minvcg.C:224-254, 283-301)
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
      // scalars of the next direction update (minvcg.C:206-222)
      const double an = S->c / S->cp;
      S->a = an;
      const int iz = S->iz;
      for (int s = 1; s < ns; s++) S->as[s] = an * (S->z[iz][s] * S->bs[s]) / (S->z[1 - iz][s] * S->b);
    }
  }
}

// psi_s += -bs_s p_s (shifts not frozen at the start of the iteration), then
// the next directions p_0 = a p_0 + r, p_s = z_s r + as_s p_s; r read once.
template <int P, int PX, int NT>
__global__ void __launch_bounds__(NT) ms_xp_update_kernel(Geom g, SpinorPtr r, ShiftPtrs p, ShiftPtrs psi, MsState *S,
                                                          Reduce red) {
  typedef typename PrecTraits<P>::real T;
  typedef typename PrecTraits<PX>::real TX;
  __shared__ double sh[NT / 32];
  if (S->done_applied) return;
  const long n = g.nsites;
  const int ns = S->nshift;
  const bool single = S->type == 1;
  const bool done = S->done != 0;
  const int iz = S->iz;
  double acc = 0;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) {
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
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int c = 0; c < 3; c++) pv.c[q][c] = cscale(a, pv.c[q][c]) + rv.c[q][c];
        } else {
          const T z = (T)S->z[iz][s], as = (T)S->as[s];
#pragma unroll
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int c = 0; c < 3; c++) pv.c[q][c] = cscale(z, rv.c[q][c]) + cscale(as, pv.c[q][c]);
        }
        store_spinor<P>(p.v[s], i, pv);
        if (s == 0) acc += norm2(rounded<P>(pv));
      }
    }
    if (single) store_spinor<PX>(psi.v[0], i, x0);
  }
  const double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x)) {
    const double pp = ordered_sum<NT>(red.partial, gridDim.x, sh);
    if (threadIdx.x == 0) {
      if (!S->conv[0]) S->pp = pp;
      if (S->done) S->done_applied = 1;
    }
  }
}

static int ms_blocks(long n) {
  long nb = (n + 255) / 256;
  if (nb > 148L * 8) nb = 148L * 8;
  return (int)(nb < 1 ? 1 : nb);
}

cudaError_t launch_ms_r_update(int prec, const Geom &g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p0, MsState *S,
                               Reduce red, cudaStream_t st) {
  const int nb = ms_blocks(g.nsites);
  if (prec == P64) ms_r_update_kernel<P64, 256><<<nb, 256, 0, st>>>(g, r, Ap, p0, S, red);
  else if (prec == P32) ms_r_update_kernel<P32, 256><<<nb, 256, 0, st>>>(g, r, Ap, p0, S, red);
  else ms_r_update_kernel<P16, 256><<<nb, 256, 0, st>>>(g, r, Ap, p0, S, red);
  return launched();
}

cudaError_t launch_ms_xp_update(int prec, int px, const Geom &g, SpinorPtr r, const ShiftPtrs &p, const ShiftPtrs &psi,
                                MsState *S, Reduce red, cudaStream_t st) {
  const int nb = ms_blocks(g.nsites);
  if (prec == P64 && px == P64) ms_xp_update_kernel<P64, P64, 256><<<nb, 256, 0, st>>>(g, r, p, psi, S, red);
  else if (prec == P32 && px == P32) ms_xp_update_kernel<P32, P32, 256><<<nb, 256, 0, st>>>(g, r, p, psi, S, red);
  else if (prec == P16 && px == P32) ms_xp_update_kernel<P16, P32, 256><<<nb, 256, 0, st>>>(g, r, p, psi, S, red);
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

// chi: FP64 source (packed); x: outputs (FP64 fields, nshift of them for MULTI,
// one for SINGLE).  Returns the CPS iteration count in res->iters.
int multishift(Gauge *G, const cpsb_dirac_params &p, const cpsb_cg_arg &a, Field &chi, std::vector<Field> &x,
               const double *shift, int nshift, double *rsd, int type, const double *alpha, cpsb_solve_result *res,
               cudaStream_t st, CgSolver *refiner) {
  auto t0 = std::chrono::steady_clock::now();
  if (nshift < 1 || nshift > MAX_SHIFT) throw Error{CPSB_ERR_ARG, "nshift must be in [1, 32]"};
  for (int s = 1; s < nshift; s++)
    if (shift[s] < shift[0]) throw Error{CPSB_ERR_ARG, "shift[0] must be the smallest shift (minvcg.C:141-165)"};
  const int prec = a.precision;
  const bool refine = prec != P64;
  const int ktype = refine ? 0 : type;  // sloppy SINGLE runs as MULTI and combines after refinement
  Operator op(G, p, prec, 1);
  const Geom &g = op.geom;
  const long n = g.nsites;
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
  DevBuf dres(sizeof(double) * 4);
  // |chi|^2 (FmatEvlMInv's NormSqGlbSum, f_dwf_base.C:248)
  double chi_norm = 0;
  CK(launch_redot(P64, g, chi.ptr(), chi.ptr(), red_m.r((double *)dres.p), st));
  CK(cudaMemcpyAsync(&chi_norm, dres.p, sizeof(double), cudaMemcpyDeviceToHost, st));
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
  MsState hs;
  memset(&hs, 0, sizeof(hs));
  hs.c = chi_norm;
  hs.pp = chi_norm;
  hs.nshift = nshift;
  hs.type = ktype;
  hs.max_iter = a.max_num_iter;
  for (int s = 0; s < nshift; s++) {
    hs.mass[s] = shift[s];
    const double rr = rsd[s] > floor_rsd ? rsd[s] : floor_rsd;
    hs.rsd_sq[s] = chi_norm * (rr * rr);
    hs.alpha[s] = alpha ? alpha[s] : 1.0;
  }
  DevBuf state(sizeof(MsState));
  MsState *S = (MsState *)state.p;
  MsState *hst = nullptr;
  CK(cudaMallocHost((void **)&hst, sizeof(MsState)));
  struct PinGuard {
    MsState *p;
    ~PinGuard() { cudaFreeHost(p); }
  } pin_guard{hst};
  CK(cudaMemcpyAsync(state.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st));
  ShiftPtrs pp_, xx_;
  memset(&pp_, 0, sizeof(pp_));
  memset(&xx_, 0, sizeof(xx_));
  for (int s = 0; s < nshift; s++) pp_.v[s] = pv[s].ptr();
  for (int s = 0; s < nx; s++) xx_.v[s] = psi[s].ptr();
  if (chi_norm > 0 && a.max_num_iter > 0) {
    Reduce rd = red_d.r(&S->d_mm), rr = red_r.r(nullptr), rp = red_p.r(nullptr);
    const int *skip = &S->done_applied;
    op.mdagm(Ap, pv[0], &rd, skip, st);  // uncaptured application: tunes the launch shapes
    CK(cudaMemcpyAsync(state.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st));
    const int batch = a.batch > 0 ? a.batch : 16;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try {
      for (int j = 0; j < batch; j++) {
        op.mdagm(Ap, pv[0], &rd, skip, st);
        CK(launch_ms_r_update(prec, g, r.ptr(), Ap.ptr(), pv[0].ptr(), S, rr, st));
        CK(launch_ms_xp_update(prec, px, g, r.ptr(), pp_, xx_, S, rp, st));
      }
    } catch (...) {
      set_capturing(false);
      cudaStreamEndCapture(st, &graph);
      throw;
    }
    set_capturing(false);
    CK(cudaStreamEndCapture(st, &graph));
    size_t nn = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &nn));
    cudaGraphExec_t exec;
    CK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    struct ExecGuard {
      cudaGraphExec_t e;
      ~ExecGuard() { cudaGraphExecDestroy(e); }
    } exec_guard{exec};
    for (;;) {
      CK(cudaGraphLaunch(exec, st));
      count_launch(nn);
      CK(cudaMemcpyAsync(hst, state.p, sizeof(MsState), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (hst->done_applied) break;
    }
  } else {
    memcpy(hst, &hs, sizeof(hs));
    hst->k = 0;
  }
  const MsState h = *hst;
  // Residuals as MInvCG reports them (minvcg.C:306-326)
  std::vector<double> ms_rsd(nshift);
  for (int s = 0; s < nshift; s++)
    ms_rsd[s] = h.conv[s] ? sqrt(h.css[s]) : sqrt(h.c * h.z[h.iz][s] * h.z[h.iz][s]);
  int status = h.breakdown ? CPSB_ERR_BREAKDOWN : CPSB_OK;
  int total_iters = h.k;
  int nupd = 0;
  if (!refine) {
    for (int s = 0; s < nx; s++) CK(launch_convert(P64, x[s].ptr(), px, psi[s].ptr(), n, st));
    for (int s = 0; s < nshift; s++) {
      rsd[s] = ms_rsd[s];
      if (!h.conv[s]) status = status < 0 ? status : CPSB_NOT_CONVERGED;
    }
  } else {
    // Refine every shift with mixed-precision CG on (A + shift_s) to its own
    // tolerance, checked with the FP64 true residual.
    CgSolver *cg = refiner ? refiner : get_solver(G, p, prec, 1);
    std::unique_lock<std::mutex> lk(cg->busy, std::defer_lock);
    if (!refiner) lk.lock();  // the cached solver may be shared between threads
    CK(launch_convert(P64, cg->b64.ptr(), P64, chi.ptr(), n, st));
    for (int s = 0; s < nshift; s++) {
      CK(launch_convert(P64, cg->x64.ptr(), px, psi[s].ptr(), n, st));
      cpsb_cg_arg ca = a;
      ca.stop_rsd = rsd[s];
      cpsb_solve_result rs;
      const int rc = cg->solve(ca, &rs, st, shift[s]);
      total_iters += rs.iters - 1;
      nupd += rs.reliable_updates;
      rsd[s] = rs.true_rsd;
      if (rc < 0) status = rc;
      else if (rc == CPSB_NOT_CONVERGED && status == CPSB_OK) status = rc;
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
  if (res) {
    res->iters = total_iters;
    res->true_rsd = 0;
    for (int s = 0; s < nshift; s++) res->true_rsd = rsd[s] > res->true_rsd ? rsd[s] : res->true_rsd;
    res->iter_rsd = ms_rsd[0];
    res->reliable_updates = nupd;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->status = status;
  }
  return status;
}

}  // namespace cpsb

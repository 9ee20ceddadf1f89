// serve.cu -- the request loop (cpsb_serve_*): concurrent CG solves of
// differing lattice, Ls, mass, tolerance and right-hand-side count against
// gauge fields that stay resident on the device.
//
// CPS solves one system at a time (DiracOp::scope_lock, cps_pp/src/util/
// dirac_op/d_op_base/comsrc/dirac_op_base.C:26,112-118); this loop is the
// device-side replacement for a caller that issues many FmatEvlInv solves
// (lattice.h:942).  Design:
//
//  * A request (nrhs right-hand sides of one system) is split into work items
//    of at most g right-hand sides, g the largest group whose device footprint
//    fits the server's HBM budget; a request whose single right-hand side does
//    not fit is refused at submission (CPSB_ERR_OOM).
//  * `slots` worker threads, each with its own non-blocking CUDA stream, take
//    work items in arrival order as soon as a slot is free and the item's
//    footprint fits the budget still unreserved (admission by free HBM).  A
//    smaller item may overtake one that does not fit; after 4*slots such
//    overtakes the oldest item is served next (no starvation).
//  * Each item runs the multi-RHS CG of solver.cu on its own workspace, so
//    work of different requests overlaps on the device and a request's
//    arithmetic is the same whether it runs alone or in a mix: the result
//    depends only on the request (and on the launch shapes the autotuner has
//    cached for its operator shapes).
//  * Multishift requests (cpsb_serve_submit_minvcg, DiracOp::MInvCG as the
//    RHMC pseudofermion and pole solves issue them) are one work item each with
//    their own refinement solver, so the solves of many pseudofermions overlap.
//  * Latency is host time from submission to the completion of the last item.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "abi.h"

using namespace cpsb;

namespace cpsb {

static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Device bytes a CgSolver for nrhs right-hand sides of n sites each holds,
// plus the one-vector CPS-order FP64 staging buffer of the work item.
static size_t solve_footprint(const cpsb_dirac_params &p, long n, int sloppy, int nrhs) {
  const long N = n * nrhs;
  const int op_tmp = p.action >= CPSB_MOBIUS ? 3 : 2;   // Operator::t1, t2 (t3 for Mobius / zMobius)
  size_t b = field_bytes(P64, N) * 3 + field_bytes(P64, n);  // x, b, r; staging
  if (sloppy == P64) {
    b += field_bytes(P64, N) * (3 + op_tmp);             // r, p, Ap; temporaries of the FP64 operator
  } else {
    b += field_bytes(P64, n) * op_tmp;                   // one-RHS FP64 operator (true residuals)
    b += field_bytes(sloppy, N) * (3 + op_tmp) + field_bytes(P32, N);  // r, p, Ap, temporaries; x
  }
  return b + (size_t)(8u << 20);                         // reduction slots, state, graph
}

// Device bytes of one multishift solve (multishift.cu): FP64 source and
// solutions, Krylov vectors in the Krylov precision, the operator's
// temporaries, and the one-RHS refinement solver of reduced-precision runs.
static size_t multishift_footprint(const cpsb_dirac_params &p, long n, int prec, int nshift, int nvec) {
  const int op_tmp = p.action >= CPSB_MOBIUS ? 3 : 2;
  const int px = prec == P64 ? P64 : P32;
  size_t b = field_bytes(P64, n) * (2 + nvec);                        // chi, staging, x[s]
  b += field_bytes(prec, n) * (2 + nshift + op_tmp) + field_bytes(px, n) * nshift;  // r, Ap, p_s, temps; psi_s
  if (prec != P64) b += solve_footprint(p, n, prec, 1);
  return b + (size_t)(8u << 20);
}

struct ServeRequest {
  unsigned long long id = 0;
  cpsb_gauge h = nullptr;
  cpsb_dirac_params p;
  std::vector<double> zb, zc;  // zMobius coefficients owned by the request (p points here)
  cpsb_cg_arg a;
  int nrhs = 0;
  std::vector<double *> x;
  std::vector<const double *> b;
  std::vector<cpsb_solve_result> res;
  // multishift requests (DiracOp::MInvCG): shifts, per-shift tolerances in and
  // reported residuals out, type and weights
  bool multishift = false;
  std::vector<double> shift, alpha;
  double *rsd = nullptr;
  int ms_type = CPSB_MULTI;
  int items_left = 0;
  int status = CPSB_OK;
  std::string err;
  double t_submit = 0, t_done = 0;
  bool done = false;
};

struct ServeItem {
  ServeRequest *req;
  int rhs0, nrhs;
  size_t bytes;
};

struct Server {
  int device = 0;
  size_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServeItem> queue;
  std::map<unsigned long long, std::unique_ptr<ServeRequest>> reqs;
  std::vector<std::thread> workers;
  unsigned long long next_id = 1;
  size_t reserved = 0, peak_reserved = 0;
  int running = 0, peak_running = 0, slots = 0, head_skips = 0;
  bool stopping = false;
  // statistics of completed requests
  std::vector<double> lat_ms;
  long completed = 0, failed = 0, rhs_done = 0;
  double t_first_submit = -1, t_last_done = 0;

  void worker_main();
  bool pick(ServeItem *out);
  void run_item(const ServeItem &it, cudaStream_t st);
};

// Chooses the next item under mu: the oldest that fits, or -- after too many
// overtakes -- only the oldest.
bool Server::pick(ServeItem *out) {
  for (size_t i = 0; i < queue.size(); i++) {
    if (i > 0 && head_skips >= 4 * slots) break;
    if (reserved + queue[i].bytes <= budget) {
      *out = queue[i];
      if (i == 0) head_skips = 0;
      else head_skips++;
      queue.erase(queue.begin() + (long)i);
      return true;
    }
  }
  return false;
}

// One work item: pack the item's right-hand sides and guesses, solve, unpack.
void Server::run_item(const ServeItem &it, cudaStream_t st) {
  ServeRequest &r = *it.req;
  Gauge *G = &r.h->g;
  const long n = cb_sites(r.h, &r.p);
  const Geom g1 = geom_of(r.h, &r.p, 1);
  const size_t each = (size_t)n * 24 * sizeof(double);
  if (r.multishift) {
    const int nshift = (int)r.shift.size();
    const int nvec = r.ms_type == CPSB_SINGLE ? 1 : nshift;
    Field chi(P64, n);
    DevBuf stage(each);
    CK(cudaMemcpyAsync(stage.p, r.b[0], each, cudaMemcpyHostToDevice, st));
    CK(launch_pack(P64, chi.ptr(), (const double *)stage.p, g1, st));
    std::vector<Field> xs(nvec);
    for (int i = 0; i < nvec; i++) {
      xs[i].create(P64, n);
      CK(cudaMemsetAsync(xs[i].data.p, 0, xs[i].data.bytes, st));
    }
    // a private refinement solver: concurrent requests do not queue on the cached one
    std::unique_ptr<CgSolver> refiner;
    if (r.a.precision != P64) refiner.reset(new CgSolver(G, r.p, r.a.precision, 1));
    const int rc = multishift(G, r.p, r.a, chi, xs, r.shift.data(), nshift, r.rsd, r.ms_type,
                              r.alpha.empty() ? nullptr : r.alpha.data(), r.res.data(), st, refiner.get());
    for (int i = 0; i < nvec; i++) {
      CK(launch_unpack(P64, (double *)stage.p, xs[i].ptr(), g1, st));
      CK(cudaMemcpyAsync(r.x[i], stage.p, each, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    if (rc != CPSB_OK) throw Error{rc, "multishift solve did not converge"};
    return;
  }
  CgSolver s(G, r.p, r.a.precision, it.nrhs);
  DevBuf stage(each);
  for (int q = 0; q < it.nrhs; q++) {
    CK(cudaMemcpyAsync(stage.p, r.x[it.rhs0 + q], each, cudaMemcpyHostToDevice, st));
    CK(launch_pack(P64, s.x64.view((long)q * n), (const double *)stage.p, g1, st));
    CK(cudaMemcpyAsync(stage.p, r.b[it.rhs0 + q], each, cudaMemcpyHostToDevice, st));
    CK(launch_pack(P64, s.b64.view((long)q * n), (const double *)stage.p, g1, st));
  }
  const int rc = s.solve(r.a, r.res.data() + it.rhs0, st);
  for (int q = 0; q < it.nrhs; q++) {
    CK(launch_unpack(P64, (double *)stage.p, s.x64.view((long)q * n), g1, st));
    CK(cudaMemcpyAsync(r.x[it.rhs0 + q], stage.p, each, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  if (rc != CPSB_OK) throw Error{rc, "solve did not converge"};
}

void Server::worker_main() {
  cudaSetDevice(device);
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) st = nullptr;
  for (;;) {
    ServeItem it{nullptr, 0, 0, 0};
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return (stopping && queue.empty()) || (!queue.empty() && pick(&it)); });
      if (it.req == nullptr) break;  // stopping and nothing left to serve
      reserved += it.bytes;
      peak_reserved = std::max(peak_reserved, reserved);
      running++;
      peak_running = std::max(peak_running, running);
    }
    int rc = CPSB_OK;
    std::string msg;
    if (!st) {
      rc = CPSB_ERR_CUDA;
      msg = "stream creation failed";
    } else {
      try {
        run_item(it, st);
      } catch (const Error &e) {
        rc = e.code;
        msg = e.msg;
      } catch (...) {
        rc = CPSB_ERR_CUDA;
        msg = "unexpected exception";
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      reserved -= it.bytes;
      running--;
      ServeRequest &r = *it.req;
      r.h->g.inflight -= 1;  // the item no longer touches the gauge field
      if (rc != CPSB_OK && (r.status == CPSB_OK || (r.status > 0 && rc < 0))) {
        r.status = rc;
        r.err = msg;
      }
      if (--r.items_left == 0) {
        r.done = true;
        r.t_done = now_ms();
        t_last_done = r.t_done;
        if (r.status < 0) failed++;
        else {
          completed++;
          rhs_done += r.nrhs;
          lat_ms.push_back(r.t_done - r.t_submit);
        }
      }
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
  if (st) cudaStreamDestroy(st);
}

static double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace cpsb

struct cpsb_server_s {
  Server s;
};

extern "C" {

int cpsb_serve_create(cpsb_server *out, int slots, double hbm_fraction, unsigned long long hbm_bytes) {
  return guarded([&] {
    need_init();
    if (!out || slots < 1 || slots > 64) throw Error{CPSB_ERR_ARG, "bad server handle / slot count"};
    if (!(hbm_fraction > 0 && hbm_fraction <= 1) && hbm_bytes == 0)
      throw Error{CPSB_ERR_ARG, "give hbm_fraction in (0, 1] or hbm_bytes > 0"};
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    size_t budget = hbm_fraction > 0 && hbm_fraction <= 1 ? (size_t)(hbm_fraction * (double)fr) : fr;
    if (hbm_bytes) budget = std::min(budget, (size_t)hbm_bytes);
    std::unique_ptr<cpsb_server_s> h(new cpsb_server_s);
    Server &S = h->s;
    S.device = ctx().device;
    S.budget = budget;
    S.slots = slots;
    for (int i = 0; i < slots; i++) S.workers.emplace_back([&S] { S.worker_main(); });
    *out = h.release();
    return CPSB_OK;
  });
}

int cpsb_serve_submit(cpsb_server srv, cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs,
                      double **x, const double *const *b, unsigned long long *id) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (!srv || !id || !x || !b || nrhs < 1 || nrhs > 4096) throw Error{CPSB_ERR_ARG, "bad submit arguments"};
    for (int i = 0; i < nrhs; i++)
      if (!x[i] || !b[i]) throw Error{CPSB_ERR_ARG, "null vector"};
    Server &S = srv->s;
    const long n = cb_sites(h, p);
    int g = std::min(nrhs, MAX_RHS);
    while (g > 0 && solve_footprint(*p, n, a->precision, g) > S.budget) g--;
    if (g == 0) throw Error{CPSB_ERR_OOM, "one right-hand side of this request exceeds the server's HBM budget"};
    std::unique_ptr<ServeRequest> r(new ServeRequest);
    r->h = h;
    r->p = *p;
    if (p->action == CPSB_ZMOBIUS) {
      r->zb.assign(p->zmobius_b, p->zmobius_b + 2 * p->ls);
      r->zc.assign(p->zmobius_c, p->zmobius_c + 2 * p->ls);
      r->p.zmobius_b = r->zb.data();
      r->p.zmobius_c = r->zc.data();
    }
    r->a = *a;
    r->nrhs = nrhs;
    r->x.assign(x, x + nrhs);
    r->b.assign(b, b + nrhs);
    r->res.assign(nrhs, cpsb_solve_result());
    const int nitems = (nrhs + g - 1) / g;
    r->items_left = nitems;
    {
      std::lock_guard<std::mutex> lk(S.mu);
      if (S.stopping) throw Error{CPSB_ERR_BUSY, "server is shutting down"};
      r->id = S.next_id++;
      r->t_submit = now_ms();
      if (S.t_first_submit < 0) S.t_first_submit = r->t_submit;
      // near-equal groups of at most g right-hand sides
      int r0 = 0;
      for (int k = 0; k < nitems; k++) {
        const int m = nrhs / nitems + (k < nrhs % nitems ? 1 : 0);
        S.queue.push_back(ServeItem{r.get(), r0, m, solve_footprint(*p, n, a->precision, m)});
        r0 += m;
      }
      h->g.inflight += nitems;
      *id = r->id;
      S.reqs[r->id] = std::move(r);
    }
    S.cv_work.notify_all();
    return CPSB_OK;
  });
}

int cpsb_serve_submit_minvcg(cpsb_server srv, cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a,
                             double **x, const double *b, const double *shift, int nshift, double *rsd, int type,
                             const double *alpha, unsigned long long *id) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (!srv || !id || !x || !b || !shift || !rsd || nshift < 1 || nshift > 32)
      throw Error{CPSB_ERR_ARG, "bad multishift submit arguments"};
    if (type != CPSB_MULTI && type != CPSB_SINGLE) throw Error{CPSB_ERR_UNSUPPORTED, "only MULTI and SINGLE"};
    if (type == CPSB_SINGLE && !alpha) throw Error{CPSB_ERR_ARG, "SINGLE needs alpha"};
    const int nvec = type == CPSB_SINGLE ? 1 : nshift;
    for (int i = 0; i < nvec; i++)
      if (!x[i]) throw Error{CPSB_ERR_ARG, "null solution vector"};
    Server &S = srv->s;
    const long n = cb_sites(h, p);
    const size_t bytes = multishift_footprint(*p, n, a->precision, nshift, nvec);
    if (bytes > S.budget) throw Error{CPSB_ERR_OOM, "this multishift solve exceeds the server's HBM budget"};
    std::unique_ptr<ServeRequest> r(new ServeRequest);
    r->h = h;
    r->p = *p;
    if (p->action == CPSB_ZMOBIUS) {
      r->zb.assign(p->zmobius_b, p->zmobius_b + 2 * p->ls);
      r->zc.assign(p->zmobius_c, p->zmobius_c + 2 * p->ls);
      r->p.zmobius_b = r->zb.data();
      r->p.zmobius_c = r->zc.data();
    }
    r->a = *a;
    r->nrhs = 1;
    r->multishift = true;
    r->x.assign(x, x + nvec);
    r->b.assign(&b, &b + 1);
    r->res.assign(1, cpsb_solve_result());
    r->shift.assign(shift, shift + nshift);
    if (alpha) r->alpha.assign(alpha, alpha + nshift);
    r->rsd = rsd;
    r->ms_type = type;
    r->items_left = 1;
    {
      std::lock_guard<std::mutex> lk(S.mu);
      if (S.stopping) throw Error{CPSB_ERR_BUSY, "server is shutting down"};
      r->id = S.next_id++;
      r->t_submit = now_ms();
      if (S.t_first_submit < 0) S.t_first_submit = r->t_submit;
      S.queue.push_back(ServeItem{r.get(), 0, 1, bytes});
      h->g.inflight += 1;
      *id = r->id;
      S.reqs[r->id] = std::move(r);
    }
    S.cv_work.notify_all();
    return CPSB_OK;
  });
}

int cpsb_serve_poll(cpsb_server srv, unsigned long long id, int *done) {
  return guarded([&] {
    if (!srv || !done) throw Error{CPSB_ERR_ARG, "bad poll arguments"};
    Server &S = srv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    auto itr = S.reqs.find(id);
    if (itr == S.reqs.end()) throw Error{CPSB_ERR_ARG, "unknown request id"};
    *done = itr->second->done ? 1 : 0;
    return CPSB_OK;
  });
}

int cpsb_serve_wait(cpsb_server srv, unsigned long long id, cpsb_solve_result *res, double *latency_ms) {
  return guarded([&] {
    if (!srv) throw Error{CPSB_ERR_ARG, "null server"};
    Server &S = srv->s;
    std::unique_ptr<ServeRequest> r;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      auto itr = S.reqs.find(id);
      if (itr == S.reqs.end()) throw Error{CPSB_ERR_ARG, "unknown request id"};
      ServeRequest *rp = itr->second.get();
      S.cv_done.wait(lk, [&] { return rp->done; });
      r = std::move(itr->second);
      S.reqs.erase(itr);
    }
    if (res) memcpy(res, r->res.data(), sizeof(cpsb_solve_result) * r->nrhs);
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    if (r->status < 0) throw Error{r->status, r->err};
    return r->status;
  });
}

int cpsb_serve_stats(cpsb_server srv, cpsb_serve_stats_t *st) {
  return guarded([&] {
    if (!srv || !st) throw Error{CPSB_ERR_ARG, "bad stats arguments"};
    Server &S = srv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    memset(st, 0, sizeof(*st));
    st->completed = S.completed;
    st->failed = S.failed;
    st->rhs_completed = S.rhs_done;
    st->p50_ms = percentile(S.lat_ms, 0.50);
    st->p99_ms = percentile(S.lat_ms, 0.99);
    double sum = 0, mx = 0;
    for (double v : S.lat_ms) {
      sum += v;
      mx = std::max(mx, v);
    }
    st->mean_ms = S.lat_ms.empty() ? 0 : sum / (double)S.lat_ms.size();
    st->max_ms = mx;
    const double span = S.t_last_done - S.t_first_submit;
    st->requests_per_s = span > 0 ? 1e3 * (double)S.completed / span : 0;
    st->rhs_per_s = span > 0 ? 1e3 * (double)S.rhs_done / span : 0;
    st->peak_running = S.peak_running;
    st->queued = (int)S.queue.size();
    st->running = S.running;
    st->budget_bytes = (double)S.budget;
    st->peak_reserved_bytes = (double)S.peak_reserved;
    return CPSB_OK;
  });
}

int cpsb_serve_destroy(cpsb_server srv) {
  return guarded([&] {
    if (!srv) return CPSB_OK;
    {
      std::lock_guard<std::mutex> lk(srv->s.mu);
      srv->s.stopping = true;
    }
    srv->s.cv_work.notify_all();
    for (auto &t : srv->s.workers) t.join();
    delete srv;
    return CPSB_OK;
  });
}

}  // extern "C"

// capi.cu -- the extern "C" boundary (include/cpsb200.h).  Validates arguments,
// moves host vectors in CPS order through pinned staging buffers, packs them
// into the device layout and converts every library error into a status code.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <complex>

#include "abi.h"

using namespace cpsb;

namespace cpsb {
void drop_solvers(Gauge *G);
}

namespace cpsb {

std::string &last_error_slot() {
  thread_local std::string msg;
  return msg;
}

void need_init() {
  if (ctx().device < 0) throw Error{CPSB_ERR_NO_DEVICE, "cpsb_init has not been called"};
  CK(cudaSetDevice(ctx().device));
}

void check_params(cpsb_gauge h, const cpsb_dirac_params *p) {
  if (!h || !p) throw Error{CPSB_ERR_ARG, "null gauge handle or parameters"};
  if (p->action < CPSB_WILSON || p->action > CPSB_ZMOBIUS) throw Error{CPSB_ERR_ARG, "unknown action"};
  if (p->action == CPSB_ZMOBIUS && (!p->zmobius_b || !p->zmobius_c))
    throw Error{CPSB_ERR_ARG, "zMobius needs the zmobius_b and zmobius_c coefficient arrays"};
  if (p->action != CPSB_WILSON && (p->ls < 2 || p->ls > 64)) throw Error{CPSB_ERR_ARG, "ls must be in [2, 64]"};
}

void check_cg(const cpsb_cg_arg *a) {
  if (!a) throw Error{CPSB_ERR_ARG, "null cg arguments"};
  if (!(a->stop_rsd >= 0) || a->max_num_iter < 0) throw Error{CPSB_ERR_ARG, "bad stop_rsd / max_num_iter"};
  if (a->precision < CPSB_PREC_F64 || a->precision > CPSB_PREC_F16) throw Error{CPSB_ERR_ARG, "bad precision"};
}

long cb_sites(cpsb_gauge h, const cpsb_dirac_params *p) {
  return h->g.n4cb * (p->action == CPSB_WILSON ? 1 : p->ls);
}

Geom geom_of(cpsb_gauge h, const cpsb_dirac_params *p, int nrhs) {
  return make_geom(h->g.dims, p->action == CPSB_WILSON ? 1 : p->ls, nrhs, p->action == CPSB_DWF);
}

}  // namespace cpsb

namespace {

// Pinned staging buffer reused across calls (grown on demand).
// Host <-> device staging of CPS-order vectors: two pinned buffers and two
// device buffers of one vector each.  While vector i is copied by DMA (and
// packed on the device), vector i+1 is copied into the other pinned buffer by
// several host threads, so host copy and transfer overlap.
struct Staging {
  void *pin[2] = {nullptr, nullptr};
  DevBuf dev[2];
  cudaEvent_t done[2] = {nullptr, nullptr};  // last use of pin[k] by the device is over
  size_t bytes = 0;
  std::mutex mu;
  void ensure(size_t n) {
    if (!done[0]) {
      CK(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
    }
    if (n <= bytes) return;
    for (int k = 0; k < 2; k++) {
      if (pin[k]) cudaFreeHost(pin[k]);
      pin[k] = nullptr;
    }
    bytes = 0;
    for (int k = 0; k < 2; k++) {
      CK(cudaMallocHost(&pin[k], n));
      dev[k].alloc(n);
    }
    bytes = n;
  }
};
Staging &staging() {
  static Staging s;
  return s;
}

// memcpy of large vectors split over host threads.
void par_copy(void *dst, const void *src, size_t n) {
  const size_t chunk = 32u << 20;
  const int nt = (int)std::min<size_t>(8, (n + chunk - 1) / chunk);
  if (nt <= 1) {
    memcpy(dst, src, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t part = (n + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const size_t off = (size_t)t * part;
    if (off >= n) break;
    const size_t len = std::min(part, n - off);
    th.emplace_back([=] { memcpy((char *)dst + off, (const char *)src + off, len); });
  }
  for (auto &x : th) x.join();
}

}  // namespace

extern "C" {

const char *cpsb_error_string(int code) {
  switch (code) {
    case CPSB_OK: return "ok";
    case CPSB_NOT_CONVERGED: return "not converged within max_num_iter";
    case CPSB_ERR_ARG: return "invalid argument";
    case CPSB_ERR_CUDA: return "CUDA error";
    case CPSB_ERR_OOM: return "out of device memory";
    case CPSB_ERR_UNSUPPORTED: return "unsupported configuration";
    case CPSB_ERR_BREAKDOWN: return "solver breakdown (p.Ap = 0)";
    case CPSB_ERR_NO_DEVICE: return "no CUDA device / cpsb_init not called";
    case CPSB_ERR_BUSY: return "resource busy";
  }
  return "unknown status";
}

const char *cpsb_last_error(void) { return last_error_slot().c_str(); }

int cpsb_init(int device) {
  return guarded([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error{CPSB_ERR_NO_DEVICE, "no CUDA device"};
    if (device < 0 || device >= n) throw Error{CPSB_ERR_ARG, "device index out of range"};
    Context &c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.device == device) return CPSB_OK;
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    c.nsm = prop.multiProcessorCount;
    if (!c.stream) CK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.device = device;
    return CPSB_OK;
  });
}

int cpsb_mem_info(unsigned long long *free_b, unsigned long long *total_b) {
  return guarded([&] {
    need_init();
    size_t f = 0, t = 0;
    CK(cudaMemGetInfo(&f, &t));
    if (free_b) *free_b = f;
    if (total_b) *total_b = t;
    return CPSB_OK;
  });
}

int cpsb_gauge_load(cpsb_gauge *out, const double *u, const int dims[4], int order, int bc_t) {
  return guarded([&] {
    need_init();
    if (!out || !u || !dims) throw Error{CPSB_ERR_ARG, "null argument"};
    for (int i = 0; i < 4; i++)
      if (dims[i] < 2 || dims[i] % 2) throw Error{CPSB_ERR_ARG, "lattice extents must be even and >= 2"};
    if (order != CPSB_ORDER_CANONICAL && order != CPSB_ORDER_WILSON) throw Error{CPSB_ERR_ARG, "bad gauge order"};
    std::unique_ptr<cpsb_gauge_s> h(new cpsb_gauge_s);
    Gauge &G = h->g;
    for (int i = 0; i < 4; i++) G.dims[i] = dims[i];
    G.bc_t = bc_t ? 1 : 0;
    const long vol = (long)dims[0] * dims[1] * dims[2] * dims[3];
    G.n4cb = vol / 2;
    const size_t bytes = (size_t)vol * 72 * sizeof(double);
    cudaStream_t st = ctx().stream;
    G.canon.alloc(bytes);
    std::vector<double> canon;
    const double *src = u;
    if (order == CPSB_ORDER_WILSON) {
      // WILSON -> CANONICAL: even sites first, links transposed (convert_func.C:371-405)
      canon.resize((size_t)vol * 72);
      const int lx = dims[0], ly = dims[1], lz = dims[2], lt = dims[3];
      for (int t = 0; t < lt; t++)
        for (int z = 0; z < lz; z++)
          for (int y = 0; y < ly; y++)
            for (int x = 0; x < lx; x++) {
              long cs = x + lx * (y + (long)ly * (z + (long)lz * t));
              long ws = (x - x % 2 + lx * (y + (long)ly * (z + (long)lz * t)) + vol * ((x + y + z + t) % 2)) / 2;
              for (int mu = 0; mu < 4; mu++)
                for (int row = 0; row < 3; row++)
                  for (int col = 0; col < 3; col++)
                    for (int r = 0; r < 2; r++)
                      canon[72 * cs + r + 2 * (col + 3 * (row + 3 * mu))] = u[72 * ws + r + 2 * (row + 3 * (col + 3 * mu))];
            }
      src = canon.data();
    }
    CK(cudaMemcpyAsync(G.canon.p, src, bytes, cudaMemcpyHostToDevice, st));
    G.u64.alloc((size_t)vol * 4 * 144);
    CK(launch_gauge_pack(P64, G.u64.p, (const double *)G.canon.p, G.dims, G.bc_t, st));
    DevBuf flag(8);
    CK(cudaMemsetAsync(flag.p, 0, 8, st));
    CK(launch_unitarity((const double *)G.canon.p, vol * 4, G.dims, G.bc_t, (unsigned long long *)flag.p, st));
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, flag.p, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double worst;
    memcpy(&worst, &bits, 8);
    G.recon_err = worst;
    G.recon_ok = worst < 1e-6;
    *out = h.release();
    return CPSB_OK;
  });
}

int cpsb_gauge_free(cpsb_gauge h) {
  return guarded([&] {
    if (!h) return CPSB_OK;
    need_init();
    if (h->g.inflight.load() > 0)
      throw Error{CPSB_ERR_BUSY, "gauge field has queued or running requests of the request loop; wait for them"};
    CK(cudaStreamSynchronize(ctx().stream));
    drop_solvers(&h->g);
    delete h;
    return CPSB_OK;
  });
}

}  // extern "C"

namespace {

// Copies nvec host vectors (each nsites_each*24 doubles, CPS order) into the
// multi-RHS field f one right-hand side at a time through a pinned buffer and
// a device buffer of one vector, packing each into its slice of f.
void upload(Field &f, const double *const *host, int nvec, const Geom &g1, cudaStream_t st) {
  const long nsites_each = g1.nsites;
  const size_t each = (size_t)nsites_each * 24 * sizeof(double);
  Staging &sg = staging();
  std::lock_guard<std::mutex> lk(sg.mu);
  sg.ensure(each);
  for (int i = 0; i < nvec; i++) {
    const int k = i & 1;
    CK(cudaEventSynchronize(sg.done[k]));  // the device is done with pin[k] / dev[k]
    par_copy(sg.pin[k], host[i], each);
    CK(cudaMemcpyAsync(sg.dev[k].p, sg.pin[k], each, cudaMemcpyHostToDevice, st));
    CK(launch_pack(f.prec, f.view((long)i * nsites_each), (const double *)sg.dev[k].p, g1, st));
    CK(cudaEventRecord(sg.done[k], st));
  }
  CK(cudaStreamSynchronize(st));
}

void download(double *const *host, int nvec, const Geom &g1, const Field &f, cudaStream_t st) {
  const long nsites_each = g1.nsites;
  const size_t each = (size_t)nsites_each * 24 * sizeof(double);
  Staging &sg = staging();
  std::lock_guard<std::mutex> lk(sg.mu);
  sg.ensure(each);
  // vector i is unpacked and transferred while vector i-1 is copied out on the host
  for (int i = 0; i <= nvec; i++) {
    if (i < nvec) {
      const int k = i & 1;
      CK(launch_unpack(f.prec, (double *)sg.dev[k].p, f.view((long)i * nsites_each), g1, st));
      CK(cudaMemcpyAsync(sg.pin[k], sg.dev[k].p, each, cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(sg.done[k], st));
    }
    if (i > 0) {
      const int k = (i - 1) & 1;
      CK(cudaEventSynchronize(sg.done[k]));
      par_copy(host[i - 1], sg.pin[k], each);
    }
  }
}

}  // namespace

extern "C" {

int cpsb_dslash(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, int cb, int dag) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (!out || !in || (cb != 0 && cb != 1) || (dag != 0 && dag != 1)) throw Error{CPSB_ERR_ARG, "bad argument"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    Field fi(P64, op.nsites()), fo(P64, op.nsites());
    upload(fi, &in, 1, op.geom, st);
    op.dslash(fo, fi, cb, dag, st);
    download(&out, 1, op.geom, fo, st);
    return CPSB_OK;
  });
}

int cpsb_matpc(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, int dag) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (!out || !in || (dag != 0 && dag != 1)) throw Error{CPSB_ERR_ARG, "bad argument"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    Field fi(P64, op.nsites()), fo(P64, op.nsites());
    upload(fi, &in, 1, op.geom, st);
    op.matpc(fo, fi, dag, nullptr, nullptr, st);
    download(&out, 1, op.geom, fo, st);
    return CPSB_OK;
  });
}

int cpsb_mdagm(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, double *dot) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (!out || !in) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    Field fi(P64, op.nsites()), fo(P64, op.nsites());
    RedSlot rs;
    DevBuf d(sizeof(double) * MAX_RHS);
    Reduce r = rs.r((double *)d.p);
    upload(fi, &in, 1, op.geom, st);
    op.mdagm(fo, fi, &r, nullptr, st);
    if (dot) CK(cudaMemcpyAsync(dot, d.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    download(&out, 1, op.geom, fo, st);
    return CPSB_OK;
  });
}

int cpsb_dslash_ex(cpsb_gauge h, const cpsb_dirac_params *p, int precision, double *out, const double *in, int cb,
                   int dag) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (precision < CPSB_PREC_F64 || precision > CPSB_PREC_F16) throw Error{CPSB_ERR_ARG, "bad precision"};
    if (!out || !in || (cb != 0 && cb != 1) || (dag != 0 && dag != 1)) throw Error{CPSB_ERR_ARG, "bad argument"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, precision, 1);
    Field fi(precision, op.nsites()), fo(precision, op.nsites());
    upload(fi, &in, 1, op.geom, st);
    op.dslash(fo, fi, cb, dag, st);
    download(&out, 1, op.geom, fo, st);
    return CPSB_OK;
  });
}

int cpsb_mdagm_ex(cpsb_gauge h, const cpsb_dirac_params *p, int precision, double *out, const double *in,
                  double *dot) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (precision < CPSB_PREC_F64 || precision > CPSB_PREC_F16) throw Error{CPSB_ERR_ARG, "bad precision"};
    if (!out || !in) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, precision, 1);
    Field fi(precision, op.nsites()), fo(precision, op.nsites());
    RedSlot rs;
    DevBuf d(sizeof(double) * MAX_RHS);
    Reduce r = rs.r((double *)d.p);
    upload(fi, &in, 1, op.geom, st);
    op.mdagm(fo, fi, &r, nullptr, st);
    if (dot) CK(cudaMemcpyAsync(dot, d.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    download(&out, 1, op.geom, fo, st);
    return CPSB_OK;
  });
}

int cpsb_mdagm_dev(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, double *dot,
                   void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (!out || !in) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    Field fi(P64, op.nsites()), fo(P64, op.nsites());
    RedSlot rs;
    DevBuf d(sizeof(double) * MAX_RHS);
    Reduce r = rs.r((double *)d.p);
    CK(launch_pack(P64, fi.ptr(), in, op.geom, st));
    op.mdagm(fo, fi, &r, nullptr, st);
    CK(launch_unpack(P64, out, fo.ptr(), op.geom, st));
    if (dot) CK(cudaMemcpyAsync(dot, d.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return CPSB_OK;
  });
}

int cpsb_dslash_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, double *out,
                          const double *in, int cb, int dag, void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (precision < CPSB_PREC_F64 || precision > CPSB_PREC_F16) throw Error{CPSB_ERR_ARG, "bad precision"};
    if (nrhs < 1 || nrhs > MAX_RHS) throw Error{CPSB_ERR_ARG, "nrhs out of range"};
    if (!out || !in || (cb != 0 && cb != 1) || (dag != 0 && dag != 1)) throw Error{CPSB_ERR_ARG, "bad argument"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    Operator op(&h->g, *p, precision, nrhs);
    Field fi(precision, op.nsites()), fo(precision, op.nsites());
    CK(launch_pack(precision, fi.ptr(), in, op.geom, st));
    op.dslash(fo, fi, cb, dag, st);
    CK(launch_unpack(precision, out, fo.ptr(), op.geom, st));
    CK(cudaStreamSynchronize(st));
    return CPSB_OK;
  });
}

int cpsb_mdagm_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, double *out,
                         const double *in, double *dot, void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (precision < CPSB_PREC_F64 || precision > CPSB_PREC_F16) throw Error{CPSB_ERR_ARG, "bad precision"};
    if (nrhs < 1 || nrhs > MAX_RHS) throw Error{CPSB_ERR_ARG, "nrhs out of range"};
    if (!out || !in) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    Operator op(&h->g, *p, precision, nrhs);
    Field fi(precision, op.nsites()), fo(precision, op.nsites());
    RedSlot rs;
    DevBuf d(sizeof(double) * MAX_RHS);
    Reduce r = rs.r((double *)d.p);
    CK(launch_pack(precision, fi.ptr(), in, op.geom, st));
    op.mdagm(fo, fi, &r, nullptr, st);
    CK(launch_unpack(precision, out, fo.ptr(), op.geom, st));
    if (dot) CK(cudaMemcpyAsync(dot, d.p, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return CPSB_OK;
  });
}


int cpsb_invcg_multi(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs, double **x,
                     const double *const *b, cpsb_solve_result *res) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (nrhs < 1 || nrhs > MAX_RHS || !x || !b || !res) throw Error{CPSB_ERR_ARG, "bad nrhs / vectors"};
    for (int i = 0; i < nrhs; i++)
      if (!x[i] || !b[i]) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = ctx().stream;
    CgSolver *s = get_solver(&h->g, *p, a->precision, nrhs);
    std::lock_guard<std::mutex> lk(s->busy);
    const Geom g1 = geom_of(h, p, 1);
    upload(s->x64, (const double *const *)x, nrhs, g1, st);
    upload(s->b64, b, nrhs, g1, st);
    int rc = s->solve(*a, res, st);
    download(x, nrhs, g1, s->x64, st);
    return rc;
  });
}

int cpsb_invcg(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *x, const double *b,
               cpsb_solve_result *res) {
  double *xs[1] = {x};
  const double *bs[1] = {b};
  return cpsb_invcg_multi(h, p, a, 1, xs, bs, res);
}

int cpsb_invcg_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs, double *x,
                         const double *b, cpsb_solve_result *res, void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (nrhs < 1 || nrhs > MAX_RHS || !x || !b || !res) throw Error{CPSB_ERR_ARG, "bad nrhs / vectors"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    CgSolver *s = get_solver(&h->g, *p, a->precision, nrhs);
    std::lock_guard<std::mutex> lk(s->busy);
    CK(launch_pack(P64, s->x64.ptr(), x, s->geom, st));
    CK(launch_pack(P64, s->b64.ptr(), b, s->geom, st));
    int rc = s->solve(*a, res, st);
    CK(launch_unpack(P64, x, s->x64.ptr(), s->geom, st));
    CK(cudaStreamSynchronize(st));
    return rc;
  });
}

int cpsb_invcg_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *x, const double *b,
                   cpsb_solve_result *res, void *stream) {
  return cpsb_invcg_multi_dev(h, p, a, 1, x, b, res, stream);
}

int cpsb_minvcg(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double **x, const double *b,
                const double *shift, int nshift, double *rsd, int type, const double *alpha,
                cpsb_solve_result *res) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (!x || !b || !shift || !rsd || nshift < 1 || nshift > 32) throw Error{CPSB_ERR_ARG, "bad multishift arguments"};
    if (type != CPSB_MULTI && type != CPSB_SINGLE) throw Error{CPSB_ERR_UNSUPPORTED, "only MULTI and SINGLE are implemented"};
    if (type == CPSB_SINGLE && !alpha) throw Error{CPSB_ERR_ARG, "SINGLE needs alpha"};
    const int nvec = type == CPSB_SINGLE ? 1 : nshift;
    for (int i = 0; i < nvec; i++)
      if (!x[i]) throw Error{CPSB_ERR_ARG, "null solution vector"};
    cudaStream_t st = ctx().stream;
    const long n = cb_sites(h, p);
    const Geom g1 = geom_of(h, p, 1);
    Field chi(P64, n);
    upload(chi, &b, 1, g1, st);
    std::vector<Field> xs(nvec);
    for (int i = 0; i < nvec; i++) {
      xs[i].create(P64, n);
      CK(cudaMemsetAsync(xs[i].data.p, 0, xs[i].data.bytes, st));
    }
    cpsb_solve_result r;
    memset(&r, 0, sizeof(r));
    const int rc = multishift(&h->g, *p, *a, chi, xs, shift, nshift, rsd, type, alpha, &r, st);
    for (int i = 0; i < nvec; i++) download(&x[i], 1, g1, xs[i], st);
    if (res) *res = r;
    return rc;
  });
}

int cpsb_minvcg_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *const *x,
                    const double *b, const double *shift, int nshift, double *rsd, int type, const double *alpha,
                    cpsb_solve_result *res, void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (!x || !b || !shift || !rsd || nshift < 1 || nshift > 32) throw Error{CPSB_ERR_ARG, "bad multishift arguments"};
    if (type != CPSB_MULTI && type != CPSB_SINGLE) throw Error{CPSB_ERR_UNSUPPORTED, "only MULTI and SINGLE are implemented"};
    if (type == CPSB_SINGLE && !alpha) throw Error{CPSB_ERR_ARG, "SINGLE needs alpha"};
    const int nvec = type == CPSB_SINGLE ? 1 : nshift;
    for (int i = 0; i < nvec; i++)
      if (!x[i]) throw Error{CPSB_ERR_ARG, "null solution vector"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    const long n = cb_sites(h, p);
    const Geom g1 = geom_of(h, p, 1);
    Field chi(P64, n);
    CK(launch_pack(P64, chi.ptr(), b, g1, st));
    std::vector<Field> xs(nvec);
    for (int i = 0; i < nvec; i++) {
      xs[i].create(P64, n);
      CK(cudaMemsetAsync(xs[i].data.p, 0, xs[i].data.bytes, st));
    }
    cpsb_solve_result r;
    memset(&r, 0, sizeof(r));
    const int rc = multishift(&h->g, *p, *a, chi, xs, shift, nshift, rsd, type, alpha, &r, st);
    for (int i = 0; i < nvec; i++) CK(launch_unpack(P64, x[i], xs[i].ptr(), g1, st));
    CK(cudaStreamSynchronize(st));
    if (res) *res = r;
    return rc;
  });
}

static void check_minvcg_multi(int nvec, const void *x, const void *b, const double *shift, int nshift,
                               const double *rsd, int type, const double *alpha, const cpsb_solve_result *res) {
  if (nvec < 1 || nvec > MAX_RHS) throw Error{CPSB_ERR_ARG, "nvec must be in [1, 16]"};
  if (!x || !b || !shift || !rsd || !res || nshift < 1 || nshift > 32) throw Error{CPSB_ERR_ARG, "bad multishift arguments"};
  if (type != CPSB_MULTI && type != CPSB_SINGLE) throw Error{CPSB_ERR_UNSUPPORTED, "only MULTI and SINGLE are implemented"};
  if (type == CPSB_SINGLE && !alpha) throw Error{CPSB_ERR_ARG, "SINGLE needs alpha"};
}

int cpsb_minvcg_multi(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nvec, double **x,
                      const double *const *b, const double *shift, int nshift, double *rsd, int type,
                      const double *alpha, cpsb_solve_result *res) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    check_minvcg_multi(nvec, x, b, shift, nshift, rsd, type, alpha, res);
    const int nsol = type == CPSB_SINGLE ? 1 : nshift;
    for (int i = 0; i < nvec * nsol; i++)
      if (!x[i]) throw Error{CPSB_ERR_ARG, "null solution vector"};
    for (int q = 0; q < nvec; q++)
      if (!b[q]) throw Error{CPSB_ERR_ARG, "null source vector"};
    cudaStream_t st = ctx().stream;
    const long n1 = cb_sites(h, p);
    const Geom g1 = geom_of(h, p, 1);
    Field chi(P64, n1 * nvec);
    upload(chi, b, nvec, g1, st);
    std::vector<Field> xs(nsol);
    for (int s = 0; s < nsol; s++) {
      xs[s].create(P64, n1 * nvec);
      CK(cudaMemsetAsync(xs[s].data.p, 0, xs[s].data.bytes, st));
    }
    const int rc = multishift_multi(&h->g, *p, *a, nvec, chi, xs, shift, nshift, rsd, type, alpha, res, st);
    std::vector<double *> hx(nvec);
    for (int s = 0; s < nsol; s++) {
      for (int q = 0; q < nvec; q++) hx[q] = x[q * nsol + s];
      download(hx.data(), nvec, g1, xs[s], st);
    }
    return rc;
  });
}

int cpsb_minvcg_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nvec,
                          double *const *x, const double *b, const double *shift, int nshift, double *rsd, int type,
                          const double *alpha, cpsb_solve_result *res, void *stream) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    check_minvcg_multi(nvec, x, b, shift, nshift, rsd, type, alpha, res);
    const int nsol = type == CPSB_SINGLE ? 1 : nshift;
    for (int i = 0; i < nvec * nsol; i++)
      if (!x[i]) throw Error{CPSB_ERR_ARG, "null solution vector"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    const long n1 = cb_sites(h, p);
    const Geom g1 = geom_of(h, p, 1);
    Field chi(P64, n1 * nvec);
    CK(launch_pack(P64, chi.ptr(), b, geom_of(h, p, nvec), st));
    std::vector<Field> xs(nsol);
    for (int s = 0; s < nsol; s++) {
      xs[s].create(P64, n1 * nvec);
      CK(cudaMemsetAsync(xs[s].data.p, 0, xs[s].data.bytes, st));
    }
    const int rc = multishift_multi(&h->g, *p, *a, nvec, chi, xs, shift, nshift, rsd, type, alpha, res, st);
    for (int s = 0; s < nsol; s++)
      for (int q = 0; q < nvec; q++) CK(launch_unpack(P64, x[q * nsol + s], xs[s].view((long)q * n1), g1, st));
    CK(cudaStreamSynchronize(st));
    return rc;
  });
}

// out = fa x + fb y (y optional) on FP64 fields of one right-hand side.
static void lin64(const Geom &g, const Field &o, double fa, const Field &x, double fb, const Field *y,
                  cudaStream_t st) {
  Reduce none;
  memset(&none, 0, sizeof(none));
  Scal2 c;
  for (int i = 0; i < MAX_RHS; i++) {
    c.a[i] = fa;
    c.b[i] = fb;
  }
  CK(launch_axpby(P64, o.ptr(), P64, x.ptr(), P64, y ? y->ptr() : SpinorPtr{}, g, c, nullptr, none, 0, st));
}

// DiracOpMobius::Dminus (d_op_mobius.C:745-777): mobius_dminus (mobius_dminus.C:
// 29-86) hops each checkerboard into the other on every s slice with the fixed
// 4-D parity of the input, on -c/2 times the input; then out = -(k in + out),
// k = c(4 - M5) - a5_inv.  Here: out_x = (c/2) D_W in_y - k in_x.
static void mobius_dminus_dev(Operator &op, const cpsb_dirac_params &p, const Field &out_e, const Field &out_o,
                              const Field &in_e, const Field &in_o, cudaStream_t st) {
  const double c = p.mobius_c;
  const double k = 0.5 * (2 * (c * (4 - p.m5) - p.a5_inv));
  op.hop(out_e.ptr(), in_o.ptr(), 1, 0, 1.0, nullptr, nullptr, nullptr, st);
  op.hop(out_o.ptr(), in_e.ptr(), 0, 0, 1.0, nullptr, nullptr, nullptr, st);
  lin64(op.geom, out_e, 0.5 * c, out_e, -k, &in_e, st);
  lin64(op.geom, out_o, 0.5 * c, out_o, -k, &in_o, st);
}

// DiracOpZMobius::Dminus (d_op_zmobius.C:1213-1272, zmobius_dminus.C:44-116):
// out_x = (c_s/2) D_W in_y - (c_s(4 - M5) - a5_inv) in_x per slice s (complex c_s),
// x, y the two checkerboards (o: the solve checkerboard).
static void zmobius_dminus_dev(Operator &op, const Field &out_o, const Field &out_e, const Field &in_o,
                               const Field &in_e, cudaStream_t st) {
  Reduce none;
  memset(&none, 0, sizeof(none));
  const ZM5Tab *t = (const ZM5Tab *)op.ztab.p;
  Field th(P64, op.nsites());
  for (int half = 0; half < 2; half++) {
    const Field &src_other = half ? in_o : in_e, &src_same = half ? in_e : in_o;
    const Field &dst = half ? out_e : out_o;
    op.hop(th.ptr(), src_other.ptr(), half ? 1 : 0, 0, 1.0, nullptr, nullptr, nullptr, st);
    CK(launch_m5z(P64, 0, op.geom, dst.ptr(), src_same.ptr(), SpinorPtr{}, t + 11, 0, 0, none, nullptr, st));
    CK(launch_m5z(P64, 0, op.geom, dst.ptr(), th.ptr(), dst.ptr(), t + 12, 1, 0, none, nullptr, st));
  }
}

// fmat: the Lattice::FmatInv form (Mobius: Dminus of the source when dminus;
// zMobius: f_zmobius.C:70-130, Dminus for dminus == 1, then 2 kappa_b(s) per
// slice); otherwise DiracOp*::MatInv.
static int matinv_impl(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *out,
                       const double *in, int dminus, bool fmat, cpsb_solve_result *res) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    check_cg(a);
    if (!out || !in || !res) throw Error{CPSB_ERR_ARG, "null vector or result"};
    const bool zm = p->action == CPSB_ZMOBIUS;
    if (zm && p->pc_type != 0 && p->pc_type != 2 && p->pc_type != 5)  // d_op_zmobius.C:929-1080
      throw Error{CPSB_ERR_UNSUPPORTED, "zMobius MatInv: ZMOB_PC_SYM2, ORIG and SYM3 only (as the reference)"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    const long n = op.nsites();
    const Geom &g = op.geom;
    // solve-checkerboard (c) and other (e) halves of the full vectors
    const bool mob = p->action == CPSB_MOBIUS;
    const double *in_c = in + (mob ? 24 * n : 0), *in_e = in + (mob ? 0 : 24 * n);
    double *out_c = out + (mob ? 24 * n : 0), *out_e = out + (mob ? 0 : 24 * n);
    Field fin_c(P64, n), fin_e(P64, n), fout_c(P64, n), fout_e(P64, n), t(P64, n), t2(P64, n);
    upload(fin_c, &in_c, 1, g, st);
    upload(fin_e, &in_e, 1, g, st);
    upload(fout_c, (const double *const *)&out_c, 1, g, st);
    Reduce none;
    memset(&none, 0, sizeof(none));
    const ZM5Tab *zt = zm ? (const ZM5Tab *)op.ztab.p : nullptr;
    if (fmat && mob && dminus) {
      // f_mobius.C:45-117: the source becomes Dminus(source) before MatInv
      mobius_dminus_dev(op, *p, t, t2, fin_e, fin_c, st);
      CK(cudaMemcpyAsync(fin_e.data.p, t.data.p, t.data.bytes, cudaMemcpyDeviceToDevice, st));
      CK(cudaMemcpyAsync(fin_c.data.p, t2.data.p, t2.data.bytes, cudaMemcpyDeviceToDevice, st));
    }
    if (fmat && zm) {
      // f_zmobius.C:70-130: Dminus (dminus == 1), then 2 kappa_b(s) on both halves
      if (dminus == 1) {
        zmobius_dminus_dev(op, t, t2, fin_c, fin_e, st);
        CK(cudaMemcpyAsync(fin_c.data.p, t.data.p, t.data.bytes, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(fin_e.data.p, t2.data.p, t2.data.bytes, cudaMemcpyDeviceToDevice, st));
      }
      CK(launch_m5z(P64, 0, g, fin_c.ptr(), fin_c.ptr(), SpinorPtr{}, zt + 13, 0, 0, none, nullptr, st));
      CK(launch_m5z(P64, 0, g, fin_e.ptr(), fin_e.ptr(), SpinorPtr{}, zt + 13, 0, 0, none, nullptr, st));
    }
    auto lin = [&](const Field &o, double fa, const Field &x, double fb, const Field *y) {
      lin64(g, o, fa, x, fb, y, st);
    };
    double kb = 0;
    if (zm) {
      // d_op_zmobius.C:829-1080: t = kb . D4(M5^-1 in_e, CHKB_EVEN) + in_o (kb per
      // slice, commuting with the slice-local hop); SYM2: guess = M5 guess
      const SpinorPtr xc = fin_c.ptr();
      CK(launch_m5z(P64, 0, g, t.ptr(), fin_e.ptr(), SpinorPtr{}, zt + 6, 0, 0, none, nullptr, st));
      CK(launch_m5z(P64, 0, g, t2.ptr(), t.ptr(), SpinorPtr{}, zt + 4, 0, 0, none, nullptr, st));
      op.hop(t.ptr(), t2.ptr(), 0, 0, 1.0, &xc, nullptr, nullptr, st);
      if (p->pc_type == 2 || p->pc_type == 5) {
        CK(cudaMemcpyAsync(t2.data.p, fout_c.data.p, fout_c.data.bytes, cudaMemcpyDeviceToDevice, st));
        CK(launch_m5z(P64, 0, g, fout_c.ptr(), t2.ptr(), t2.ptr(), zt + 5, 1, 0, none, nullptr, st));
      }
    } else if (!mob) {
      // d_op_wilson.C:257-334, d_op_dwf.C:316-507
      op.dslash(t, fin_e, 0, 0, st);
      lin(t, op.kappa, t, 1.0, &fin_c);        // t = kappa D in_e + in_o
    } else {
      // d_op_mobius.C:389-640 (ZMOB_PC_ORIG, SYM1, SYM2)
      kb = op.kappa_b;
      op.mobius_m5inv(t.ptr(), fin_e.ptr(), st);
      op.mobius_d4(t2.ptr(), t.ptr(), 0, st);
      lin(t, kb, t2, 1.0, &fin_c);             // t = kappa_b D4 M5^-1 in_e + in_o
      if (p->pc_type == 2) {                   // SYM2: guess = M5 guess
        CK(cudaMemcpyAsync(t2.data.p, fout_c.data.p, fout_c.data.bytes, cudaMemcpyDeviceToDevice, st));
        const double kappa_c = 1.0 / (2 * (p->mobius_c * (4 - p->m5) - p->a5_inv));
        op.mobius_hop5_add(fout_c.ptr(), t2.ptr(), t2.ptr(), kb / kappa_c, st);
      }
      if (p->pc_type == 1) {                   // SYM1: source = M5^-1 source
        op.mobius_m5inv(t2.ptr(), t.ptr(), st);
        CK(cudaMemcpyAsync(t.data.p, t2.data.p, t.data.bytes, cudaMemcpyDeviceToDevice, st));
      }
    }
    CgSolver *s = get_solver(&h->g, *p, a->precision, 1);
    std::lock_guard<std::mutex> lk(s->busy);
    op.matpc(s->b64, t, 1, nullptr, nullptr, st);  // src = MatPcDag t
    CK(cudaMemcpyAsync(s->x64.data.p, fout_c.data.p, fout_c.data.bytes, cudaMemcpyDeviceToDevice, st));
    const int rc = s->solve(*a, res, st);
    CK(cudaMemcpyAsync(fout_c.data.p, s->x64.data.p, fout_c.data.bytes, cudaMemcpyDeviceToDevice, st));
    if (zm) {
      // SYM2 / SYM3: out_o = M5^-1 out_o; out_e = M5^-1(kb . D4(out_o, CHKB_ODD)) + M5^-1 in_e
      if (p->pc_type == 2 || p->pc_type == 5) {
        CK(launch_m5z(P64, 0, g, t.ptr(), fout_c.ptr(), SpinorPtr{}, zt + 6, 0, 0, none, nullptr, st));
        CK(cudaMemcpyAsync(fout_c.data.p, t.data.p, t.data.bytes, cudaMemcpyDeviceToDevice, st));
      }
      CK(launch_m5z(P64, 0, g, t2.ptr(), fout_c.ptr(), SpinorPtr{}, zt + 4, 0, 0, none, nullptr, st));
      op.hop(t.ptr(), t2.ptr(), 1, 0, 1.0, nullptr, nullptr, nullptr, st);
      CK(launch_m5z(P64, 0, g, t2.ptr(), fin_e.ptr(), SpinorPtr{}, zt + 6, 0, 0, none, nullptr, st));
      CK(launch_m5z(P64, 0, g, fout_e.ptr(), t.ptr(), t2.ptr(), zt + 6, 1, 0, none, nullptr, st));
    } else if (!mob) {
      op.dslash(t, fout_c, 1, 0, st);
      lin(fout_e, op.kappa, t, 1.0, &fin_e);   // out_e = kappa D out_o + in_e
    } else {
      if (p->pc_type == 2) {                   // SYM2: the solution is M5 out_o
        op.mobius_m5inv(t.ptr(), fout_c.ptr(), st);
        CK(cudaMemcpyAsync(fout_c.data.p, t.data.p, t.data.bytes, cudaMemcpyDeviceToDevice, st));
      }
      op.mobius_d4(t.ptr(), fout_c.ptr(), 1, st);
      lin(t2, kb, t, 0.0, nullptr);            // kappa_b D4 out_o
      op.mobius_m5inv(fout_e.ptr(), t2.ptr(), st);
      op.mobius_m5inv(t.ptr(), fin_e.ptr(), st);
      lin(fout_e, 1.0, fout_e, 1.0, &t);       // + M5^-1 in_e
      lin(fout_e, 2 * kb, fout_e, 0.0, nullptr);
      lin(fout_c, 2 * kb, fout_c, 0.0, nullptr);
    }
    download(&out_c, 1, g, fout_c, st);
    download(&out_e, 1, g, fout_e, st);
    return rc;
  });
}

int cpsb_matinv(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *out, const double *in,
                cpsb_solve_result *res) {
  return matinv_impl(h, p, a, out, in, 0, false, res);
}

int cpsb_fmatinv(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *out, const double *in,
                 int dminus, cpsb_solve_result *res) {
  if (p && p->action == CPSB_ZMOBIUS && dminus == -1) {  // f_zmobius.C:98: out = Dminus(in), no solve
    if (res) memset(res, 0, sizeof(*res));
    return cpsb_dminus(h, p, out, in);
  }
  return matinv_impl(h, p, a, out, in, dminus, true, res);
}

int cpsb_dminus(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (p->action != CPSB_MOBIUS && p->action != CPSB_ZMOBIUS)
      throw Error{CPSB_ERR_ARG, "Dminus is a Mobius / zMobius operator"};
    if (!out || !in) throw Error{CPSB_ERR_ARG, "null vector"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    const long n = op.nsites();
    if (out < in + 48 * n && in < out + 48 * n) throw Error{CPSB_ERR_ARG, "out and in overlap"};
    // DiracOpMobius keeps the even half first, DiracOpZMobius the odd half
    const bool zm = p->action == CPSB_ZMOBIUS;
    const double *in_e = in + (zm ? 24 * n : 0), *in_o = in + (zm ? 0 : 24 * n);
    double *out_e = out + (zm ? 24 * n : 0), *out_o = out + (zm ? 0 : 24 * n);
    Field fe(P64, n), fo(P64, n), ge(P64, n), go(P64, n);
    upload(fe, &in_e, 1, op.geom, st);
    upload(fo, &in_o, 1, op.geom, st);
    if (!zm) mobius_dminus_dev(op, *p, ge, go, fe, fo, st);
    else zmobius_dminus_dev(op, go, ge, fo, fe, st);
    download(&out_e, 1, op.geom, ge, st);
    download(&out_o, 1, op.geom, go, st);
    return CPSB_OK;
  });
}

int cpsb_fermion_convert(const int dims[4], int ls, int order, int direction, double *out, const double *in,
                         void *stream) {
  return guarded([&] {
    need_init();
    if (!dims || !out || !in || out == in) throw Error{CPSB_ERR_ARG, "bad vectors (out and in must differ)"};
    for (int k = 0; k < 4; k++)
      if (dims[k] < 2 || dims[k] % 2) throw Error{CPSB_ERR_ARG, "lattice extents must be even and >= 2"};
    if (ls < 1 || ls > 64) throw Error{CPSB_ERR_ARG, "ls out of range"};
    if ((order != CPSB_FERMION_CB && order != CPSB_FERMION_4D_EE) || (direction != 0 && direction != 1))
      throw Error{CPSB_ERR_ARG, "bad order / direction"};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    CK(launch_fconvert(out, in, dims, ls, order, direction, st));
    CK(cudaStreamSynchronize(st));
    return CPSB_OK;
  });
}

int cpsb_minresext(cpsb_gauge h, const cpsb_dirac_params *p, double *psi, const double *phi, double **v,
                   double **vm, int degree, double *resid) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (!psi || !phi || degree < 0 || degree > 16 || (degree > 0 && (!v || !vm)))
      throw Error{CPSB_ERR_ARG, "bad MinResExt arguments"};
    for (int i = 0; i < degree; i++)
      if (!v[i] || !vm[i]) throw Error{CPSB_ERR_ARG, "null previous solution"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, P64, 1);
    const long n = op.nsites();
    const Geom &g = op.geom;
    if (degree == 0) {  // minresext.C:57-61: no guess
      memset(psi, 0, sizeof(double) * 24 * n);
      if (resid) *resid = 1.0;
      return CPSB_OK;
    }
    Field fphi(P64, n), fpsi(P64, n), fr(P64, n);
    std::vector<Field> fv(degree), fvm(degree);
    upload(fphi, &phi, 1, g, st);
    for (int i = 0; i < degree; i++) {
      fv[i].create(P64, n);
      fvm[i].create(P64, n);
      upload(fv[i], (const double *const *)&v[i], 1, g, st);
    }
    RedSlot rs;
    DevBuf dres(sizeof(double) * 4);
    double hres[2];
    auto fetch = [&](int k) {
      CK(cudaMemcpyAsync(hres, dres.p, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    };
    auto cdot = [&](const Field &a, const Field &b) {
      CK(launch_cdot(a.ptr(), b.ptr(), n, rs.r((double *)dres.p), st));
      fetch(2);
      return std::complex<double>(hres[0], hres[1]);
    };
    auto norm2 = [&](const Field &a) {
      Geom g1 = g;
      CK(launch_redot(P64, g1, a.ptr(), a.ptr(), rs.r((double *)dres.p), st));
      fetch(1);
      return hres[0];
    };
    auto scale = [&](const Field &a, double f) {
      Scal2 c;
      for (int q = 0; q < MAX_RHS; q++) {
        c.a[q] = f;
        c.b[q] = 0.0;
      }
      Reduce none;
      memset(&none, 0, sizeof(none));
      CK(launch_axpby(P64, a.ptr(), P64, a.ptr(), P64, SpinorPtr{}, g, c, nullptr, none, 0, st));
    };
    typedef std::complex<double> cplx_t;
    std::vector<std::vector<cplx_t>> G(degree, std::vector<cplx_t>(degree));
    std::vector<cplx_t> a(degree), b(degree);
    // orthonormalise (minresext.C:84-93)
    for (int i = 0; i < degree; i++) {
      scale(fv[i], 1 / sqrt(norm2(fv[i])));
      for (int j = i + 1; j < degree; j++) {
        const cplx_t xp = cdot(fv[i], fv[j]);
        CK(launch_caxpy(fv[j].ptr(), -xp.real(), -xp.imag(), fv[i].ptr(), fv[j].ptr(), n, st));
      }
    }
    // right-hand side and the A-images (minresext.C:95-101)
    for (int i = 0; i < degree; i++) {
      b[i] = cdot(fv[i], fphi);
      Reduce rd = rs.r((double *)dres.p);
      op.mdagm(fvm[i], fv[i], &rd, nullptr, st);
      fetch(1);
      G[i][i] = cplx_t(hres[0], 0.0);
    }
    for (int j = 0; j < degree; j++)
      for (int k = j + 1; k < degree; k++) {
        G[j][k] = cdot(fv[j], fvm[k]);
        G[k][j] = std::conj(G[j][k]);
      }
    // the reference's elimination with its diagonal pivot test (minresext.C:113-135)
    for (int i = 0; i < degree; i++) {
      int k = i;
      for (int j = i + 1; j < degree; j++)
        if (std::abs(G[j][j]) > std::abs(G[k][k])) k = j;
      if (k != i) {
        std::swap(b[k], b[i]);
        std::swap(G[k], G[i]);
      }
      for (int j = i + 1; j < degree; j++) {
        const cplx_t xp = G[j][i] / G[i][i];
        b[j] -= xp * b[i];
        for (int m = 0; m < degree; m++) G[j][m] -= xp * G[i][m];
      }
    }
    CK(cudaMemsetAsync(fpsi.data.p, 0, fpsi.data.bytes, st));
    CK(cudaMemcpyAsync(fr.data.p, fphi.data.p, fphi.data.bytes, cudaMemcpyDeviceToDevice, st));
    for (int i = degree - 1; i >= 0; i--) {
      a[i] = 0.0;
      for (int j = i + 1; j < degree; j++) a[i] += G[i][j] * a[j];
      a[i] = (b[i] - a[i]) / G[i][i];
      CK(launch_caxpy(fpsi.ptr(), a[i].real(), a[i].imag(), fv[i].ptr(), fpsi.ptr(), n, st));
      CK(launch_caxpy(fr.ptr(), -a[i].real(), -a[i].imag(), fvm[i].ptr(), fr.ptr(), n, st));
    }
    if (resid) *resid = sqrt(norm2(fr) / norm2(fphi));
    download(&psi, 1, g, fpsi, st);
    for (int i = 0; i < degree; i++) {
      download(&v[i], 1, g, fv[i], st);
      download(&vm[i], 1, g, fvm[i], st);
    }
    return CPSB_OK;
  });
}

int cpsb_kernel_launches(unsigned long long *count) {
  if (!count) return CPSB_ERR_ARG;
  *count = launch_count();
  return CPSB_OK;
}

int cpsb_bench_dslash(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, int reps, double *ms,
                      double *bytes) {
  return guarded([&] {
    need_init();
    check_params(h, p);
    if (reps < 1 || nrhs < 1 || nrhs > MAX_RHS) throw Error{CPSB_ERR_ARG, "bad reps / nrhs"};
    cudaStream_t st = ctx().stream;
    Operator op(&h->g, *p, precision, nrhs);
    // Enough (in, out) field pairs that consecutive applications together touch
    // more than twice the 126 MB L2: no launch finds its input left in L2 by the
    // previous one.  Inputs are seeded Gaussian spinors (every right-hand side
    // the same vector).
    const size_t pair_bytes = 2 * field_bytes(precision, op.nsites());
    const int npairs = (int)std::min<size_t>(8, (252u << 20) / pair_bytes + 1);
    std::vector<std::unique_ptr<Field>> fin, fout;
    {
      const Geom g1 = geom_of(h, p, 1);
      const long n1 = g1.nsites;
      std::vector<double> v((size_t)n1 * 24);
      unsigned long long st_rng = 0x9E3779B97F4A7C15ull;
      for (auto &x : v) {  // uniform in [-1, 1) from a 64-bit LCG (values only feed timing)
        st_rng = st_rng * 6364136223846793005ull + 1442695040888963407ull;
        x = (double)(st_rng >> 11) * (2.0 / 9007199254740992.0) - 1.0;
      }
      DevBuf dv(v.size() * sizeof(double));
      CK(cudaMemcpyAsync(dv.p, v.data(), dv.bytes, cudaMemcpyHostToDevice, st));
      for (int k = 0; k < npairs; k++) {
        fin.emplace_back(new Field(precision, op.nsites()));
        fout.emplace_back(new Field(precision, op.nsites()));
        for (int q = 0; q < nrhs; q++)
          CK(launch_pack(precision, fin.back()->view((long)q * n1), (const double *)dv.p, g1, st));
      }
      CK(cudaStreamSynchronize(st));
    }
    for (int i = 0; i < 3; i++) op.hop(*fout[0], *fin[0], 1, 0, 1.0, nullptr, nullptr, nullptr, st);  // tunes, warms
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
    for (int i = 0; i < reps; i++)
      op.hop(*fout[i % npairs], *fin[i % npairs], 1, 0, 1.0, nullptr, nullptr, nullptr, st);
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t / reps;
    if (bytes) *bytes = op.hop_bytes();
    return CPSB_OK;
  });
}

}  // extern "C"

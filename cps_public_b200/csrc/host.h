// host.h -- host-side objects of libcpsb200: device context, resident gauge
// fields, device spinor fields, the fermion operators and the solvers.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <complex>
#include <functional>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cpsb200.h"
#include "blas.h"
#include "cg_state.h"
#include "cpsb_kernels.h"

namespace cpsb {

// Thrown inside the library, converted to a status code at the C ABI.
struct Error {
  int code;
  std::string msg;
};
void check_cuda(cudaError_t e, const char *what);
#define CK(call) ::cpsb::check_cuda((call), #call)

struct Context {
  int device = -1;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
};
Context &ctx();

// Device allocation that remembers its size; freed on destruction.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  explicit DevBuf(size_t n);
  ~DevBuf();
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  void alloc(size_t n);
};

struct Gauge {
  int dims[4];
  int bc_t = 0;
  long n4cb = 0;
  DevBuf u64;          // 18 reals per link, BondCond applied
  DevBuf u32, u16;     // rows 0,1 per link (made on first use)
  DevBuf canon;        // CANONICAL copy kept for building reduced precisions
  bool recon_ok = false;
  double recon_err = 0;
  std::mutex mu;
  // Work items of the request loop (serve.cu) queued or running on this field;
  // cpsb_gauge_free refuses (CPSB_ERR_BUSY) while it is nonzero.
  std::atomic<int> inflight{0};
  GaugePtr ptr(int prec);
};

// A device spinor field in the chunked layout of cpsb_device.cuh.
struct Field {
  int prec = P64;
  long nsites = 0;
  DevBuf data, norm;
  Field() = default;
  Field(int prec, long nsites) { create(prec, nsites); }
  void create(int prec, long nsites);
  SpinorPtr ptr() const { return SpinorPtr{data.p, (float *)norm.p, nsites}; }
  // The entries [off, off + n) of the field as a field of its own: one
  // right-hand side of a multi-RHS field.  off is a multiple of 8 (a whole
  // number of 8-entry blocks; every right-hand side is, since n4cb is).
  SpinorPtr view(long off) const {
    const long chunks = prec == P64 ? 12 : prec == P32 ? 6 : 3;
    return SpinorPtr{(char *)data.p + off * chunks * 16, norm.p ? (float *)norm.p + off : nullptr, nsites - off};
  }
  size_t bytes() const { return data.bytes + norm.bytes; }
};
size_t field_bytes(int prec, long nsites);

// Geometry of the checkerboard fields of an operator on a lattice of dims:
// Ls slices (1 for Wilson), nrhs right-hand sides, DWF 5-D checkerboarding
// (five_d: two slice classes) or one class.
Geom make_geom(const int dims[4], int ls, int nrhs, bool five_d);

// Reduction slot: partials for every block of a launch, a ticket and results.
struct RedSlot {
  DevBuf buf;
  Reduce r(double *result);
  RedSlot();
};

struct Operator {
  Gauge *G;
  cpsb_dirac_params p;
  int prec;
  int nrhs;
  Geom geom;
  double kappa = 0;        // Wilson / DWF
  double kappa_b = 0;      // Mobius
  M5Coef m5c[2];           // Mobius M5^-1 coefficient sets (dag 0, dag 1)
  // zMobius: the per-slice coefficients (copied from the parameters) and the
  // m5z tables of the MatPc / MatPcDag stages of the three preconditioners, in
  // device memory
  std::vector<std::complex<double>> zb, zc;
  DevBuf ztab;
  Field t1, t2, t3;
  RedSlot red_inner;

  Operator(Gauge *G, const cpsb_dirac_params &p, int prec, int nrhs);
  long nsites() const { return geom.nsites; }
  // out = a * D(cb, dag) in [+ x] with optional |out|^2 into red.  Vectors are
  // views (SpinorPtr) with nsites() sites each; the Field forms pass whole fields.
  void hop(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, double a, const SpinorPtr *x,
           const Reduce *red, const int *skip, cudaStream_t st);
  // Mobius: the hop with the M5 operation that follows it fused in (launch_hop_m5):
  // dag 0 out = a mix(M5^-1 D in), dag 1 out = [x +] a M5^-dag(mix^dag(D^dag in)).
  // Returns false, launching nothing, where no fused form exists or fusion is
  // switched off (CPSB_M5_FUSE=0 in the environment).
  bool hop_m5(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, double a, const M5Coef &cf,
              const SpinorPtr *x, const Reduce *red, const int *skip, cudaStream_t st);
  bool fuse_m5 = true;
  // DiracOp::Dslash front end
  void dslash(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, cudaStream_t st);
  // out = MatPc in (dag 0) or MatPcDag in (dag 1); |out|^2 into red when given.
  void matpc(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red, const int *skip, cudaStream_t st);
  // out = MatPcDagMatPc in; |MatPc in|^2 into red when given.
  void mdagm(const SpinorPtr &out, const SpinorPtr &in, const Reduce *red, const int *skip, cudaStream_t st);
  void hop(const Field &out, const Field &in, int cb, int dag, double a, const Field *x, const Reduce *red,
           const int *skip, cudaStream_t st) {
    const SpinorPtr xp = x ? x->ptr() : SpinorPtr{};
    hop(out.ptr(), in.ptr(), cb, dag, a, x ? &xp : nullptr, red, skip, st);
  }
  void dslash(const Field &out, const Field &in, int cb, int dag, cudaStream_t st) {
    dslash(out.ptr(), in.ptr(), cb, dag, st);
  }
  void matpc(const Field &out, const Field &in, int dag, const Reduce *red, const int *skip, cudaStream_t st) {
    matpc(out.ptr(), in.ptr(), dag, red, skip, st);
  }
  void mdagm(const Field &out, const Field &in, const Reduce *red, const int *skip, cudaStream_t st) {
    mdagm(out.ptr(), in.ptr(), red, skip, st);
  }
  // MatPcDagMatPc p with the CG residual update fused into its last hop
  // (Wilson / DWF, every precision): |MatPc p|^2 -> red_d, then
  // r -= alpha (A p + shift p), |r|^2 and the recurrence scalars in S, and with
  // x given x += alpha p; A p is not stored (scratch receives it only while a
  // launch shape is being tuned).
  bool can_fuse_cg_r() const { return p.action == CPSB_WILSON || p.action == CPSB_DWF; }
  bool mobius_like() const { return p.action == CPSB_MOBIUS || p.action == CPSB_ZMOBIUS; }
  void matpc_zmobius(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red, const int *skip,
                     cudaStream_t st);
  void mdagm_cg_r(const SpinorPtr &scratch, const SpinorPtr &in, const Reduce *red_d, const int *skip, CgState *S,
                  const SpinorPtr &r, const Reduce *red_r, bool shifted, const SpinorPtr *x, cudaStream_t st);
  // Mobius pieces of DiracOpMobius::MatInv (SYM2): out = M5^-1 in
  // (zmobius_m5inv, dag 0); out = D4(cb) in (zmobius_dslash_4, dag 0);
  // out = x + f H5 in (zmobius_kappa_dslash_5_plus_cmplx with factor f, dag 0).
  void matpc_orig_sym1(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red, const int *skip,
                       cudaStream_t st);
  void mobius_m5inv(const SpinorPtr &out, const SpinorPtr &in, cudaStream_t st);
  void mobius_d4(const SpinorPtr &out, const SpinorPtr &in, int cb, cudaStream_t st);
  void mobius_hop5_add(const SpinorPtr &out, const SpinorPtr &in, const SpinorPtr &x, double f, cudaStream_t st);
  // Bytes one hop application must move (spinors in + out + links), for the roofline.
  double hop_bytes() const;
};

// Workspace and state of one CG solve (reused across solves with the same shape).
struct CgSolver {
  Gauge *G;
  cpsb_dirac_params p;
  int sloppy;
  int nrhs;
  std::unique_ptr<Operator> op64, opS;  // op64: one RHS (applied per RHS) when sloppy != P64
  Geom geom;                           // all right-hand sides
  Field x64, b64, r64;                // FP64 (x64/b64 are the caller's vectors packed; r64 = b - A x)
  Field rS, pS, ApS, xS;              // sloppy (xS is FP32 when sloppy is FP16)
  DevBuf state;                       // CgState
  CgState *hstate = nullptr;          // pinned mirror
  DevBuf scal;                        // misc per-RHS scalars
  double *hscal = nullptr;            // pinned: |b|^2 read back without its own synchronisation
  RedSlot red_d, red_r, red_p, red_misc;
  double shift = 0;                   // sigma of the solve in progress
  cudaGraphExec_t graph = nullptr;
  int graph_batch = 0;
  bool graph_shifted = false;
  bool graph_loop = false;            // the graph is a device-side loop of batches
  unsigned long long graph_nodes = 0;  // kernels per batch (per loop body)
  DevBuf loop;                        // LoopCtl
  LoopCtl *hloop = nullptr;           // pinned: [0] to the device, [1] read back
  DevBuf pcg_partial, pcg_bar;        // FP64 persistent loop: block partials; barrier words + error flag
  std::mutex busy;

  CgSolver(Gauge *G, const cpsb_dirac_params &p, int sloppy, int nrhs);
  ~CgSolver();
  // Solves with x64 (initial guess) and b64 already packed; fills res[nrhs].
  // stop_q: per-right-hand-side stop_rsd (nullptr: a.stop_rsd for all).
  int solve(const cpsb_cg_arg &a, cpsb_solve_result *res, cudaStream_t st, double sigma = 0.0,
            const double *stop_q = nullptr);

 private:
  void launch_batch(int k, cudaStream_t st);
  void run_batches(int batch, cudaStream_t st, const bool *done, bool any);
  // FP64 solves on small lattices: every iteration in one cooperative kernel
  // (cg_persistent.cu).  Returns false, launching nothing, where it does not apply.
  bool run_persistent(cudaStream_t st);
  void true_residual(double *rr_out, const double *bnorm, cudaStream_t st, const int *skip_h = nullptr,
                     const int *skip_d = nullptr);
};

int tuned_variant(const DslashArgs &A, int prec, int xpay, int norm, cudaStream_t st);

// Device-side iteration loops (graph_loop.cu): record(h) records one batch
// followed by a condition kernel for handle h into the body of a graph WHILE
// node; returns false where the driver has no conditional nodes (the caller
// then replays plain batches).  CPSB_GRAPH_LOOP=0 in the environment turns the
// loops off.
bool graph_loops_enabled();
bool build_loop_graph(cudaStream_t st, const std::function<void(cudaGraphConditionalHandle)> &record,
                      cudaGraphExec_t *exec, size_t *body_nodes);
cudaError_t launch_cg_loop_cond(cudaGraphConditionalHandle h, const CgState *S, LoopCtl *L, int nrhs, int any,
                                cudaStream_t st);
struct MsBatch;
cudaError_t launch_ms_loop_cond(cudaGraphConditionalHandle h, const MsBatch *B, LoopCtl *L, int nvec,
                                cudaStream_t st);

CgSolver *get_solver(Gauge *G, const cpsb_dirac_params &p, int sloppy, int nrhs);

// The persistent FP64 CG loop (cg_persistent.cu).  CPSB_PERSISTENT_CG in the
// environment: 0 off, 1 (default) for Wilson fields of at most PCG_AUTO_SITES
// entries (its direction-parallel form, faster than the graph loop there), 2
// for any action and any size that fits one cooperative launch.
constexpr long PCG_AUTO_SITES = 1L << 14;
constexpr size_t PCG_PARTIAL_SLOTS = (size_t)MAX_RHS * 148 * 16;
int persistent_cg_mode();
cudaError_t launch_persistent_cg(const DslashArgs &base, double mkappa2, SpinorPtr t1, SpinorPtr t2, SpinorPtr r,
                                 SpinorPtr p, SpinorPtr x, CgState *S, double *partial, size_t partial_slots,
                                 unsigned *bar_err, cudaStream_t st);

// refiner: the solver for the per-shift refinement of reduced-precision
// Krylov runs, one right-hand side per source vector (nullptr: the library's
// cached one, taken under its lock).
int multishift(Gauge *G, const cpsb_dirac_params &p, const cpsb_cg_arg &a, Field &b64, std::vector<Field> &x,
               const double *shift, int nshift, double *rsd, int type, const double *alpha, cpsb_solve_result *res,
               cudaStream_t st, CgSolver *refiner = nullptr);
// nvec source vectors with the same shifts solved together (multishift.cu):
// chi and every x[s] hold nvec x n sites; rsd[q * nshift + s]; res[nvec].
int multishift_multi(Gauge *G, const cpsb_dirac_params &p, const cpsb_cg_arg &a, int nvec, Field &chi,
                     std::vector<Field> &x, const double *shift, int nshift, double *rsd, int type,
                     const double *alpha, cpsb_solve_result *res, cudaStream_t st, CgSolver *refiner = nullptr);

}  // namespace cpsb

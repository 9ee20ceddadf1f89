// operator.cu -- device context, resident gauge fields, spinor fields and the
// Wilson / DWF / Mobius preconditioned operators built from the kernels.
//
// Operator composition restates CPS:
//  Wilson  MatPc = 1 - kappa^2 D_eo D_oe, kappa = 1/(2(m+4))
//          (d_op_wilson/noarch/wilson_m.C:49-85, d_op_wilson.C:134-137)
//  DWF     MatPc = 1 - kappa^2 D(cb=0) D(cb=1), kappa = 1/(2(4+a5_inv-M5)), D the
//          5-D hop (dwf_m.C:31-63, dwf_init.C:97-98)
//  Mobius  MatPc (SYM2) = 1 - kappa_b D4(0) M5^-1 kappa_b D4(1) M5^-1 with
//          kappa_b = 1/(2(b(4-M5)+a5_inv)), kappa_c = 1/(2(c(4-M5)-a5_inv))
//          (d_op_zmobius/noarch/zmobius_m-sym2.h:1-127, zmobius_mdag-sym2.h,
//          d_op_mobius/d_op_mobius.C:106-109)
//  MatPcDagMatPc = MatPcDag(MatPc in), |MatPc in|^2 fused into the MatPc pass
//          (dwf_mdagm.C:32-62, mobius_mdagm.C:33-60, wilson_mdagm.C:83-160).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>

#include "host.h"
#include "cg_state.h"

namespace cpsb {

void check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = (e == cudaErrorMemoryAllocation) ? CPSB_ERR_OOM : CPSB_ERR_CUDA;
  cudaGetLastError();  // clear a non-sticky error
  throw Error{code, std::string(what) + ": " + cudaGetErrorString(e)};
}

static std::atomic<unsigned long long> g_launches{0};
static thread_local bool t_capturing = false;
void count_launch(unsigned long long n) {
  if (!t_capturing) g_launches += n;
}
void set_capturing(bool on) { t_capturing = on; }
unsigned long long launch_count() { return g_launches.load(); }

Context &ctx() {
  static Context c;
  return c;
}

DevBuf::DevBuf(size_t n) { alloc(n); }
void DevBuf::alloc(size_t n) {
  if (p) {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  if (n == 0) return;
  CK(cudaMalloc(&p, n));
  bytes = n;
}
DevBuf::~DevBuf() {
  if (p) cudaFree(p);
}

size_t field_bytes(int prec, long nsites) {
  if (prec == P64) return (size_t)nsites * 192;
  if (prec == P32) return (size_t)nsites * 96;
  return (size_t)nsites * 48 + (size_t)nsites * 4;
}

Geom make_geom(const int dims[4], int ls, int nrhs, bool five_d) {
  Geom g;
  memset(&g, 0, sizeof(g));
  g.lx = dims[0];
  g.ly = dims[1];
  g.lz = dims[2];
  g.lt = dims[3];
  g.lxh = g.lx / 2;
  g.n4cb = g.lx * g.ly * g.lz * g.lt / 2;
  g.ls = ls;
  g.nrhs = nrhs;
  g.nsites = (long)g.n4cb * ls * nrhs;
  g.ncls = five_d ? 2 : 1;
  g.cs[0] = five_d ? (ls + 1) / 2 : ls;
  g.cs[1] = five_d ? ls / 2 : 0;
  g.kb1 = g.n4cb * g.cs[0];
  return g;
}

void Field::create(int pr, long n) {
  prec = pr;
  nsites = n;
  data.alloc((size_t)n * (pr == P64 ? 192 : pr == P32 ? 96 : 48));
  if (pr == P16) norm.alloc((size_t)n * 4);
  else norm.alloc(0);
}

RedSlot::RedSlot() {
  // partials: grid_blocks cap (148*16) * MAX_RHS; + ticket + padding
  const size_t nparts = 148 * 16 * MAX_RHS;
  buf.alloc(nparts * sizeof(double) + 256);
  // The ticket must be zero before the first kernel that uses the slot runs.
  // cudaMemset goes to the legacy stream, which does not order against the
  // library's non-blocking streams, so wait for it here.
  CK(cudaMemset(buf.p, 0, buf.bytes));
  CK(cudaStreamSynchronize(cudaStreamLegacy));
}
Reduce RedSlot::r(double *result) {
  Reduce q;
  q.partial = (double *)buf.p;
  q.ticket = (unsigned *)((char *)buf.p + 148 * 16 * MAX_RHS * sizeof(double));
  q.result = result;
  return q;
}

GaugePtr Gauge::ptr(int prec) {
  if (prec == P64) return GaugePtr{u64.p, n4cb};
  std::lock_guard<std::mutex> lk(mu);
  DevBuf &b = prec == P32 ? u32 : u16;
  if (!b.p) {
    if (!recon_ok)
      throw Error{CPSB_ERR_UNSUPPORTED,
                  "gauge field is not SU(3) to reduced-precision accuracy; recon-12 storage unavailable"};
    b.alloc((size_t)n4cb * 2 * 4 * (prec == P32 ? 48 : 24));
    CK(launch_gauge_pack(prec, b.p, (const double *)canon.p, dims, bc_t, ctx().stream));
    CK(cudaStreamSynchronize(ctx().stream));
  }
  return GaugePtr{b.p, n4cb};
}

// ----------------------------------------------------------------- Operator
static void m5_coefficients(double K, double mass, int ls, M5Coef *c0, M5Coef *c1) {
  // dag 0 (zmobius_m5inv.C:247-400 with K[s] = K for all s)
  memset(c0, 0, sizeof(M5Coef));
  memset(c1, 0, sizeof(M5Coef));
  double prod = 1.0;
  for (int i = 0; i < ls; i++) prod *= -K;
  prod *= mass;
  const double invd0 = 1.0 / (1.0 + prod);
  double fl = K * mass * invd0;
  for (int s = 0; s <= ls - 2; s++) {
    c0->f1[s] = fl;
    fl *= -K;
  }
  double pr = 1.0;
  for (int i = 0; i < ls - 1; i++) pr *= -K;
  double fr = -pr * mass * invd0;
  for (int s = ls - 2; s >= 0; s--) {
    c0->f2[s] = fr;
    fr /= -K;
  }
  c0->K = K;
  c0->invd = invd0;
  // dag 1 (zmobius_m5inv.C:534-686)
  prod = 1.0;
  for (int i = 0; i < ls; i++) prod *= K;
  prod *= mass;
  const double invd1 = 1.0 / (1.0 + prod);
  double fr1 = K * mass * invd1;
  for (int s = 0; s <= ls - 2; s++) {
    c1->f1[s] = fr1;
    fr1 *= -K;
  }
  pr = 1.0;
  for (int i = 0; i < ls - 2; i++) pr *= -K;
  pr *= -K;
  double fl1 = -pr * mass * invd1;
  for (int s = ls - 2; s >= 0; s--) {
    c1->f2[s] = fl1;
    if (s > 0) fl1 /= -K;
  }
  c1->K = K;
  c1->invd = invd1;
}

// zMobius (DiracOpZMobius with complex b_s, c_s): kappa_b(s) = 1/(2(b_s(4-M5)+a5_inv)),
// kappa_c(s) = 1/(2(c_s(4-M5)-a5_inv)), K_s = kappa_b(s)/kappa_c(s) (reset_mobius_arg,
// d_op_zmobius.C:246-295), and the four m5z tables of MatPc / MatPcDag (SYM2,
// zmobius_m-sym2.h, zmobius_mdag-sym2.h) in the step order of zmobius_m5inv.C:
//   dag 0  t1 = kb  . mix(M5^-1 in);  t3 = D_W(1) t1;
//          t1 = -kb . mix(M5^-1 t3);  out = in + D_W(0) t1
//   dag 1  t1 = D_W^dag(1) in;  t3 = conj(kb) . M5^-dag(mix^dag(-conj(kb) . t1));
//          t1 = D_W^dag(0) t3;  out = in + M5^-dag(mix^dag(t1))
// (the per-slice factors commute with the 4-D hop, which acts slice by slice).
typedef std::complex<double> zc_t;
static double2 d2(zc_t z) { return make_double2(z.real(), z.imag()); }

static void zmobius_sweeps(ZM5Tab &t, int dag, int ls, double m, const zc_t *K) {
  const zc_t one(1.0, 0.0);
  if (!dag) {
    zc_t prod = one;
    for (int i = 0; i < ls; i++) prod *= -K[i];
    prod *= m;
    const zc_t invd = one / (one + prod);
    // upper: chain first (v_{s+1} += -K_{s+1} v_s), walls from the last slice
    t.walls_first[0] = 0;
    for (int s = 0; s <= ls - 2; s++) t.a[0][s] = d2(-K[s + 1]);
    zc_t pr = one;
    for (int i = 0; i < ls - 1; i++) pr *= -K[i];
    zc_t fr = -(m * pr) * invd;
    for (int s = ls - 2; s >= 0; s--) {
      t.w[0][s] = d2(fr);
      fr /= -K[s];
    }
    t.invd[0] = d2(invd);
    // lower: walls first (v_last += f v_s), then v_s += -K_s v_{s+1}
    t.walls_first[1] = 1;
    zc_t fl = m * K[ls - 1] * invd;
    for (int s = 0; s <= ls - 2; s++) {
      t.w[1][s] = d2(fl);
      fl *= -K[s];
    }
    for (int s = 0; s <= ls - 2; s++) t.a[1][s] = d2(-K[s]);
    t.invd[1] = d2(invd);
  } else {
    zc_t prod = one;
    for (int i = 0; i < ls; i++) prod *= K[i];
    prod *= m;
    const zc_t invd = std::conj(one / (one + prod));
    // upper: walls first, then v_s += -conj(K_{s+1}) v_{s+1}
    t.walls_first[0] = 1;
    zc_t fr = m * std::conj(K[0]) * invd;
    for (int s = 0; s <= ls - 2; s++) {
      t.w[0][s] = d2(fr);
      fr *= -std::conj(K[s + 1]);
    }
    for (int s = 0; s <= ls - 2; s++) t.a[0][s] = d2(-std::conj(K[s + 1]));
    t.invd[0] = d2(invd);
    // lower: chain first (v_{s+1} += -conj(K_s) v_s), walls from the last slice
    t.walls_first[1] = 0;
    for (int s = 0; s <= ls - 2; s++) t.a[1][s] = d2(-std::conj(K[s]));
    zc_t pr = one;
    for (int i = 0; i < ls - 2; i++) pr *= -K[i];
    pr *= -K[ls - 1];
    zc_t fl = -(m * std::conj(pr)) * invd;
    for (int s = ls - 2; s >= 0; s--) {
      t.w[1][s] = d2(fl);
      if (s > 0) fl /= -std::conj(K[s - 1]);
    }
    t.invd[1] = d2(invd);
  }
  t.sweep = 1;
}

// b_s v_s + c-hop (zmobius_dslash_4.C:90-121 with zmobius_dslash_5_plus.C:125-376,
// dag 0) or its adjoint (dag 1: conj(b_s), conjugated and index-shifted c).
static void zmobius_mix(ZM5Tab &t, int dag, int ls, double m, const zc_t *b, const zc_t *c) {
  for (int s = 0; s < ls; s++) t.bb[s] = d2(dag ? std::conj(b[s]) : b[s]);
  if (!dag) {
    for (int s = 0; s < ls; s++) {
      t.cc[0][s] = d2(s == 0 ? -m * c[0] : c[s]);             // upper: from s-1
      t.cc[1][s] = d2(s == ls - 1 ? -m * c[ls - 1] : c[s]);   // lower: from s+1
    }
  } else {
    for (int s = 0; s < ls; s++) {
      t.cc[0][s] = d2(s == ls - 1 ? -m * std::conj(c[0]) : std::conj(c[s + 1]));  // upper: from s+1
      t.cc[1][s] = d2(s == 0 ? -m * std::conj(c[ls - 1]) : std::conj(c[s - 1]));  // lower: from s-1
    }
  }
  t.mix = 1;
}

static void zmobius_setup(Operator &op, const cpsb_dirac_params &pp) {
  const int ls = op.geom.ls;
  if (pp.pc_type < 0 || pp.pc_type > 5)
    throw Error{CPSB_ERR_UNSUPPORTED, "zMobius preconditioners: ZMOB_PC_ORIG .. ZMOB_PC_SYM3 (0 .. 5)"};
  if (!pp.zmobius_b || !pp.zmobius_c) throw Error{CPSB_ERR_ARG, "zMobius needs zmobius_b and zmobius_c"};
  op.zb.resize(ls);
  op.zc.resize(ls);
  std::vector<zc_t> kb(ls), K(ls);
  for (int s = 0; s < ls; s++) {
    op.zb[s] = zc_t(pp.zmobius_b[2 * s], pp.zmobius_b[2 * s + 1]);
    op.zc[s] = zc_t(pp.zmobius_c[2 * s], pp.zmobius_c[2 * s + 1]);
    kb[s] = 1.0 / (2.0 * (op.zb[s] * (4 - pp.m5) + pp.a5_inv));
    const zc_t kc = 1.0 / (2.0 * (op.zc[s] * (4 - pp.m5) - pp.a5_inv));
    K[s] = kb[s] / kc;
  }
  // Tables (the stage each one applies; kb, K per slice):
  //   0 dag0 kb . mix(M5^-1 .)        1 dag0 -kb . mix(M5^-1 .)     4 dag0 kb . mix(.)
  //   5 dag0 K-weighted H5 (b = 0)    6 dag0 M5^-1 alone
  //   2 dag1 conj(kb) . M5^-dag(mix^dag(-conj(kb) .))              3 dag1 M5^-dag(mix^dag(.))
  //   7 dag1 mix^dag alone            8 dag1 K-weighted H5^dag       9 dag1 -conj(kb) . M5^-dag(.)
  //  10 dag1 conj(kb) . M5^-dag(mix^dag(.))
  //  11 dag0 -(c_s (4 - M5) - a5_inv) .    12 dag0 (c_s / 2) .   (DiracOpZMobius::Dminus)
  //  13 dag0 2 kb .                          (the source scale of Fzmobius::FmatInv)
  //  MIT preconditioners (zmobius_B_MIT / zmobius_Binv_MIT, d_op_zmobius.C:132-238, f = c/b):
  //  14 dag0 B = b . (1 + f H5)   15 dag1 B^dag = (1 + f H5)^dag conj(b) .
  //  16 dag0 B^-1 = M5^-1[K = f] (1/b .)   17 dag1 B^-dag = 1/conj(b) . M5^-dag[K = f]
  //  18 dag0 mix(M5^-1 .) without a scale (SYM3)
  const int NT = 19;
  std::vector<ZM5Tab> t(NT);
  memset(t.data(), 0, sizeof(ZM5Tab) * NT);
  const std::vector<zc_t> zero(ls, zc_t(0.0, 0.0));
  auto dag_of = [](int k) {
    return (k == 0 || k == 1 || k == 4 || k == 5 || k == 6 || k == 11 || k == 12 || k == 13 || k == 14 || k == 16 ||
            k == 18) ? 0 : 1;
  };
  std::vector<zc_t> fact(ls), one(ls, zc_t(1.0, 0.0));
  for (int s = 0; s < ls; s++) fact[s] = op.zc[s] / op.zb[s];
  for (int k = 0; k < NT; k++) {
    const int dag = dag_of(k);
    if (k >= 11 && k <= 13) continue;  // scale-only tables
    if (k == 14 || k == 15) {  // B, B^dag: mixing 1 + f H5
      zmobius_mix(t[k], dag, ls, pp.mass, one.data(), fact.data());
      continue;
    }
    if (k == 16 || k == 17) {  // B^-1, B^-dag: sweeps with K = f
      zmobius_sweeps(t[k], dag, ls, pp.mass, fact.data());
      continue;
    }
    if (k != 4 && k != 5 && k != 7 && k != 8) zmobius_sweeps(t[k], dag, ls, pp.mass, K.data());
    if (k == 5 || k == 8) zmobius_mix(t[k], dag, ls, pp.mass, zero.data(), K.data());
    else if (k != 6 && k != 9) zmobius_mix(t[k], dag, ls, pp.mass, op.zb.data(), op.zc.data());
  }
  for (int s = 0; s < ls; s++) {
    t[11].post[s] = d2(-(op.zc[s] * (4 - pp.m5) - pp.a5_inv));
    t[12].post[s] = d2(0.5 * op.zc[s]);
    t[13].post[s] = d2(2.0 * kb[s]);
    t[14].post[s] = d2(op.zb[s]);
    t[15].pre[s] = d2(std::conj(op.zb[s]));
    t[16].pre[s] = d2(1.0 / op.zb[s]);
    t[17].post[s] = d2(1.0 / std::conj(op.zb[s]));
  }
  t[11].post_on = t[12].post_on = t[13].post_on = 1;
  t[14].post_on = t[15].pre_on = t[16].pre_on = t[17].post_on = 1;
  for (int s = 0; s < ls; s++) {
    t[0].post[s] = t[4].post[s] = d2(kb[s]);
    t[1].post[s] = d2(-kb[s]);
    t[2].pre[s] = t[9].post[s] = d2(-std::conj(kb[s]));
    t[2].post[s] = t[10].post[s] = d2(std::conj(kb[s]));
  }
  t[0].post_on = t[1].post_on = t[4].post_on = t[9].post_on = t[10].post_on = 1;
  t[2].pre_on = t[2].post_on = 1;
  op.ztab.alloc(sizeof(ZM5Tab) * NT);
  CK(cudaMemcpy(op.ztab.p, t.data(), sizeof(ZM5Tab) * NT, cudaMemcpyHostToDevice));
  op.kappa_b = kb[0].real();
}

Operator::Operator(Gauge *g, const cpsb_dirac_params &pp, int pr, int nr) : G(g), p(pp), prec(pr), nrhs(nr) {
  if (p.action < 0 || p.action > 3) throw Error{CPSB_ERR_ARG, "unknown action"};
  p.zmobius_b = p.zmobius_c = nullptr;  // the caller's arrays are read here only (zb, zc keep copies)
  const int ls = p.action == CPSB_WILSON ? 1 : p.ls;
  if (ls < 1 || ls > 64) throw Error{CPSB_ERR_ARG, "ls out of range"};
  if (nrhs < 1 || nrhs > MAX_RHS) throw Error{CPSB_ERR_ARG, "nrhs out of range"};
  geom = make_geom(G->dims, ls, nrhs, p.action == CPSB_DWF);
  if (const char *f = getenv("CPSB_M5_FUSE")) fuse_m5 = atoi(f) != 0;
  if (p.action == CPSB_WILSON) kappa = 1.0 / (2.0 * (p.mass + 4.0));
  if (p.action == CPSB_DWF) kappa = 1.0 / (2 * (4 + p.a5_inv - p.m5));
  if (mobius_like()) {
    const int ok[] = {4, 8, 12, 16, 20, 24, 32};
    bool found = false;
    for (int v : ok) found |= (v == ls);
    if (!found) throw Error{CPSB_ERR_UNSUPPORTED, "Mobius Ls must be one of 4,8,12,16,20,24,32"};
    t3.create(prec, geom.nsites);
  }
  if (p.action == CPSB_ZMOBIUS) zmobius_setup(*this, pp);
  if (p.action == CPSB_MOBIUS) {
    if (p.pc_type < 0 || p.pc_type > 2)
      throw Error{CPSB_ERR_UNSUPPORTED, "Mobius preconditioners: ZMOB_PC_ORIG (0), ZMOB_PC_SYM1 (1), ZMOB_PC_SYM2 (2)"};
    kappa_b = 1.0 / (2 * (p.mobius_b * (4 - p.m5) + p.a5_inv));
    const double kappa_c = 1.0 / (2 * (p.mobius_c * (4 - p.m5) - p.a5_inv));
    m5_coefficients(kappa_b / kappa_c, p.mass, ls, &m5c[0], &m5c[1]);
    for (int d = 0; d < 2; d++) {
      m5c[d].b = p.mobius_b;
      m5c[d].c = p.mobius_c;
      m5c[d].mass = p.mass;
      m5c[d].scale = 1.0;
    }
  }
  t1.create(prec, geom.nsites);
  t2.create(prec, geom.nsites);
}

double Operator::hop_bytes() const {
  const double spin = prec == P64 ? 192 : prec == P32 ? 96 : 52;
  const double link = prec == P64 ? 144 : prec == P32 ? 48 : 24;
  return 2.0 * spin * (double)geom.nsites + link * 4.0 * 2.0 * (double)geom.n4cb;
}

void Operator::hop(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, double a, const SpinorPtr *x,
                   const Reduce *red, const int *skip, cudaStream_t st) {
  DslashArgs A;
  memset(&A, 0, sizeof(A));
  A.g = geom;
  A.U = G->ptr(prec);
  A.in = in;
  A.out = out;
  if (x) A.x = *x;
  A.cb = cb;
  A.dag = dag;
  A.five_d = p.action == CPSB_DWF;
  A.hop5 = p.action == CPSB_DWF;
  A.hop5_fact = 2.0 * p.a5_inv;
  A.hop5_wall = -2.0 * p.mass * p.a5_inv;
  A.a = a;
  A.bc_t_sign = (prec != P64 && G->bc_t) ? -1.0 : 1.0;
  if (red) A.red = *red;
  A.skip = skip;
  const int v = tuned_variant(A, prec, x != nullptr, red != nullptr, st);
  CK(launch_dslash(prec, A, x != nullptr, red != nullptr, v, st));
}

bool Operator::hop_m5(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, double a, const M5Coef &cf,
                      const SpinorPtr *x, const Reduce *red, const int *skip, cudaStream_t st) {
  if (!fuse_m5 || p.action != CPSB_MOBIUS) return false;
  DslashArgs A;
  memset(&A, 0, sizeof(A));
  A.g = geom;
  A.U = G->ptr(prec);
  A.in = in;
  A.out = out;
  if (x) A.x = *x;
  A.cb = cb;
  A.dag = dag;
  A.a = a;
  A.bc_t_sign = (prec != P64 && G->bc_t) ? -1.0 : 1.0;
  if (red) A.red = *red;
  A.skip = skip;
  const cudaError_t e = launch_hop_m5(prec, A, cf, x != nullptr, red != nullptr, st);
  if (e == cudaErrorNotSupported) return false;
  CK(e);
  return true;
}

void Operator::dslash(const SpinorPtr &out, const SpinorPtr &in, int cb, int dag, cudaStream_t st) {
  if (p.action == CPSB_ZMOBIUS)
    throw Error{CPSB_ERR_UNSUPPORTED,
                "zMobius Dslash: DiracOpZMobius::Dslash is the unpreconditioned operator on full vectors"};
  if (p.action != CPSB_MOBIUS) {
    hop(out, in, cb, dag, 1.0, nullptr, nullptr, nullptr, st);
    return;
  }
  // mobius_dslash (d_op_mobius/noarch/mobius_dslash.C:23-43): D4 (zmobius_dslash_4)
  // plus the 5th-direction hop of the input with factor 1/kappa_c.
  M5Coef mix;
  memset(&mix, 0, sizeof(mix));
  mix.K = 0.0;
  mix.invd = 1.0;
  mix.b = p.mobius_b;
  mix.c = p.mobius_c;
  mix.mass = p.mass;
  mix.scale = 1.0;
  Reduce none;
  memset(&none, 0, sizeof(none));
  if (!dag) {
    CK(launch_m5(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, mix, 0, 0, none, nullptr, st));
    hop(out, t1.ptr(), cb, 0, 1.0, nullptr, nullptr, nullptr, st);
  } else {
    hop(t1.ptr(), in, cb, 1, 1.0, nullptr, nullptr, nullptr, st);
    CK(launch_m5(prec, 1, geom, out, t1.ptr(), SpinorPtr{}, mix, 0, 0, none, nullptr, st));
  }
  const double kappa_c = 1.0 / (2 * (p.mobius_c * (4 - p.m5) - p.a5_inv));
  M5Coef h5 = mix;
  h5.b = 0.0;
  h5.c = 1.0 / kappa_c;
  // out = out + H5(in): the m5 kernel in xpay mode (K = 0 makes the sweep the identity)
  CK(launch_m5(prec, dag, geom, out, in, out, h5, 1, 0, none, nullptr, st));
}

void Operator::matpc(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red, const int *skip,
                     cudaStream_t st) {
  if (p.action == CPSB_ZMOBIUS) {
    matpc_zmobius(out, in, dag, red, skip, st);
    return;
  }
  if (p.action != CPSB_MOBIUS) {
    hop(t1.ptr(), in, 1, dag, 1.0, nullptr, nullptr, skip, st);
    hop(out, t1.ptr(), 0, dag, -kappa * kappa, &in, red, skip, st);
    return;
  }
  Reduce none;
  memset(&none, 0, sizeof(none));
  if (p.pc_type != 2) {
    matpc_orig_sym1(out, in, dag, red, skip, st);
    return;
  }
  // Each hop that an M5 operation follows runs with it fused in where a fused
  // form exists (hop_m5: the M5 output scale folded into the hop's).
  if (!dag) {
    CK(launch_m5(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, m5c[0], 0, 0, none, skip, st));
    if (hop_m5(t3.ptr(), t1.ptr(), 1, 0, kappa_b * m5c[0].scale, m5c[0], nullptr, nullptr, skip, st)) {
      hop(out, t3.ptr(), 0, 0, -kappa_b, &in, red, skip, st);
      return;
    }
    hop(t3.ptr(), t1.ptr(), 1, 0, kappa_b, nullptr, nullptr, skip, st);
    CK(launch_m5(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, m5c[0], 0, 0, none, skip, st));
    hop(out, t1.ptr(), 0, 0, -kappa_b, &in, red, skip, st);
  } else {
    if (hop_m5(t3.ptr(), in, 1, 1, -kappa_b * kappa_b, m5c[1], nullptr, nullptr, skip, st) &&
        hop_m5(out, t3.ptr(), 0, 1, m5c[1].scale, m5c[1], &in, red, skip, st))
      return;
    hop(t1.ptr(), in, 1, 1, -kappa_b, nullptr, nullptr, skip, st);
    M5Coef c = m5c[1];
    c.scale = kappa_b;
    CK(launch_m5(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, c, 0, 0, none, skip, st));
    hop(t1.ptr(), t3.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
    CK(launch_m5(prec, 1, geom, out, t1.ptr(), in, m5c[1], 1, red != nullptr, red ? *red : none, skip,
                 st));
  }
}

// ZMOB_PC_ORIG (zmobius_m-orig.h:3-126, zmobius_mdag-orig.h) and ZMOB_PC_SYM1
// (zmobius_m-sym1.h, zmobius_mdag-sym1.h) from the same kernels as SYM2: the m5
// kernel with K = 0 is the D4 prefix b in + c H5 in (or, with b = 0, the
// 5th-direction hop alone), with b = 1, c = 0 it is M5^-1 alone.
//   ORIG  M    = in - kb D4(0) M5^-1 kb D4(1) in + (kb/kc) H5 in
//         M^dag = in + D4^dag(0) kb M5^-dag D4^dag(1) (-kb in) + (kb/kc) H5^dag in
//   SYM1  M    = in - M5^-1 kb D4(0) M5^-1 kb D4(1) in
//         M^dag = in + D4^dag(0) kb M5^-dag D4^dag(1) (-kb M5^-dag in)
// D4(cb) = hop(cb) (b + c H5) and D4^dag(cb) = (b + c H5)^dag hop^dag(cb)
// (zmobius_dslash_4.C:90-121, :176-202).
void Operator::matpc_orig_sym1(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red,
                               const int *skip, cudaStream_t st) {
  Reduce none;
  memset(&none, 0, sizeof(none));
  const bool orig = p.pc_type == 0;
  const double kc = 1.0 / (2 * (p.mobius_c * (4 - p.m5) - p.a5_inv));
  M5Coef mix;  // K = 0: identity sweeps, then the b/c mixing
  memset(&mix, 0, sizeof(mix));
  mix.invd = 1.0;
  mix.b = p.mobius_b;
  mix.c = p.mobius_c;
  mix.mass = p.mass;
  mix.scale = 1.0;
  M5Coef h5 = mix;  // (kb/kc) H5
  h5.b = 0.0;
  h5.c = kappa_b / kc;
  const Reduce rd = red ? *red : none;
  if (!dag) {
    CK(launch_m5(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, mix, 0, 0, none, skip, st));
    hop(t3.ptr(), t1.ptr(), 1, 0, kappa_b, nullptr, nullptr, skip, st);
    CK(launch_m5(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, m5c[0], 0, 0, none, skip, st));
    if (orig) {
      hop(out, t1.ptr(), 0, 0, -kappa_b, &in, nullptr, skip, st);
      CK(launch_m5(prec, 0, geom, out, in, out, h5, 1, red != nullptr, rd, skip, st));
    } else {
      hop(t3.ptr(), t1.ptr(), 0, 0, -kappa_b, nullptr, nullptr, skip, st);
      M5Coef inv = m5c[0];
      inv.b = 1.0;
      inv.c = 0.0;
      inv.scale = 1.0;
      CK(launch_m5(prec, 0, geom, out, t3.ptr(), in, inv, 1, red != nullptr, rd, skip, st));
    }
    return;
  }
  if (orig) {
    hop(t1.ptr(), in, 1, 1, -kappa_b, nullptr, nullptr, skip, st);
  } else {
    M5Coef inv = m5c[1];
    inv.b = 1.0;
    inv.c = 0.0;
    inv.scale = -kappa_b;
    CK(launch_m5(prec, 1, geom, t3.ptr(), in, SpinorPtr{}, inv, 0, 0, none, skip, st));
    hop(t1.ptr(), t3.ptr(), 1, 1, 1.0, nullptr, nullptr, skip, st);
  }
  M5Coef c = m5c[1];
  c.scale = kappa_b;
  CK(launch_m5(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, c, 0, 0, none, skip, st));
  hop(t1.ptr(), t3.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
  if (orig) {
    CK(launch_m5(prec, 1, geom, out, t1.ptr(), in, mix, 1, 0, none, skip, st));
    CK(launch_m5(prec, 1, geom, out, in, out, h5, 1, red != nullptr, rd, skip, st));
  } else {
    CK(launch_m5(prec, 1, geom, out, t1.ptr(), in, mix, 1, red != nullptr, rd, skip, st));
  }
}

void Operator::matpc_zmobius(const SpinorPtr &out, const SpinorPtr &in, int dag, const Reduce *red,
                             const int *skip, cudaStream_t st) {
  Reduce none;
  memset(&none, 0, sizeof(none));
  const ZM5Tab *t = (const ZM5Tab *)ztab.p;
  const Reduce rd = red ? *red : none;
  const int nr = red != nullptr;
  const int pc = p.pc_type;
  if (pc >= 3) {
    // SYM1_MIT (zmobius_m-sym1-MIT.h):  in + B M5^-1 (-kb) D4(0) M5^-1 kb D4(1) B^-1 in
    // SYM2_MIT (zmobius_m-sym2-MIT.h):  in + B (-kb) D4(0) M5^-1 kb D4(1) M5^-1 B^-1 in
    // SYM3 (zmobius_m-sym3.h):          in + D4(0) M5^-1 D4(1) M5^-1 in
    // and their adjoints (the mdag files), D4 = hop . mix, D4^dag = mix^dag . hop^dag.
    if (!dag) {
      if (pc == 5) {
        CK(launch_m5z(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, t + 18, 0, 0, none, skip, st));
        hop(t3.ptr(), t1.ptr(), 1, 0, 1.0, nullptr, nullptr, skip, st);
        CK(launch_m5z(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 18, 0, 0, none, skip, st));
        hop(out, t1.ptr(), 0, 0, 1.0, &in, red, skip, st);
        return;
      }
      CK(launch_m5z(prec, 0, geom, t3.ptr(), in, SpinorPtr{}, t + 16, 0, 0, none, skip, st));
      CK(launch_m5z(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + (pc == 3 ? 4 : 0), 0, 0, none, skip, st));
      hop(t3.ptr(), t1.ptr(), 1, 0, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 1, 0, 0, none, skip, st));
      hop(t3.ptr(), t1.ptr(), 0, 0, 1.0, nullptr, nullptr, skip, st);
      if (pc == 3) {
        CK(launch_m5z(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 6, 0, 0, none, skip, st));
        CK(launch_m5z(prec, 0, geom, out, t1.ptr(), in, t + 14, 1, nr, rd, skip, st));
      } else {
        CK(launch_m5z(prec, 0, geom, out, t3.ptr(), in, t + 14, 1, nr, rd, skip, st));
      }
      return;
    }
    if (pc == 5) {
      hop(t1.ptr(), in, 1, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, t + 3, 0, 0, none, skip, st));
      hop(t1.ptr(), t3.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, out, t1.ptr(), in, t + 3, 1, nr, rd, skip, st));
      return;
    }
    CK(launch_m5z(prec, 1, geom, t3.ptr(), in, SpinorPtr{}, t + 15, 0, 0, none, skip, st));
    if (pc == 3) {
      CK(launch_m5z(prec, 1, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 9, 0, 0, none, skip, st));
      hop(t3.ptr(), t1.ptr(), 1, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 10, 0, 0, none, skip, st));
      hop(t3.ptr(), t1.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 7, 0, 0, none, skip, st));
    } else {
      hop(t1.ptr(), t3.ptr(), 1, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, t + 2, 0, 0, none, skip, st));
      hop(t1.ptr(), t3.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, t + 3, 0, 0, none, skip, st));
    }
    CK(launch_m5z(prec, 1, geom, out, pc == 3 ? t1.ptr() : t3.ptr(), in, t + 17, 1, nr, rd, skip, st));
    return;
  }
  if (!dag) {
    // SYM2 (zmobius_m-sym2.h): in - kb D4(0) M5^-1 kb D4(1) M5^-1 in
    // ORIG (zmobius_m-orig.h): in - kb D4(0) M5^-1 kb D4(1) in + K H5 in
    // SYM1 (zmobius_m-sym1.h): in - M5^-1 kb D4(0) M5^-1 kb D4(1) in
    CK(launch_m5z(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, t + (pc == 2 ? 0 : 4), 0, 0, none, skip, st));
    hop(t3.ptr(), t1.ptr(), 1, 0, 1.0, nullptr, nullptr, skip, st);
    CK(launch_m5z(prec, 0, geom, t1.ptr(), t3.ptr(), SpinorPtr{}, t + 1, 0, 0, none, skip, st));
    if (pc == 2) {
      hop(out, t1.ptr(), 0, 0, 1.0, &in, red, skip, st);
    } else if (pc == 0) {
      hop(out, t1.ptr(), 0, 0, 1.0, &in, nullptr, skip, st);
      CK(launch_m5z(prec, 0, geom, out, in, out, t + 5, 1, nr, rd, skip, st));
    } else {
      hop(t3.ptr(), t1.ptr(), 0, 0, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 0, geom, out, t3.ptr(), in, t + 6, 1, nr, rd, skip, st));
    }
  } else {
    // the adjoints (zmobius_mdag-sym2.h, -orig.h, -sym1.h)
    if (pc == 1) {
      CK(launch_m5z(prec, 1, geom, t3.ptr(), in, SpinorPtr{}, t + 9, 0, 0, none, skip, st));
      hop(t1.ptr(), t3.ptr(), 1, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, t + 10, 0, 0, none, skip, st));
    } else {
      hop(t1.ptr(), in, 1, 1, 1.0, nullptr, nullptr, skip, st);
      CK(launch_m5z(prec, 1, geom, t3.ptr(), t1.ptr(), SpinorPtr{}, t + 2, 0, 0, none, skip, st));
    }
    hop(t1.ptr(), t3.ptr(), 0, 1, 1.0, nullptr, nullptr, skip, st);
    if (pc == 2) {
      CK(launch_m5z(prec, 1, geom, out, t1.ptr(), in, t + 3, 1, nr, rd, skip, st));
    } else if (pc == 0) {
      CK(launch_m5z(prec, 1, geom, out, t1.ptr(), in, t + 7, 1, 0, none, skip, st));
      CK(launch_m5z(prec, 1, geom, out, in, out, t + 8, 1, nr, rd, skip, st));
    } else {
      CK(launch_m5z(prec, 1, geom, out, t1.ptr(), in, t + 7, 1, nr, rd, skip, st));
    }
  }
}

void Operator::mobius_m5inv(const SpinorPtr &out, const SpinorPtr &in, cudaStream_t st) {
  M5Coef c = m5c[0];
  c.b = 1.0;  // no mixing after the sweeps
  c.c = 0.0;
  c.scale = 1.0;
  Reduce none;
  memset(&none, 0, sizeof(none));
  CK(launch_m5(prec, 0, geom, out, in, SpinorPtr{}, c, 0, 0, none, nullptr, st));
}

void Operator::mobius_d4(const SpinorPtr &out, const SpinorPtr &in, int cb, cudaStream_t st) {
  M5Coef mix;  // K = 0: the sweeps are the identity, leaving b in + c H5 in
  memset(&mix, 0, sizeof(mix));
  mix.invd = 1.0;
  mix.b = p.mobius_b;
  mix.c = p.mobius_c;
  mix.mass = p.mass;
  mix.scale = 1.0;
  Reduce none;
  memset(&none, 0, sizeof(none));
  CK(launch_m5(prec, 0, geom, t1.ptr(), in, SpinorPtr{}, mix, 0, 0, none, nullptr, st));
  hop(out, t1.ptr(), cb, 0, 1.0, nullptr, nullptr, nullptr, st);
}

void Operator::mobius_hop5_add(const SpinorPtr &out, const SpinorPtr &in, const SpinorPtr &x, double f,
                               cudaStream_t st) {
  M5Coef h;
  memset(&h, 0, sizeof(h));
  h.invd = 1.0;
  h.b = 0.0;
  h.c = f;
  h.mass = p.mass;
  h.scale = 1.0;
  Reduce none;
  memset(&none, 0, sizeof(none));
  CK(launch_m5(prec, 0, geom, out, in, x, h, 1, 0, none, nullptr, st));
}

void Operator::mdagm_cg_r(const SpinorPtr &scratch, const SpinorPtr &in, const Reduce *red_d, const int *skip,
                          CgState *S, const SpinorPtr &r, const Reduce *red_r, bool shifted, const SpinorPtr *x,
                          cudaStream_t st) {
  if (!can_fuse_cg_r()) throw Error{CPSB_ERR_UNSUPPORTED, "fused residual update needs the Wilson or DWF operator"};
  matpc(t2.ptr(), in, 0, red_d, skip, st);  // |MatPc p|^2 -> d
  hop(t1.ptr(), t2.ptr(), 1, 1, 1.0, nullptr, nullptr, skip, st);
  // the last hop of MatPcDag: out = t2 - kappa^2 D t1 = A p, consumed in registers
  DslashArgs A;
  memset(&A, 0, sizeof(A));
  A.g = geom;
  A.U = G->ptr(prec);
  A.in = t1.ptr();
  A.out = scratch;
  A.x = t2.ptr();
  A.cb = 0;
  A.dag = 1;
  A.five_d = p.action == CPSB_DWF;
  A.hop5 = p.action == CPSB_DWF;
  A.hop5_fact = 2.0 * p.a5_inv;
  A.hop5_wall = -2.0 * p.mass * p.a5_inv;
  A.a = -kappa * kappa;
  A.bc_t_sign = G->bc_t ? -1.0 : 1.0;
  A.skip = skip;
  // launch shape of the same hop without the fused update (tuned on the scratch output)
  const int v = tuned_variant(A, prec, 1, 0, st);
  A.red = *red_r;
  A.cg = S;
  A.cg_r = r;
  A.cg_p = in;
  A.cg_shift = shifted ? 1 : 0;
  if (x) A.cg_x = *x;
  CK(launch_dslash(prec, A, 1, 1, v, st));
}

void Operator::mdagm(const SpinorPtr &out, const SpinorPtr &in, const Reduce *red, const int *skip, cudaStream_t st) {
  matpc(t2.ptr(), in, 0, red, skip, st);
  matpc(out, t2.ptr(), 1, nullptr, skip, st);
}

}  // namespace cpsb

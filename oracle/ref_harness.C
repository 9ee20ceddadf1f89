// ref_harness.C -- TEST INFRASTRUCTURE ONLY (the oracle, never the product).
//
// A small driver, written for this project, that runs the *unmodified* CPS
// noarch fermion-matrix code (compiled from the reference sources by
// oracle/build_ref.sh) on fields supplied from a file, and writes the results
// back to a file.  It is used to generate the golden fixtures under
// tests/golden/ and to pin the C restatement in oracle/cps_oracle.c.
//
// Calls made into CPS (reference paths relative to cps_pp/):
//   Start / GJP.Initialize / GJP.InitializeExt      src/util/gjp/gjp.C
//   GwilsonFwilson / GwilsonFdwf / GwilsonFmobius  include/util/lattice/lattice_types.h:400,438,455
//   DiracOp*::Dslash / MatPc / MatPcDag / MatPcDagMatPc
//        d_op_wilson/noarch/d_op_wilson.C:150-240, d_op_dwf/d_op_dwf.C:174-300,
//        d_op_mobius/d_op_mobius.C:198-372
//   DiracOp::InvCgShift                             d_op_base/comsrc/inv_cg.C:84-447
//     (exactly what Lattice::FmatEvlInv reaches through InvCg(&true_res); the
//      4-argument InvCg wrapper at inv_cg.C:449-454 has no return statement, so
//      it is bypassed here)
//   Lattice::FmatEvlInv                             f_dwf_base.C:189-209, f_mobius.C:582, f_wilson.C:159
//   Lattice::FmatEvlMInv -> DiracOp::MInvCG         f_dwf_base.C:232-270, minvcg.C:47-353
//   DiracOp*::MatInv (full-lattice solve)           d_op_wilson.C:257-334, d_op_dwf.C:316-507,
//                                                   d_op_mobius.C:389-640
//   DiracOp::MinResExt (chronological guess)        d_op_base/comsrc/minresext.C:32-156
//   DiracOpMobius::Dminus                           d_op_mobius/d_op_mobius.C:745-777
//   Fmobius::FmatInv(..., dminus)                   lattice/f_mobius/f_mobius.C:45-117
//   Lattice::Fconvert (fermion storage order)       lattice/convert/convert.C:444-570 (Wilson),
//                                                   :635-1010 (DWF / Mobius)
//   zmobius_m5inv / zmobius_dslash_4                d_op_zmobius/noarch/zmobius_m5inv.C:807-845,
//                                                   zmobius_dslash_4.C:210-221
//
// Protocol (little endian):
//   request  = int64 hdr[32], double par[32], gauge (V*4*18 doubles, CANONICAL
//              order: site x+lx*(y+ly*(z+lz*t)), link mu, row-major 3x3 complex),
//              then op-specific doubles (see below).
//   response = int64 rhdr[8], double rpar[64], then op-specific doubles.
//   hdr: 0 op, 1 action (0 Wilson, 1 DWF, 2 Mobius, 3 zMobius), 2..5 lx ly lz lt, 6 ls,
//        7 cb, 8 dag, 9 max_iter, 10 nshift, 11 multishift type (0 MULTI,
//        1 SINGLE), 12 zmobius pc type, 13 t boundary (0 periodic, 1 antiperiodic),
//        14 repetitions (OP_BENCH: MatPcDagMatPc applied this many times),
//        15 fermion order for OP_FCONVERT (0 WILSON, 1 DWF_4D_EOPREC_EE),
//        16 OP_FCONVERT direction (0 CANONICAL -> order, 1 order -> CANONICAL),
//        17 OP_MINRESEXT degree (number of previous solutions),
//        18 OP_FMATINV dminus flag,
//        19, 20 (the build with the B200 bridge, -DUSE_B200, only) the bridge's
//        inner precision of FmatEvlInv / FmatInv and of FmatEvlMInv (-1: its default)
//   rpar[44] = device kernels the B200 library launched during the request
//   (-DUSE_B200 builds; 0 otherwise)
//   rpar[10] = wall seconds spent inside the timed CPS call(s) (MINVCG: rpar[42],
//   since rpar[0..nshift) holds the per-shift residuals); OP_BENCH also
//   returns the start and end of that window (steady clock, seconds) in
//   rpar[11], rpar[12], so that concurrent processes can be checked for overlap
//   par: 0 mass, 1 M5 (dwf_height), 2 a5_inv, 3 mobius b, 4 mobius c, 5 stop_rsd,
//        8.. shifts[nshift], 24.. unused
//   zMobius (action 3) only: 4*ls doubles right after par, before the gauge:
//        b_s as (re, im) pairs for s = 0..ls-1, then c_s likewise
//        (DoArgExt zmobius_b_coeff / zmobius_c_coeff, src/util/gjp/gjp.C:167-178)
#include <config.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <vector>
#include <chrono>
#include <util/lattice.h>
#include <util/gjp.h>
#include <util/verbose.h>
#include <util/dirac_op.h>
#include <util/dwf.h>
#include <util/zmobius.h>
#include <util/error.h>
#include <alg/do_arg.h>
#include <alg/cg_arg.h>
#ifdef USE_B200
#include <util/b200_bridge.h>
#endif

USING_NAMESPACE_CPS

enum { OP_DSLASH = 1, OP_MATPC = 2, OP_MDAGM = 3, OP_INVCG = 4, OP_MINVCG = 5,
       OP_M5INV = 6, OP_MOBIUS_D4 = 7, OP_BENCH = 8, OP_MATINV = 9, OP_FCONVERT = 10,
       OP_MINRESEXT = 11, OP_DMINUS = 12, OP_FMATINV = 13, OP_FMATEVLINV = 14 };

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void die(const char *m) { fprintf(stderr, "cpsref: %s\n", m); exit(2); }
static void trace(const char *m) { if (getenv("CPSREF_TRACE")) fprintf(stderr, "cpsref: %s\n", m); }

static void read_all(FILE *f, void *p, size_t n) {
  if (n && fread(p, 1, n, f) != n) die("short read");
}
static void write_all(FILE *f, const void *p, size_t n) {
  if (n && fwrite(p, 1, n, f) != n) die("short write");
}

// Applies one operator of a concrete DiracOp (MatPcDag is not virtual in CPS).
template <class D>
static double apply_op(D &d, int op, Vector *out, Vector *in, int cb, int dag) {
  Float dot = 0;
  if (op == OP_DSLASH) d.Dslash(out, in, (ChkbType)cb, (DagType)dag);
  else if (op == OP_MATPC) { if (dag) d.MatPcDag(out, in); else d.MatPc(out, in); }
  else d.MatPcDagMatPc(out, in, &dot);
  return dot;
}

// DiracOpZMobius's constructor (d_op_zmobius.C:315-368) resets the kappa arrays
// but never fills Dwf::zmobius_b / zmobius_c, which zmobius_dslash_4 reads
// (zmobius_dslash_4.C:61-62, :151-152); only DiracOpMobius fills them
// (d_op_mobius.C:111-118), so as shipped every zMobius checkerboard operator
// dereferences empty arrays.  The harness copies GJP's zMobius coefficients
// into the lattice's Dwf struct once (what the disabled branch at
// zmobius_dslash_4.C:64-65 reads), so the reference's zMobius kernels run on
// the coefficients the job set.
static void fill_zmobius_coefficients(Lattice &lat, int ls) {
  Dwf *arg = (Dwf *)lat.FdiracOpInitPtr();
  arg->zmobius_b.assign(GJP.ZMobius_b(), GJP.ZMobius_b() + ls);
  arg->zmobius_c.assign(GJP.ZMobius_c(), GJP.ZMobius_c() + ls);
}

int main(int argc, char **argv) {
  if (argc != 3) { fprintf(stderr, "usage: cpsref request.bin response.bin\n"); return 2; }
  FILE *fi = fopen(argv[1], "rb");
  if (!fi) die("cannot open request");
  int64_t hdr[32]; double par[32];
  read_all(fi, hdr, sizeof hdr);
  read_all(fi, par, sizeof par);
  const int op = (int)hdr[0], action = (int)hdr[1];
  const int lx = hdr[2], ly = hdr[3], lz = hdr[4], lt = hdr[5];
  const int ls = action == 0 ? 1 : (int)hdr[6];
  const int cb = hdr[7], dag = hdr[8], max_iter = hdr[9], nshift = hdr[10];
  const size_t vol = (size_t)lx * ly * lz * lt;
  const size_t fsz = vol / 2 * 24 * ls;   // one checkerboard, doubles

  int pargc = 1; char *pargv0 = argv[0]; char **pargv = &pargv0;
  trace("start");
  Start(&pargc, &pargv);

  DoArg do_arg;
  do_arg.x_sites = lx; do_arg.y_sites = ly; do_arg.z_sites = lz; do_arg.t_sites = lt;
  do_arg.s_sites = ls;
  do_arg.x_node_sites = lx; do_arg.y_node_sites = ly; do_arg.z_node_sites = lz;
  do_arg.t_node_sites = lt; do_arg.s_node_sites = ls;
  do_arg.x_nodes = do_arg.y_nodes = do_arg.z_nodes = do_arg.t_nodes = do_arg.s_nodes = 1;
  do_arg.x_bc = do_arg.y_bc = do_arg.z_bc = BND_CND_PRD;
  do_arg.t_bc = hdr[13] ? BND_CND_APRD : BND_CND_PRD;
  do_arg.start_conf_kind = START_CONF_ORD;
  do_arg.start_seed_kind = START_SEED_FIXED;
  do_arg.dwf_height = par[1];
  do_arg.dwf_a5_inv = par[2];
  do_arg.verbose_level = 0;
  DoArgExt ext;
  ext.mobius_b_coeff = par[3];
  ext.mobius_c_coeff = par[4];
  // DoArgExt's constructor leaves the zMobius coefficient arrays uninitialised
  // (src/alg/alg_arg/do_arg_init.C:75-93); empty them so InitializeExt skips them,
  // except for zMobius, which reads its b_s, c_s from them.
  ext.zmobius_b_coeff.zmobius_b_coeff_len = 0;
  ext.zmobius_b_coeff.zmobius_b_coeff_val = 0;
  ext.zmobius_c_coeff.zmobius_c_coeff_len = 0;
  ext.zmobius_c_coeff.zmobius_c_coeff_val = 0;
  std::vector<double> zb(2 * ls), zc(2 * ls);
  if (action == 3) {
    read_all(fi, zb.data(), zb.size() * sizeof(double));
    read_all(fi, zc.data(), zc.size() * sizeof(double));
    ext.zmobius_b_coeff.zmobius_b_coeff_len = 2 * ls;
    ext.zmobius_b_coeff.zmobius_b_coeff_val = zb.data();
    ext.zmobius_c_coeff.zmobius_c_coeff_len = 2 * ls;
    ext.zmobius_c_coeff.zmobius_c_coeff_val = zc.data();
  }
  trace("gjp");
  GJP.Initialize(do_arg);
  GJP.InitializeExt(ext);
  VRB.Level(VERBOSE_NONE_LEVEL);
  if (action >= 2) GJP.ZMobius_PC_Type((ZMobiusPCType)hdr[12]);

  Lattice *latp = 0;
  if (action == 0) latp = new GwilsonFwilson;
  else if (action == 1) latp = new GwilsonFdwf;
  else if (action == 2) latp = new GwilsonFmobius;
  else if (action == 3) latp = new GwilsonFzmobius;
  else die("bad action");
  Lattice &lat = *latp;
  if (action == 3) fill_zmobius_coefficients(lat, ls);  // kept by the lattice's Dwf struct
  trace("lattice");
  read_all(fi, (void *)lat.GaugeField(), vol * 4 * 18 * sizeof(double));

  trace("gauge");
  CgArg cg_arg;
  cg_arg.mass = par[0];
  cg_arg.stop_rsd = par[5];
  cg_arg.max_num_iter = max_iter;
  cg_arg.Inverter = CG;

  int64_t rhdr[8] = {0}; double rpar[64] = {0};
#ifdef USE_B200
  if (hdr[19] >= 0 || hdr[20] >= 0)
    b200_set_precision(hdr[19] >= 0 ? (int)hdr[19] : CPSB_PREC_F16, hdr[20] >= 0 ? (int)hdr[20] : CPSB_PREC_F32);
  unsigned long long launches0 = 0, launches1 = 0;
  cpsb_kernel_launches(&launches0);
#endif
  std::vector<double> out_payload;

  Vector *in = (Vector *)smalloc(fsz * sizeof(double));
  Vector *out = (Vector *)smalloc(fsz * sizeof(double));
  memset(out, 0, fsz * sizeof(double));

  if (op == OP_DSLASH || op == OP_MATPC || op == OP_MDAGM || op == OP_M5INV ||
      op == OP_MOBIUS_D4) {
    read_all(fi, in, fsz * sizeof(double));
    if (op == OP_M5INV || op == OP_MOBIUS_D4) {
      if (action < 2) die("M5INV / MOBIUS_D4 need the Mobius or zMobius action");
      DiracOp *dp = action == 2 ? (DiracOp *)new DiracOpMobius(lat, out, in, &cg_arg, CNV_FRM_NO)
                                : (DiracOp *)new DiracOpZMobius(lat, out, in, &cg_arg, CNV_FRM_NO);
      Dwf *arg = (Dwf *)lat.FdiracOpInitPtr();
      if (op == OP_M5INV)
        zmobius_m5inv(out, in, cg_arg.mass, dag, arg, arg->zmobius_kappa_ratio.data());
      else
        zmobius_dslash_4(out, (Matrix *)lat.GaugeField(), in, cb, dag, arg, cg_arg.mass);
      delete dp;
    } else if (action == 3) {
      // DiracOpZMobius::Dslash is the unpreconditioned operator on full
      // vectors; only MatPc / MatPcDag / MatPcDagMatPc are checkerboard operators.
      if (op == OP_DSLASH) die("zMobius Dslash is not a checkerboard operator");
      trace("zmobius ctor");
      DiracOpZMobius d(lat, out, in, &cg_arg, CNV_FRM_NO);
      trace("zmobius op");
      rpar[0] = apply_op(d, op, out, in, cb, dag);
      trace("zmobius done");
    } else if (action == 0) {
      DiracOpWilson d(lat, out, in, &cg_arg, CNV_FRM_NO);
      rpar[0] = apply_op(d, op, out, in, cb, dag);
    } else if (action == 1) {
      DiracOpDwf d(lat, out, in, &cg_arg, CNV_FRM_NO);
      rpar[0] = apply_op(d, op, out, in, cb, dag);
    } else {
      DiracOpMobius d(lat, out, in, &cg_arg, CNV_FRM_NO);
      rpar[0] = apply_op(d, op, out, in, cb, dag);
    }
    out_payload.assign((double *)out, (double *)out + fsz);
  } else if (op == OP_BENCH) {
    read_all(fi, in, fsz * sizeof(double));
    const int reps = (int)hdr[14];
    double t0 = 0, t1 = 0;
    Float dot = 0;
    if (action == 0) {
      DiracOpWilson d(lat, out, in, &cg_arg, CNV_FRM_NO);
      t0 = now_s(); for (int i = 0; i < reps; i++) d.MatPcDagMatPc(out, in, &dot); t1 = now_s();
    } else if (action == 1) {
      DiracOpDwf d(lat, out, in, &cg_arg, CNV_FRM_NO);
      t0 = now_s(); for (int i = 0; i < reps; i++) d.MatPcDagMatPc(out, in, &dot); t1 = now_s();
    } else {
      DiracOpMobius d(lat, out, in, &cg_arg, CNV_FRM_NO);
      t0 = now_s(); for (int i = 0; i < reps; i++) d.MatPcDagMatPc(out, in, &dot); t1 = now_s();
    }
    rpar[0] = dot; rpar[10] = t1 - t0; rhdr[0] = reps;
    rpar[11] = t0; rpar[12] = t1;  // the timed window on the system-wide monotonic clock
    out_payload.assign((double *)out, (double *)out + fsz);
  } else if (op == OP_INVCG) {
    read_all(fi, in, fsz * sizeof(double));          // source
    read_all(fi, out, fsz * sizeof(double));         // initial guess
    DiracOp *d = 0;
    if (action == 0) d = new DiracOpWilson(lat, out, in, &cg_arg, CNV_FRM_NO);
    else if (action == 1) d = new DiracOpDwf(lat, out, in, &cg_arg, CNV_FRM_NO);
    else if (action == 2) d = new DiracOpMobius(lat, out, in, &cg_arg, CNV_FRM_NO);
    else d = new DiracOpZMobius(lat, out, in, &cg_arg, CNV_FRM_NO);
    Float true_res = 0;
    double t0 = now_s();
    int iters = d->InvCgShift(out, in, 0.0, &true_res, NULL);
    rpar[10] = now_s() - t0;
    delete d;
    rhdr[0] = iters; rpar[0] = true_res;
    out_payload.assign((double *)out, (double *)out + fsz);
  } else if (op == OP_FMATEVLINV) {
    // Lattice::FmatEvlInv (the entry point CPS's algorithms call), source and guess in
    read_all(fi, in, fsz * sizeof(double));
    read_all(fi, out, fsz * sizeof(double));
    Float true_res = 0;
    double t0 = now_s();
    rhdr[0] = lat.FmatEvlInv(out, in, &cg_arg, &true_res, CNV_FRM_NO);
    rpar[10] = now_s() - t0;
    rpar[0] = true_res;
    out_payload.assign((double *)out, (double *)out + fsz);
  } else if (op == OP_MINVCG) {
    read_all(fi, in, fsz * sizeof(double));
    if (nshift < 1 || nshift > 16) die("nshift out of range");
    const int type = (int)hdr[11];
    std::vector<double> alpha(nshift), rsd(nshift);
    read_all(fi, rsd.data(), nshift * sizeof(double));
    read_all(fi, alpha.data(), nshift * sizeof(double));
    std::vector<Vector *> sol(nshift);
    for (int s = 0; s < nshift; s++) {
      sol[s] = (Vector *)smalloc(fsz * sizeof(double));
      memset(sol[s], 0, fsz * sizeof(double));
    }
    std::vector<CgArg> args(nshift);
    std::vector<CgArg *> argp(nshift);
    for (int s = 0; s < nshift; s++) {
      args[s] = cg_arg; args[s].stop_rsd = rsd[s]; argp[s] = &args[s];
    }
    double t0 = now_s();
    int iters = 0;
    if (action == 3) {
      // Fzmobius inherits FdwfBase::FmatEvlMInv (f_dwf_base.C:232-270), which
      // builds a DiracOpDwf: the zMobius multishift is DiracOp::MInvCG on a
      // DiracOpZMobius, called here as FmatEvlMInv calls it.
      DiracOpZMobius d(lat, sol[0], in, argp[0], CNV_FRM_NO);
      const Float dot = in->NormSqGlbSum(fsz);
      iters = d.MInvCG(sol.data(), in, dot, par + 8, nshift, 0, rsd.data(), type == 1 ? SINGLE : MULTI,
                       alpha.data());
      for (int s = 0; s < nshift; s++) args[s].true_rsd = rsd[s];
    } else {
      iters = lat.FmatEvlMInv(sol.data(), in, par + 8, nshift, 0, argp.data(), CNV_FRM_NO,
                              type == 1 ? SINGLE : MULTI, alpha.data());
    }
    rpar[10 + 32] = now_s() - t0;
    rhdr[0] = iters;
    for (int s = 0; s < nshift; s++) rpar[s] = args[s].true_rsd;
    const int nvec = type == 1 ? 1 : nshift;
    for (int s = 0; s < nvec; s++)
      out_payload.insert(out_payload.end(), (double *)sol[s], (double *)sol[s] + fsz);
  } else if (op == OP_MATINV) {
    // full-lattice source and initial guess (2 checkerboards each, in the
    // action's full-vector order); MatInv with the source preserved.
    Vector *fin = (Vector *)smalloc(2 * fsz * sizeof(double));
    Vector *fout = (Vector *)smalloc(2 * fsz * sizeof(double));
    read_all(fi, fin, 2 * fsz * sizeof(double));
    read_all(fi, fout, 2 * fsz * sizeof(double));
    DiracOp *d = 0;
    if (action == 0) d = new DiracOpWilson(lat, fout, fin, &cg_arg, CNV_FRM_NO);
    else if (action == 1) d = new DiracOpDwf(lat, fout, fin, &cg_arg, CNV_FRM_NO);
    else if (action == 2) d = new DiracOpMobius(lat, fout, fin, &cg_arg, CNV_FRM_NO);
    else d = new DiracOpZMobius(lat, fout, fin, &cg_arg, CNV_FRM_NO);  // d_op_zmobius.C:829-1080
    Float true_res = 0;
    double t0 = now_s();
    rhdr[0] = d->MatInv(fout, fin, &true_res, PRESERVE_YES);
    rpar[10] = now_s() - t0;
    delete d;
    rpar[0] = true_res;
    out_payload.assign((double *)fout, (double *)fout + 2 * fsz);
    sfree(fin);
    sfree(fout);
  } else if (op == OP_DMINUS) {
    // Mobius only: one full vector (4-D-even half first) in, Dminus of it out.
    if (action < 2) die("Dminus is a Mobius / zMobius operator");
    Vector *fin = (Vector *)smalloc(2 * fsz * sizeof(double));
    Vector *fout = (Vector *)smalloc(2 * fsz * sizeof(double));
    read_all(fi, fin, 2 * fsz * sizeof(double));
    memset(fout, 0, 2 * fsz * sizeof(double));
    if (action == 2) {
      DiracOpMobius d(lat, fout, fin, &cg_arg, CNV_FRM_NO);
      d.Dminus(fout, fin);
    } else {  // DiracOpZMobius::Dminus, d_op_zmobius.C:1213-1272
      DiracOpZMobius d(lat, fout, fin, &cg_arg, CNV_FRM_NO);
      d.Dminus(fout, fin);
    }
    out_payload.assign((double *)fout, (double *)fout + 2 * fsz);
    sfree(fin);
    sfree(fout);
  } else if (op == OP_FMATINV) {
    // Lattice::FmatInv with the source preserved and the dminus flag of hdr[18]
    // (only Fmobius overrides the dminus form; the others ignore the flag,
    // lattice.h:1127-1132).  Full source and initial guess in.
    Vector *fin = (Vector *)smalloc(2 * fsz * sizeof(double));
    Vector *fout = (Vector *)smalloc(2 * fsz * sizeof(double));
    read_all(fi, fin, 2 * fsz * sizeof(double));
    read_all(fi, fout, 2 * fsz * sizeof(double));
    Float true_res = 0;
    double t0 = now_s();
    rhdr[0] = lat.FmatInv(fout, fin, &cg_arg, &true_res, CNV_FRM_NO, PRESERVE_YES, (int)hdr[18]);
    rpar[10] = now_s() - t0;
    rpar[0] = true_res;
    out_payload.assign((double *)fout, (double *)fout + 2 * fsz);
    sfree(fin);
    sfree(fout);
  } else if (op == OP_MINRESEXT) {
    // phi, then degree previous solutions; returns psi, the orthonormalised
    // solutions and their MatPcDagMatPc images.
    const int degree = (int)hdr[17];
    if (degree < 0 || degree > 16) die("degree out of range");
    read_all(fi, in, fsz * sizeof(double));
    std::vector<Vector *> v(degree > 0 ? degree : 1), vm(degree > 0 ? degree : 1);
    for (int i = 0; i < degree; i++) {
      v[i] = (Vector *)smalloc(fsz * sizeof(double));
      vm[i] = (Vector *)smalloc(fsz * sizeof(double));
      read_all(fi, v[i], fsz * sizeof(double));
      memset(vm[i], 0, fsz * sizeof(double));
    }
    DiracOp *d = 0;
    if (action == 0) d = new DiracOpWilson(lat, out, in, &cg_arg, CNV_FRM_NO);
    else if (action == 1) d = new DiracOpDwf(lat, out, in, &cg_arg, CNV_FRM_NO);
    else d = new DiracOpMobius(lat, out, in, &cg_arg, CNV_FRM_NO);
    d->MinResExt(out, in, v.data(), vm.data(), degree);
    delete d;
    out_payload.assign((double *)out, (double *)out + fsz);
    for (int i = 0; i < degree; i++) out_payload.insert(out_payload.end(), (double *)v[i], (double *)v[i] + fsz);
    for (int i = 0; i < degree; i++) out_payload.insert(out_payload.end(), (double *)vm[i], (double *)vm[i] + fsz);
    for (int i = 0; i < degree; i++) { sfree(v[i]); sfree(vm[i]); }
  } else if (op == OP_FCONVERT) {
    const size_t full = 2 * fsz;  // both checkerboards
    Vector *f = (Vector *)smalloc(full * sizeof(double));
    read_all(fi, f, full * sizeof(double));
    const StrOrdType order = hdr[15] ? DWF_4D_EOPREC_EE : WILSON;
    if (hdr[16] == 0) lat.Fconvert(f, order, CANONICAL);
    else lat.Fconvert(f, CANONICAL, order);
    out_payload.assign((double *)f, (double *)f + full);
    sfree(f);
  } else {
    die("unknown op");
  }
  fclose(fi);
#ifdef USE_B200
  cpsb_kernel_launches(&launches1);
  rpar[44] = (double)(launches1 - launches0);
#endif
  FILE *fo = fopen(argv[2], "wb");
  if (!fo) die("cannot open response");
  write_all(fo, rhdr, sizeof rhdr);
  write_all(fo, rpar, sizeof rpar);
  write_all(fo, out_payload.data(), out_payload.size() * sizeof(double));
  fclose(fo);
  End();
  return 0;
}

/* cps_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle for parity tests.
 *
 * A plain-C restatement of the CPS (RBC-UKQCD/CPS_public, cps_pp v5.3.1) noarch
 * fermion-matrix path: Wilson / Shamir domain-wall / Mobius (zMobius sym2 and
 * orig preconditioners) Dslash, MatPc, MatPcDag, MatPcDagMatPc, and the CG and
 * multishift-CG solvers that drive them.  Each function cites the reference
 * file:line it restates (paths relative to cps_pp/src/util/).  Floating-point
 * operations are issued in the reference's order so that, compiled without FMA
 * contraction, results agree with the reference bit for bit; the parity tests
 * pin this file against golden vectors produced by the compiled reference.
 *
 * Nothing in the product links this file.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it (as oracle/liboracle.so).
 *
 * Layouts: gauge in WILSON order (even 4-D sites first, 72 reals per site, link
 * mu at 18*mu, element (row,col) at r+2*(row+3*col)); one checkerboard spinor
 * field = sites x 24 reals, r+2*(colour+3*spin); a 5-D field is Ls consecutive
 * 4-D checkerboard slices.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define UEL(u, r, row, col, mu) (u)[(r) + 2 * ((row) + 3 * ((col) + 3 * (mu)))]
#define FRM(f, r, c, s) (f)[(r) + 2 * ((c) + 3 * (s))]

/* ------------------------------------------------------------------ */
/* Storage conversion: lattice/convert/convert_func.C:371-405          */
/* ------------------------------------------------------------------ */
void orc_canon_to_wilson(double *uw, const double *uc, const int *dims) {
  const int lx = dims[0], ly = dims[1], lz = dims[2], lt = dims[3];
  const long vol = (long)lx * ly * lz * lt;
  for (int t = 0; t < lt; t++)
    for (int z = 0; z < lz; z++)
      for (int y = 0; y < ly; y++)
        for (int x = 0; x < lx; x++) {
          long cs = x + lx * (y + (long)ly * (z + (long)lz * t));
          long ws = (x - x % 2 + lx * (y + (long)ly * (z + (long)lz * t)) +
                     vol * ((x + y + z + t) % 2)) / 2;
          for (int mu = 0; mu < 4; mu++)
            for (int row = 0; row < 3; row++)
              for (int col = 0; col < 3; col++)
                for (int r = 0; r < 2; r++)
                  uw[72 * ws + r + 2 * (row + 3 * (col + 3 * mu))] =
                      uc[72 * cs + r + 2 * (col + 3 * (row + 3 * mu))];
        }
}

/* Negates the t-direction links on the last time slice (antiperiodic time
 * boundary), as Lattice::BondCond does (lattice/lattice_base/lattice_base.C:5313-5370).
 * Operates on a CANONICAL-order field. */
void orc_bondcond_t(double *uc, const int *dims) {
  const int lx = dims[0], ly = dims[1], lz = dims[2], lt = dims[3];
  for (int z = 0; z < lz; z++)
    for (int y = 0; y < ly; y++)
      for (int x = 0; x < lx; x++) {
        long cs = x + lx * (y + (long)ly * (z + (long)lz * (lt - 1)));
        for (int i = 0; i < 18; i++) uc[72 * cs + 18 * 3 + i] = -uc[72 * cs + 18 * 3 + i];
      }
}

/* ------------------------------------------------------------------ */
/* Wilson hop: d_op_wilson/noarch/wilson_dslash.C:64-167 (helpers),    */
/* :173-516 (site loop)                                                 */
/* ------------------------------------------------------------------ */

/* (1 -/+ sdag*gamma_mu) psi; mp = 0 gives the minus sign (forward hop). */
static void proj(double *o, const double *p, int sdag, int mu, int mp) {
  const double sg = (mp == 1 ? 1.0 : -1.0) * sdag;
  for (int c = 0; c < 3; c++) {
    if (mu == 0) {
      FRM(o, 0, c, 0) = FRM(p, 0, c, 0) + sg * (-FRM(p, 1, c, 3));
      FRM(o, 1, c, 0) = FRM(p, 1, c, 0) + sg * (FRM(p, 0, c, 3));
      FRM(o, 0, c, 1) = FRM(p, 0, c, 1) + sg * (-FRM(p, 1, c, 2));
      FRM(o, 1, c, 1) = FRM(p, 1, c, 1) + sg * (FRM(p, 0, c, 2));
      FRM(o, 0, c, 2) = FRM(p, 0, c, 2) + sg * (FRM(p, 1, c, 1));
      FRM(o, 1, c, 2) = FRM(p, 1, c, 2) + sg * (-FRM(p, 0, c, 1));
      FRM(o, 0, c, 3) = FRM(p, 0, c, 3) + sg * (FRM(p, 1, c, 0));
      FRM(o, 1, c, 3) = FRM(p, 1, c, 3) + sg * (-FRM(p, 0, c, 0));
    } else if (mu == 1) {
      FRM(o, 0, c, 0) = FRM(p, 0, c, 0) + sg * (-FRM(p, 0, c, 3));
      FRM(o, 1, c, 0) = FRM(p, 1, c, 0) + sg * (-FRM(p, 1, c, 3));
      FRM(o, 0, c, 1) = FRM(p, 0, c, 1) + sg * (FRM(p, 0, c, 2));
      FRM(o, 1, c, 1) = FRM(p, 1, c, 1) + sg * (FRM(p, 1, c, 2));
      FRM(o, 0, c, 2) = FRM(p, 0, c, 2) + sg * (FRM(p, 0, c, 1));
      FRM(o, 1, c, 2) = FRM(p, 1, c, 2) + sg * (FRM(p, 1, c, 1));
      FRM(o, 0, c, 3) = FRM(p, 0, c, 3) + sg * (-FRM(p, 0, c, 0));
      FRM(o, 1, c, 3) = FRM(p, 1, c, 3) + sg * (-FRM(p, 1, c, 0));
    } else if (mu == 2) {
      FRM(o, 0, c, 0) = FRM(p, 0, c, 0) + sg * (-FRM(p, 1, c, 2));
      FRM(o, 1, c, 0) = FRM(p, 1, c, 0) + sg * (FRM(p, 0, c, 2));
      FRM(o, 0, c, 1) = FRM(p, 0, c, 1) + sg * (FRM(p, 1, c, 3));
      FRM(o, 1, c, 1) = FRM(p, 1, c, 1) + sg * (-FRM(p, 0, c, 3));
      FRM(o, 0, c, 2) = FRM(p, 0, c, 2) + sg * (FRM(p, 1, c, 0));
      FRM(o, 1, c, 2) = FRM(p, 1, c, 2) + sg * (-FRM(p, 0, c, 0));
      FRM(o, 0, c, 3) = FRM(p, 0, c, 3) + sg * (-FRM(p, 1, c, 1));
      FRM(o, 1, c, 3) = FRM(p, 1, c, 3) + sg * (FRM(p, 0, c, 1));
    } else {
      FRM(o, 0, c, 0) = FRM(p, 0, c, 0) + sg * (FRM(p, 0, c, 2));
      FRM(o, 1, c, 0) = FRM(p, 1, c, 0) + sg * (FRM(p, 1, c, 2));
      FRM(o, 0, c, 1) = FRM(p, 0, c, 1) + sg * (FRM(p, 0, c, 3));
      FRM(o, 1, c, 1) = FRM(p, 1, c, 1) + sg * (FRM(p, 1, c, 3));
      FRM(o, 0, c, 2) = FRM(p, 0, c, 2) + sg * (FRM(p, 0, c, 0));
      FRM(o, 1, c, 2) = FRM(p, 1, c, 2) + sg * (FRM(p, 1, c, 0));
      FRM(o, 0, c, 3) = FRM(p, 0, c, 3) + sg * (FRM(p, 0, c, 1));
      FRM(o, 1, c, 3) = FRM(p, 1, c, 3) + sg * (FRM(p, 1, c, 1));
    }
  }
}

/* U psi (dagger = 0) or U^dagger psi (dagger = 1), per spin component. */
static void umul(double *o, const double *u, const double *p, int mu, int dagger) {
  for (int s = 0; s < 4; s++)
    for (int c = 0; c < 3; c++) {
      if (!dagger) {
        FRM(o, 0, c, s) = UEL(u, 0, c, 0, mu) * FRM(p, 0, 0, s) + UEL(u, 0, c, 1, mu) * FRM(p, 0, 1, s) +
                          UEL(u, 0, c, 2, mu) * FRM(p, 0, 2, s) - UEL(u, 1, c, 0, mu) * FRM(p, 1, 0, s) -
                          UEL(u, 1, c, 1, mu) * FRM(p, 1, 1, s) - UEL(u, 1, c, 2, mu) * FRM(p, 1, 2, s);
        FRM(o, 1, c, s) = UEL(u, 0, c, 0, mu) * FRM(p, 1, 0, s) + UEL(u, 0, c, 1, mu) * FRM(p, 1, 1, s) +
                          UEL(u, 0, c, 2, mu) * FRM(p, 1, 2, s) + UEL(u, 1, c, 0, mu) * FRM(p, 0, 0, s) +
                          UEL(u, 1, c, 1, mu) * FRM(p, 0, 1, s) + UEL(u, 1, c, 2, mu) * FRM(p, 0, 2, s);
      } else {
        FRM(o, 0, c, s) = UEL(u, 0, 0, c, mu) * FRM(p, 0, 0, s) + UEL(u, 0, 1, c, mu) * FRM(p, 0, 1, s) +
                          UEL(u, 0, 2, c, mu) * FRM(p, 0, 2, s) + UEL(u, 1, 0, c, mu) * FRM(p, 1, 0, s) +
                          UEL(u, 1, 1, c, mu) * FRM(p, 1, 1, s) + UEL(u, 1, 2, c, mu) * FRM(p, 1, 2, s);
        FRM(o, 1, c, s) = UEL(u, 0, 0, c, mu) * FRM(p, 1, 0, s) + UEL(u, 0, 1, c, mu) * FRM(p, 1, 1, s) +
                          UEL(u, 0, 2, c, mu) * FRM(p, 1, 2, s) - UEL(u, 1, 0, c, mu) * FRM(p, 0, 0, s) -
                          UEL(u, 1, 1, c, mu) * FRM(p, 0, 1, s) - UEL(u, 1, 2, c, mu) * FRM(p, 0, 2, s);
      }
    }
}

/* chi (sites of parity 1-cb) = sum_mu (1-sdag g_mu) U_mu(x) psi(x+mu)
 *                              + (1+sdag g_mu) U_mu(x-mu)^dag psi(x-mu). */
void orc_wilson_dslash(double *chi, const double *u, const double *psi, int cb, int dag,
                       const int *dims) {
  const int lx = dims[0], ly = dims[1], lz = dims[2], lt = dims[3];
  const long vol = (long)lx * ly * lz * lt / 2;
  const int sdag = dag ? -1 : 1;
  const int cbn = 1 - cb;
  const int L[4] = {lx, ly, lz, lt};
  double tmp[24], fw[4][24], bw[4][24];
  for (int x = 0; x < lx; x++)
    for (int y = 0; y < ly; y++)
      for (int z = 0; z < lz; z++)
        for (int t = 0; t < lt; t++) {
          if ((x + y + z + t) % 2 != cbn) continue;
          long xyzt = x / 2 + (lx / 2) * (y + (long)ly * (z + (long)lz * t));
          int pos[4] = {x, y, z, t};
          for (int mu = 0; mu < 4; mu++) {
            int pp[4] = {x, y, z, t};
            pp[mu] = (pp[mu] + 1) % L[mu];
            long pi = pp[0] / 2 + (lx / 2) * (pp[1] + (long)ly * (pp[2] + (long)lz * pp[3]));
            proj(tmp, psi + 24 * pi, sdag, mu, 0);
            umul(fw[mu], u + 72 * (xyzt + vol * cbn), tmp, mu, 0);
          }
          for (int mu = 0; mu < 4; mu++) {
            int pm[4] = {x, y, z, t};
            pm[mu] = (pm[mu] - 1 + L[mu]) % L[mu];
            long mi = pm[0] / 2 + (lx / 2) * (pm[1] + (long)ly * (pm[2] + (long)lz * pm[3]));
            proj(tmp, psi + 24 * mi, sdag, mu, 1);
            umul(bw[mu], u + 72 * (mi + vol * cb), tmp, mu, 1);
          }
          (void)pos;
          double *o = chi + 24 * xyzt;
          for (int i = 0; i < 24; i++)
            o[i] = fw[0][i] + fw[1][i] + fw[2][i] + fw[3][i] + bw[0][i] + bw[1][i] + bw[2][i] + bw[3][i];
        }
}

static double *scratch(size_t n) {
  double *p = (double *)malloc(n * sizeof(double));
  return p;
}

/* wilson_m.C:49-85 (dag=0), wilson_mdag.C:50 (dag=1): out = in - k^2 D D in. */
void orc_wilson_m(double *out, const double *u, const double *in, double kappa, int dag,
                  const int *dims) {
  const long vol = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  double *t1 = scratch(24 * vol);
  orc_wilson_dslash(t1, u, in, 1, dag, dims);
  orc_wilson_dslash(out, u, t1, 0, dag, dims);
  for (long i = 0; i < 24 * vol; i++) out[i] = in[i] - kappa * kappa * out[i];
  free(t1);
}

/* wilson_mdagm.C:83-160: out = M^dag M in, *dot = |M in|^2 (sequential sum). */
void orc_wilson_mdagm(double *out, const double *u, const double *in, double kappa, double *dot,
                      const int *dims) {
  const long vol = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  double *t1 = scratch(24 * vol), *t2 = scratch(24 * vol);
  orc_wilson_dslash(t1, u, in, 1, 0, dims);
  orc_wilson_dslash(t2, u, t1, 0, 0, dims);
  double sum = 0.0;
  for (long i = 0; i < 24 * vol; i++) {
    t2[i] = in[i] - kappa * kappa * t2[i];
    sum = sum + t2[i] * t2[i];
  }
  if (dot) *dot = sum;
  orc_wilson_dslash(t1, u, t2, 1, 1, dims);
  orc_wilson_dslash(out, u, t1, 0, 1, dims);
  for (long i = 0; i < 24 * vol; i++) out[i] = t2[i] - kappa * kappa * out[i];
  free(t1);
  free(t2);
}

/* ------------------------------------------------------------------ */
/* Shamir domain wall                                                  */
/* ------------------------------------------------------------------ */

/* dwf_dslash_4.C:68-154 -- the 4-D hop on every s slice; slice s of a
 * checkerboard-cb 5-D field holds 4-D parity (s+cb)%2. */
void orc_dwf_dslash_4(double *out, const double *u, const double *in, int cb, int dag,
                      const int *dims, int ls) {
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  for (int s = 0; s < ls; s++)
    orc_wilson_dslash(out + s * n, u, in + s * n, (s + cb) % 2, dag, dims);
}

/* out = fact*in + out on 12 reals (fTimesV1PlusV2, util/vector). */
static void axpy12(double *out, double fact, const double *in) {
  for (int i = 0; i < 12; i++) out[i] = fact * in[i] + out[i];
}

/* dwf_dslash_5_plus.C:111-340 -- 5th-direction hop with 2/a5 factors and the
 * -m_f wall terms; dag swaps the chiral halves. */
void orc_dwf_dslash_5_plus(double *out, const double *in, double mass, int dag, const int *dims,
                           int ls, double a5_inv) {
  const long v = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  const long st = 24 * v;
  const double two = 2.0 * a5_inv, negm = -2.0 * mass * a5_inv;
  const int up = dag ? 12 : 0, dn = dag ? 0 : 12;
  for (int s = 1; s < ls; s++)
    for (long x = 0; x < v; x++) axpy12(out + s * st + 24 * x + up, two, in + (s - 1) * st + 24 * x + up);
  for (long x = 0; x < v; x++) axpy12(out + 24 * x + up, negm, in + (ls - 1) * st + 24 * x + up);
  for (int s = 0; s < ls - 1; s++)
    for (long x = 0; x < v; x++) axpy12(out + s * st + 24 * x + dn, two, in + (s + 1) * st + 24 * x + dn);
  for (long x = 0; x < v; x++) axpy12(out + (ls - 1) * st + 24 * x + dn, negm, in + 24 * x + dn);
}

/* dwf_dslash.C:32-51 */
void orc_dwf_dslash(double *out, const double *u, const double *in, double mass, int cb, int dag,
                    const int *dims, int ls, double a5_inv) {
  orc_dwf_dslash_4(out, u, in, cb, dag, dims, ls);
  orc_dwf_dslash_5_plus(out, in, mass, dag, dims, ls, a5_inv);
}

/* dwf_m.C:31-63 / dwf_mdag.C:32-63: out = in - k^2 D(cb=0) D(cb=1) in,
 * kappa = 1/(2(4 + a5_inv - M5)) (dwf_init.C:97-98). */
void orc_dwf_m(double *out, const double *u, const double *in, double mass, int dag,
               const int *dims, int ls, double m5, double a5_inv) {
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2 * ls;
  const double kappa = 1.0 / (2 * (4 + a5_inv - m5));
  const double mks = -kappa * kappa;
  double *t2 = scratch(n);
  orc_dwf_dslash(t2, u, in, mass, 1, dag, dims, ls, a5_inv);
  orc_dwf_dslash(out, u, t2, mass, 0, dag, dims, ls, a5_inv);
  for (long i = 0; i < n; i++) out[i] = mks * out[i] + in[i];
  free(t2);
}

/* dwf_mdagm.C:32-62 */
void orc_dwf_mdagm(double *out, const double *u, const double *in, double mass, double *dot,
                   const int *dims, int ls, double m5, double a5_inv) {
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2 * ls;
  double *t1 = scratch(n);
  orc_dwf_m(t1, u, in, mass, 0, dims, ls, m5, a5_inv);
  if (dot) {
    double sum = 0.0;
    for (long i = 0; i < n; i++) sum += t1[i] * t1[i];
    *dot = sum;
  }
  orc_dwf_m(out, u, t1, mass, 1, dims, ls, m5, a5_inv);
  free(t1);
}

/* ------------------------------------------------------------------ */
/* Mobius (zMobius code path with per-s complex coefficients)          */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cplx;
static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline cplx cconj(cplx a) { cplx r = {a.re, -a.im}; return r; }
static inline cplx cneg(cplx a) { cplx r = {-a.re, -a.im}; return r; }
static inline cplx cscal(double f, cplx a) { cplx r = {f * a.re, f * a.im}; return r; }
/* Smith's complex division a/b (the algorithm libgcc's __divdc3 uses for finite values). */
static inline cplx cdiv(cplx a, cplx b) {
  cplx r;
  if (fabs(b.re) < fabs(b.im)) {
    double ratio = b.re / b.im, den = b.re * ratio + b.im;
    r.re = (a.re * ratio + a.im) / den;
    r.im = (a.im * ratio - a.re) / den;
  } else {
    double ratio = b.im / b.re, den = b.im * ratio + b.re;
    r.re = (a.im * ratio + a.re) / den;
    r.im = (a.im - a.re * ratio) / den;
  }
  return r;
}

/* Parameters of the Mobius operator (DiracOpMobius ctor, d_op_mobius/d_op_mobius.C:100-123). */
typedef struct {
  int ls;
  double mass, m5, a5_inv;
  double b[64][2], c[64][2];  /* per-s b_s, c_s as (re, im) */
  int pc_type;                 /* 0 ZMOB_PC_ORIG, 1 ZMOB_PC_SYM1, 2 ZMOB_PC_SYM2 */
} orc_mobius_params;

/* kappa_b(s) = 1/(2(b_s(4-M5)+a5_inv)), kappa_c(s) = 1/(2(c_s(4-M5)-a5_inv)),
 * kappa_ratio = kappa_b/kappa_c.  The ctor computes these from the real
 * Mobius b, c (d_op_mobius.C:106-123); complex b_s/c_s use the same formulas. */
static void mobius_kappas(const orc_mobius_params *p, cplx *kb, cplx *kc, cplx *kr) {
  for (int s = 0; s < p->ls; s++) {
    cplx b = {p->b[s][0], p->b[s][1]}, c = {p->c[s][0], p->c[s][1]};
    cplx one = {1.0, 0.0};
    cplx db = {2 * (b.re * (4 - p->m5) + p->a5_inv), 2 * (b.im * (4 - p->m5))};
    cplx dc = {2 * (c.re * (4 - p->m5) - p->a5_inv), 2 * (c.im * (4 - p->m5))};
    if (b.im == 0 && c.im == 0) {
      /* real Mobius: exactly the reference's real expressions */
      double kbr = 1.0 / (2 * (b.re * (4 - p->m5) + p->a5_inv));
      double kcr = 1.0 / (2 * (c.re * (4 - p->m5) - p->a5_inv));
      kb[s].re = kbr; kb[s].im = 0;
      kc[s].re = kcr; kc[s].im = 0;
      cplx a = {kbr, 0}, d = {kcr, 0};
      kr[s] = cdiv(a, d);
    } else {
      kb[s] = cdiv(one, db);
      kc[s] = cdiv(one, dc);
      kr[s] = cdiv(kb[s], kc[s]);
    }
  }
}

/* zmobius_dslash_5_plus.C:125-376 -- out[s] += fact[s] P+ in[s-1] + fact[s] P- in[s+1]
 * with -m_f*fact at the walls; dag uses the conjugated, index-shifted factors. */
static void zaxpy6(double *out, cplx f, const double *in) {
  for (int i = 0; i < 6; i++) {
    cplx a = {in[2 * i], in[2 * i + 1]};
    cplx r = cmul(f, a);
    out[2 * i] = r.re + out[2 * i];
    out[2 * i + 1] = r.im + out[2 * i + 1];
  }
}
void orc_zmobius_dslash_5_plus(double *out, const double *in, double mass, int dag,
                               const int *dims, int ls, const cplx *fact_in) {
  const long v = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  const long st = 24 * v;
  cplx fact[64];
  for (int i = 0; i < ls; i++) fact[i] = dag ? cconj(fact_in[i]) : fact_in[i];
  const cplx nm0 = cscal(-mass, fact[0]), nml = cscal(-mass, fact[ls - 1]);
  const int up = dag ? 12 : 0, dn = dag ? 0 : 12;
  for (int s = 1; s < ls; s++) {
    cplx f = dag ? fact[s - 1] : fact[s];
    for (long x = 0; x < v; x++) zaxpy6(out + s * st + 24 * x + up, f, in + (s - 1) * st + 24 * x + up);
  }
  for (long x = 0; x < v; x++) zaxpy6(out + 24 * x + up, dag ? nml : nm0, in + (ls - 1) * st + 24 * x + up);
  for (int s = 0; s < ls - 1; s++) {
    cplx f = dag ? fact[s + 1] : fact[s];
    for (long x = 0; x < v; x++) zaxpy6(out + s * st + 24 * x + dn, f, in + (s + 1) * st + 24 * x + dn);
  }
  for (long x = 0; x < v; x++)
    zaxpy6(out + (ls - 1) * st + 24 * x + dn, dag ? nm0 : nml, in + 24 * x + dn);
}

/* a[i] = c * b[i] on complex pairs (vecEqualsVecTimesEquComplex, include/util/zmobius.h:235). */
static void zscale_copy(double *a, const double *b, cplx c, long nreal) {
  for (long i = 0; i < nreal / 2; i++) {
    cplx x = {b[2 * i], b[2 * i + 1]};
    cplx r = cmul(c, x);
    a[2 * i] = r.re;
    a[2 * i + 1] = r.im;
  }
}
/* a[i] *= c (vecTimesEquComplex, include/util/zmobius.h:265). */
static void zscale(double *a, cplx c, long nreal) {
  for (long i = 0; i < nreal / 2; i++) {
    cplx x = {a[2 * i], a[2 * i + 1]};
    cplx r = cmul(x, c);
    a[2 * i] = r.re;
    a[2 * i + 1] = r.im;
  }
}

/* zmobius_dslash_4.C:34-221: dag0: tmp = b_s in_s + c-hop(in), out_s = D_W(cb) tmp_s;
 * dag1: tmp_s = D_W^dag(cb) in_s, out_s = conj(b_s) tmp_s + c-hop^dag(tmp). */
void orc_mobius_dslash_4(double *out, const double *u, const double *in, int cb, int dag,
                         const int *dims, const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx b[64], c[64];
  for (int s = 0; s < ls; s++) {
    b[s].re = p->b[s][0]; b[s].im = p->b[s][1];
    c[s].re = p->c[s][0]; c[s].im = p->c[s][1];
  }
  double *tmp = scratch(n * ls);
  if (!dag) {
    for (int s = 0; s < ls; s++) zscale_copy(tmp + s * n, in + s * n, b[s], n);
    orc_zmobius_dslash_5_plus(tmp, in, p->mass, 0, dims, ls, c);
    for (int s = 0; s < ls; s++) orc_wilson_dslash(out + s * n, u, tmp + s * n, cb, 0, dims);
  } else {
    for (int s = 0; s < ls; s++) orc_wilson_dslash(tmp + s * n, u, in + s * n, cb, 1, dims);
    for (int s = 0; s < ls; s++) zscale_copy(out + s * n, tmp + s * n, cconj(b[s]), n);
    orc_zmobius_dslash_5_plus(out, tmp, p->mass, 1, dims, ls, c);
  }
  free(tmp);
}

#define ZAXPY12(f, src, dst) zaxpy6((dst), (f), (src))

/* zmobius_m5inv.C:247-400 (dag 0) and :534-686 (dag 1): in-place exact M5^-1
 * by a forward and a backward sweep along s with the wall correction. */
static void m5inv_k(double *io, int dag, const int *dims, const orc_mobius_params *p, const cplx *K);
void orc_mobius_m5inv(double *io, int dag, const int *dims, const orc_mobius_params *p) {
  cplx kb[64], kc[64], K[64];
  mobius_kappas(p, kb, kc, K);
  m5inv_k(io, dag, dims, p, K);
}

/* zmobius_m5inv with the hopping ratios K[s] given (kappa_ratio, or c_s/b_s for
 * the MIT preconditioners' B^-1). */
static void m5inv_k(double *io, int dag, const int *dims, const orc_mobius_params *p, const cplx *K) {
  const int ls = p->ls;
  const long v = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  const double mass = p->mass;
#define F(x, s) (io + 24 * ((x) + v * (long)(s)))
  if (!dag) {
    cplx prod = {1.0, 0.0};
    for (int i = 0; i < ls; i++) prod = cmul(prod, cneg(K[i]));
    prod = cscal(mass, prod);
    cplx one = {1.0, 0.0}, den = {1.0 + prod.re, prod.im};
    cplx inv_d_last = cdiv(one, den);
    for (long x = 0; x < v; x++) zscale(F(x, ls - 1) + 12, inv_d_last, 12);
    cplx factL = cmul(cscal(mass, K[ls - 1]), inv_d_last);
    for (int s = 0; s <= ls - 2; ++s) {
      for (long x = 0; x < v; x++) {
        ZAXPY12(cneg(K[s + 1]), F(x, s), F(x, s + 1));
        ZAXPY12(factL, F(x, s) + 12, F(x, ls - 1) + 12);
      }
      factL = cmul(factL, cneg(K[s]));
    }
    cplx pr = {1.0, 0.0};
    for (int i = 0; i < ls - 1; i++) pr = cmul(pr, cneg(K[i]));
    cplx factR = cneg(cmul(cscal(mass, pr), inv_d_last));
    for (int s = ls - 2; s >= 0; --s) {
      for (long x = 0; x < v; x++) {
        ZAXPY12(factR, F(x, ls - 1), F(x, s));
        ZAXPY12(cneg(K[s]), F(x, s + 1) + 12, F(x, s) + 12);
      }
      factR = cdiv(factR, cneg(K[s]));
    }
    for (long x = 0; x < v; x++) zscale(F(x, ls - 1), inv_d_last, 12);
  } else {
    cplx prod = {1.0, 0.0};
    for (int i = 0; i < ls; i++) prod = cmul(prod, K[i]);
    prod = cscal(mass, prod);
    cplx one = {1.0, 0.0}, den = {1.0 + prod.re, prod.im};
    cplx inv_d_last = cconj(cdiv(one, den));
    for (long x = 0; x < v; x++) zscale(F(x, ls - 1), inv_d_last, 12);
    cplx factR = cmul(cscal(mass, cconj(K[0])), inv_d_last);
    for (int s = 0; s <= ls - 2; ++s) {
      for (long x = 0; x < v; x++) {
        ZAXPY12(factR, F(x, s), F(x, ls - 1));
        ZAXPY12(cneg(cconj(K[s])), F(x, s) + 12, F(x, s + 1) + 12);
      }
      factR = cmul(factR, cneg(cconj(K[s + 1])));
    }
    cplx pr = {1.0, 0.0};
    for (int i = 0; i < ls - 2; i++) pr = cmul(pr, cneg(K[i]));
    pr = cmul(pr, cneg(K[ls - 1]));
    cplx factL = cneg(cmul(cscal(mass, cconj(pr)), inv_d_last));
    for (int s = ls - 2; s >= 0; --s) {
      for (long x = 0; x < v; x++) {
        ZAXPY12(cneg(cconj(K[s + 1])), F(x, s + 1), F(x, s));
        ZAXPY12(factL, F(x, ls - 1) + 12, F(x, s) + 12);
      }
      if (s > 0) factL = cdiv(factL, cneg(cconj(K[s - 1])));
    }
    for (long x = 0; x < v; x++) zscale(F(x, ls - 1) + 12, inv_d_last, 12);
  }
#undef F
}

/* zmobius_m-sym2.h:5-127: out = in - kb D4(0) M5^-1 kb D4(1) M5^-1 in. */
static void mobius_m_sym2(double *out, const double *u, const double *in, const int *dims,
                          const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(t2, in, sizeof(double) * n * ls);
  orc_mobius_m5inv(t2, 0, dims, p);
  orc_mobius_dslash_4(out, u, t2, 1, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, kb[s], n);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cneg(kb[s]), n);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  free(t2);
}

/* zmobius_mdag-sym2.h:4-109 */
static void mobius_mdag_sym2(double *out, const double *u, const double *in, const int *dims,
                             const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  for (int s = 0; s < ls; s++) zscale(out + s * n, cneg(cconj(kb[s])), n);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cconj(kb[s]), n);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  orc_mobius_m5inv(out, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  free(t2);
}

/* zmobius_m-orig.h:3-126: out = in - kb D4(0) M5^-1 kb D4(1) in + kr H5 in
 * (M5 - kb^2 D4 M5^-1 D4 with M5 = 1 + kr H5). */
static void mobius_m_orig(double *out, const double *u, const double *in, const int *dims,
                          const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  orc_mobius_dslash_4(out, u, in, 1, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, kb[s], n);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cneg(kb[s]), n);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  orc_zmobius_dslash_5_plus(out, in, p->mass, 0, dims, ls, kr);
  free(t2);
}

/* zmobius_mdag-orig.h */
static void mobius_mdag_orig(double *out, const double *u, const double *in, const int *dims,
                             const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  for (int s = 0; s < ls; s++) zscale(out + s * n, cneg(cconj(kb[s])), n);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cconj(kb[s]), n);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  orc_zmobius_dslash_5_plus(out, in, p->mass, 1, dims, ls, kr);
  free(t2);
}

/* zmobius_m-sym1.h: out = in - M5^-1 kb D4(0) M5^-1 kb D4(1) in. */
static void mobius_m_sym1(double *out, const double *u, const double *in, const int *dims,
                          const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  orc_mobius_dslash_4(out, u, in, 1, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, kb[s], n);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cneg(kb[s]), n);
  orc_mobius_m5inv(t2, 0, dims, p);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  free(t2);
}

/* zmobius_mdag-sym1.h */
static void mobius_mdag_sym1(double *out, const double *u, const double *in, const int *dims,
                             const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  orc_mobius_m5inv(out, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, cneg(cconj(kb[s])), n);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cconj(kb[s]), n);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  free(t2);
}

/* zmobius_B_MIT / zmobius_Binv_MIT (d_op_zmobius.C:132-238), fact_s = c_s / b_s:
 *   B   dag 0: v = b_s (v + fact-H5 v);        dag 1: v = conj(b_s) v + fact-H5^dag(conj(b) v)
 *   B^-1 dag 0: v = M5^-1[K = fact](v / b_s);  dag 1: v = M5^-dag[K = fact](v) / conj(b_s) */
static void b_mit(double *v, int dag, const int *dims, const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx b[64], c[64], fact[64];
  for (int s = 0; s < ls; s++) {
    b[s].re = p->b[s][0]; b[s].im = p->b[s][1];
    c[s].re = p->c[s][0]; c[s].im = p->c[s][1];
    fact[s] = cdiv(c[s], b[s]);
  }
  double *t = scratch(n * ls);
  if (!dag) {
    memcpy(t, v, sizeof(double) * n * ls);
    orc_zmobius_dslash_5_plus(v, t, p->mass, 0, dims, ls, fact);
    for (int s = 0; s < ls; s++) zscale(v + s * n, b[s], n);
  } else {
    memcpy(t, v, sizeof(double) * n * ls);
    for (int s = 0; s < ls; s++) zscale(t + s * n, cconj(b[s]), n);
    memcpy(v, t, sizeof(double) * n * ls);
    orc_zmobius_dslash_5_plus(v, t, p->mass, 1, dims, ls, fact);
  }
  free(t);
}
static void binv_mit(double *v, int dag, const int *dims, const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx b[64], fact[64];
  const cplx one = {1.0, 0.0};
  for (int s = 0; s < ls; s++) {
    cplx c = {p->c[s][0], p->c[s][1]};
    b[s].re = p->b[s][0]; b[s].im = p->b[s][1];
    fact[s] = cdiv(c, b[s]);
  }
  if (!dag) {
    for (int s = 0; s < ls; s++) zscale(v + s * n, cdiv(one, b[s]), n);
    m5inv_k(v, 0, dims, p, fact);
  } else {
    m5inv_k(v, 1, dims, p, fact);
    for (int s = 0; s < ls; s++) zscale(v + s * n, cdiv(one, cconj(b[s])), n);
  }
}

/* zmobius_m-sym1-MIT.h / zmobius_mdag-sym1-MIT.h */
static void mobius_m_sym1_mit(double *out, const double *u, const double *in, const int *dims,
                              const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(t2, in, sizeof(double) * n * ls);
  binv_mit(t2, 0, dims, p);
  orc_mobius_dslash_4(out, u, t2, 1, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, kb[s], n);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cneg(kb[s]), n);
  orc_mobius_m5inv(t2, 0, dims, p);
  b_mit(t2, 0, dims, p);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  free(t2);
}
static void mobius_mdag_sym1_mit(double *out, const double *u, const double *in, const int *dims,
                                 const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  b_mit(out, 1, dims, p);
  orc_mobius_m5inv(out, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, cneg(cconj(kb[s])), n);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cconj(kb[s]), n);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  binv_mit(out, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  free(t2);
}

/* zmobius_m-sym2-MIT.h / zmobius_mdag-sym2-MIT.h */
static void mobius_m_sym2_mit(double *out, const double *u, const double *in, const int *dims,
                              const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(t2, in, sizeof(double) * n * ls);
  binv_mit(t2, 0, dims, p);
  orc_mobius_m5inv(t2, 0, dims, p);
  orc_mobius_dslash_4(out, u, t2, 1, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, kb[s], n);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cneg(kb[s]), n);
  b_mit(t2, 0, dims, p);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  free(t2);
}
static void mobius_mdag_sym2_mit(double *out, const double *u, const double *in, const int *dims,
                                 const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(p, kb, kc, kr);
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  b_mit(out, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(out + s * n, cneg(cconj(kb[s])), n);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  for (int s = 0; s < ls; s++) zscale(t2 + s * n, cconj(kb[s]), n);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  orc_mobius_m5inv(out, 1, dims, p);
  binv_mit(out, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  free(t2);
}

/* zmobius_m-sym3.h / zmobius_mdag-sym3.h.  The reference scales GJP's b, c by
 * kappa_b i around its D4 calls, but zmobius_dslash_4 reads the DiracOp's own
 * copies (zmobius_dslash_4.C:61-62), so the operator it applies is
 *   M = 1 + D4(0) M5^-1 D4(1) M5^-1,  M^dag = 1 + M5^-dag D4^dag(0) M5^-dag D4^dag(1). */
static void mobius_m_sym3(double *out, const double *u, const double *in, const int *dims,
                          const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  double *t2 = scratch(n * ls);
  memcpy(t2, in, sizeof(double) * n * ls);
  orc_mobius_m5inv(t2, 0, dims, p);
  orc_mobius_dslash_4(out, u, t2, 1, 0, dims, p);
  orc_mobius_m5inv(out, 0, dims, p);
  orc_mobius_dslash_4(t2, u, out, 0, 0, dims, p);
  memcpy(out, in, sizeof(double) * n * ls);
  for (long i = 0; i < n * ls; i++) out[i] += t2[i];
  free(t2);
}
static void mobius_mdag_sym3(double *out, const double *u, const double *in, const int *dims,
                             const orc_mobius_params *p) {
  const int ls = p->ls;
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2;
  double *t2 = scratch(n * ls);
  memcpy(out, in, sizeof(double) * n * ls);
  orc_mobius_dslash_4(t2, u, out, 1, 1, dims, p);
  orc_mobius_m5inv(t2, 1, dims, p);
  orc_mobius_dslash_4(out, u, t2, 0, 1, dims, p);
  orc_mobius_m5inv(out, 1, dims, p);
  for (long i = 0; i < n * ls; i++) out[i] += in[i];
  free(t2);
}

/* mobius_m.C:28-42 -> zmobius_m.C:40-74 (pc dispatch); mobius_mdag.C:35-55. */
int orc_mobius_m(double *out, const double *u, const double *in, int dag, const int *dims,
                 const orc_mobius_params *p) {
  switch (p->pc_type) {  /* ZMOB_PC_ORIG, SYM1, SYM2, SYM1_MIT, SYM2_MIT, SYM3 (util/dwf.h:42-48) */
    case 0: if (dag) mobius_mdag_orig(out, u, in, dims, p); else mobius_m_orig(out, u, in, dims, p); return 0;
    case 1: if (dag) mobius_mdag_sym1(out, u, in, dims, p); else mobius_m_sym1(out, u, in, dims, p); return 0;
    case 2: if (dag) mobius_mdag_sym2(out, u, in, dims, p); else mobius_m_sym2(out, u, in, dims, p); return 0;
    case 3: if (dag) mobius_mdag_sym1_mit(out, u, in, dims, p); else mobius_m_sym1_mit(out, u, in, dims, p); return 0;
    case 4: if (dag) mobius_mdag_sym2_mit(out, u, in, dims, p); else mobius_m_sym2_mit(out, u, in, dims, p); return 0;
    case 5: if (dag) mobius_mdag_sym3(out, u, in, dims, p); else mobius_m_sym3(out, u, in, dims, p); return 0;
    default: return -1;
  }
}

/* mobius_mdagm.C:33-60 */
int orc_mobius_mdagm(double *out, const double *u, const double *in, double *dot, const int *dims,
                     const orc_mobius_params *p) {
  const long n = 24L * dims[0] * dims[1] * dims[2] * dims[3] / 2 * p->ls;
  double *t1 = scratch(n);
  if (orc_mobius_m(t1, u, in, 0, dims, p)) { free(t1); return -1; }
  if (dot) {
    double sum = 0.0;
    for (long i = 0; i < n; i++) sum += t1[i] * t1[i];
    *dot = sum;
  }
  orc_mobius_m(out, u, t1, 1, dims, p);
  free(t1);
  return 0;
}

/* mobius_dslash.C:23-43 (DiracOpMobius::Dslash): D4 then the real 5th-direction
 * hop with factor 1/kappa_c (mobius_dslash_5_plus.C:119-...). */
void orc_mobius_dslash(double *out, const double *u, const double *in, int cb, int dag,
                       const int *dims, const orc_mobius_params *p) {
  orc_mobius_dslash_4(out, u, in, cb, dag, dims, p);
  const double kc = 1.0 / (2 * (p->c[0][0] * (4 - p->m5) - p->a5_inv));
  const double fact = 1.0 / kc;
  const long v = (long)dims[0] * dims[1] * dims[2] * dims[3] / 2;
  const long st = 24 * v;
  const int ls = p->ls;
  const double negm = -p->mass * fact;
  const int up = dag ? 12 : 0, dn = dag ? 0 : 12;
  for (int s = 1; s < ls; s++)
    for (long x = 0; x < v; x++) axpy12(out + s * st + 24 * x + up, fact, in + (s - 1) * st + 24 * x + up);
  for (long x = 0; x < v; x++) axpy12(out + 24 * x + up, negm, in + (ls - 1) * st + 24 * x + up);
  for (int s = 0; s < ls - 1; s++)
    for (long x = 0; x < v; x++) axpy12(out + s * st + 24 * x + dn, fact, in + (s + 1) * st + 24 * x + dn);
  for (long x = 0; x < v; x++) axpy12(out + (ls - 1) * st + 24 * x + dn, negm, in + 24 * x + dn);
}

/* ------------------------------------------------------------------ */
/* Operator dispatch for the solvers                                   */
/* ------------------------------------------------------------------ */
typedef struct {
  int action;            /* 0 Wilson, 1 DWF, 2 Mobius */
  int dims[4];
  int ls;
  double mass, m5, a5_inv;
  const double *u;       /* WILSON-order gauge */
  orc_mobius_params mob; /* Mobius only */
} orc_op;

long orc_op_size(const orc_op *op) {
  return 24L * op->dims[0] * op->dims[1] * op->dims[2] * op->dims[3] / 2 * (op->action ? op->ls : 1);
}

/* MatPcDagMatPc of the chosen action (d_op_wilson.C:150, d_op_dwf.C:174, d_op_mobius.C:198). */
int orc_mdagm(const orc_op *op, double *out, const double *in, double *dot) {
  if (op->action == 0) {
    double kappa = 1.0 / (2.0 * (op->mass + 4.0));
    orc_wilson_mdagm(out, op->u, in, kappa, dot, op->dims);
    return 0;
  }
  if (op->action == 1) {
    orc_dwf_mdagm(out, op->u, in, op->mass, dot, op->dims, op->ls, op->m5, op->a5_inv);
    return 0;
  }
  orc_mobius_params p = op->mob;
  p.mass = op->mass;
  return orc_mobius_mdagm(out, op->u, in, dot, op->dims, &p);
}

/* MatPc (dag=0) / MatPcDag (dag=1). */
int orc_matpc(const orc_op *op, double *out, const double *in, int dag) {
  if (op->action == 0) {
    orc_wilson_m(out, op->u, in, 1.0 / (2.0 * (op->mass + 4.0)), dag, op->dims);
    return 0;
  }
  if (op->action == 1) {
    orc_dwf_m(out, op->u, in, op->mass, dag, op->dims, op->ls, op->m5, op->a5_inv);
    return 0;
  }
  orc_mobius_params p = op->mob;
  p.mass = op->mass;
  return orc_mobius_m(out, op->u, in, dag, op->dims, &p);
}

/* Dslash front end of the chosen action. */
int orc_dslash(const orc_op *op, double *out, const double *in, int cb, int dag) {
  if (op->action == 0) { orc_wilson_dslash(out, op->u, in, cb, dag, op->dims); return 0; }
  if (op->action == 1) {
    orc_dwf_dslash(out, op->u, in, op->mass, cb, dag, op->dims, op->ls, op->a5_inv);
    return 0;
  }
  orc_mobius_params p = op->mob;
  p.mass = op->mass;
  orc_mobius_dslash(out, op->u, in, cb, dag, op->dims, &p);
  return 0;
}

static double dot_seq(const double *a, const double *b, long n) {
  double s = 0.0;
  for (long i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* DiracOp::InvCgShift, d_op_base/comsrc/inv_cg.C:84-447 (shift = NULL path):
 * CG on MatPcDagMatPc sol = src from the initial guess in sol; stops when
 * |r|^2 <= stop_rsd^2 |src|^2 or after max_num_iter-1 iterations; returns the
 * iteration count (itr+1) and the true residual |src - A sol|/|src|. */
int orc_invcg(const orc_op *op, double *sol, const double *src, double stop_rsd, int max_num_iter,
              double *true_res, double *res_hist) {
  const long n = orc_op_size(op);
  double *res = scratch(n), *dir = scratch(n), *mmp = scratch(n);
  double src_norm_sq = dot_seq(src, src, n);
  double stp_cnd = src_norm_sq * stop_rsd * stop_rsd;
  orc_mdagm(op, mmp, sol, NULL);
  memcpy(res, src, n * sizeof(double));
  for (long i = 0; i < n; i++) res[i] -= mmp[i];
  memcpy(dir, res, n * sizeof(double));
  double rcur = dot_seq(res, res, n), rprv, d, a, b;
  int itr = 0, max_itr = max_num_iter - 1;
  if (rcur <= stp_cnd) max_itr = 0;
  for (int i = 0; i < max_itr; i++) {
    itr = itr + 1;
    rprv = rcur;
    orc_mdagm(op, mmp, dir, &d);
    if (d == 0.0) { itr = -1; break; }
    a = rprv / d;
    for (long k = 0; k < n; k++) sol[k] = a * dir[k] + sol[k];
    for (long k = 0; k < n; k++) res[k] = -a * mmp[k] + res[k];
    rcur = dot_seq(res, res, n);
    if (res_hist) res_hist[i] = rcur;
    if (rcur <= stp_cnd) break;
    b = rcur / rprv;
    for (long k = 0; k < n; k++) dir[k] = b * dir[k] + res[k];
  }
  orc_mdagm(op, mmp, sol, NULL);
  memcpy(res, src, n * sizeof(double));
  for (long i = 0; i < n; i++) res[i] -= mmp[i];
  double rr = dot_seq(res, res, n);
  if (true_res) *true_res = sqrt(rr / src_norm_sq);
  free(res); free(dir); free(mmp);
  return itr < 0 ? -1 : itr + 1;
}

/* DiracOp::MInvCG, d_op_base/noarch/minvcg.C:47-353 (types MULTI = 0 and
 * SINGLE = 1).  psi[s] receive the solutions (MULTI) or psi[0] the alpha-weighted
 * sum (SINGLE, psi[0] must be zero on entry).  rsd[s] holds stop_rsd on entry
 * and the iterated absolute residual sqrt(c z_s^2) on return, as CPS returns it. */
int orc_minvcg(const orc_op *op, double **psi, const double *chi, double chi_norm,
               const double *mass, int nmass, double *rsd, int type, const double *alpha,
               int max_num_iter) {
  const long n = orc_op_size(op);
  double *r = scratch(n), *Ap = scratch(n);
  double **p = (double **)malloc(sizeof(double *) * nmass);
  for (int s = 0; s < nmass; s++) p[s] = scratch(n);
  int *convsP = (int *)calloc(nmass, sizeof(int)), *converged = (int *)calloc(nmass, sizeof(int));
  double *bs = scratch(nmass), *z0 = scratch(nmass), *z1 = scratch(nmass), *rsd_sq = scratch(nmass);
  double *z[2] = {z0, z1};
  double a = 0, as, b, bp, b_tmp, css = 0, ztmp, c, d, cp;
  int iz, k, convP;
  if (type == 0)
    for (int i = 0; i < nmass; i++) memset(psi[i], 0, n * sizeof(double));
  memcpy(r, chi, n * sizeof(double));
  cp = chi_norm;
  for (int s = 0; s < nmass; s++) memcpy(p[s], r, n * sizeof(double));
  for (int s = 0; s < nmass; s++) rsd_sq[s] = cp * (rsd[s] * rsd[s]);
  if (mass[0] > 0) {
    orc_mdagm(op, Ap, p[0], NULL);
    for (long i = 0; i < n; i++) Ap[i] = mass[0] * p[0][i] + Ap[i];
    d = dot_seq(p[0], Ap, n);
  } else {
    orc_mdagm(op, Ap, p[0], &d);
  }
  b = -cp / d;
  z[0][0] = 1.0;
  z[1][0] = 1.0;
  bs[0] = b;
  iz = 1;
  for (int s = 1; s < nmass; s++) {
    z[1 - iz][s] = 1.0;
    z[iz][s] = 1.0 / (1.0 - b * (mass[s] - mass[0]));
    bs[s] = b * z[iz][s];
  }
  for (long i = 0; i < n; i++) r[i] = b * Ap[i] + r[i];
  c = dot_seq(r, r, n);
  if (type == 1) {
    for (int s = 0; s < nmass; s++) {
      b_tmp = bs[s] * alpha[s];
      for (long i = 0; i < n; i++) psi[0][i] = -b_tmp * chi[i] + psi[0][i];
    }
  } else {
    for (int s = 0; s < nmass; s++)
      for (long i = 0; i < n; i++) psi[s][i] = -bs[s] * chi[i] + psi[s][i];
  }
  convP = (c < rsd_sq[0]) ? 1 : 0;
  a = c / cp;
  for (k = 1; k <= max_num_iter && !convP; k++) {
    a = c / cp;
    for (int s = 0; s < nmass; s++) {
      if (convsP[s]) continue;
      if (s == 0) {
        for (long i = 0; i < n; i++) p[s][i] = a * p[s][i] + r[i];
      } else {
        as = a * (z[iz][s] * bs[s]) / (z[1 - iz][s] * b);
        for (long i = 0; i < n; i++) p[s][i] *= as;
        for (long i = 0; i < n; i++) p[s][i] = z[iz][s] * r[i] + p[s][i];
      }
    }
    cp = c;
    if (mass[0] > 0) {
      orc_mdagm(op, Ap, p[0], NULL);
      for (long i = 0; i < n; i++) Ap[i] = mass[0] * p[0][i] + Ap[i];
      d = dot_seq(p[0], Ap, n);
    } else {
      orc_mdagm(op, Ap, p[0], &d);
    }
    bp = b;
    b = -cp / d;
    bs[0] = b;
    iz = 1 - iz;
    for (int s = 1; s < nmass; s++) {
      if (convsP[s]) continue;
      ztmp = z[1 - iz][s] * z[iz][s] * bp /
             (b * a * (z[iz][s] - z[1 - iz][s]) + z[iz][s] * bp * (1 - b * (mass[s] - mass[0])));
      bs[s] = b * ztmp / z[1 - iz][s];
      z[iz][s] = ztmp;
    }
    for (long i = 0; i < n; i++) r[i] = b * Ap[i] + r[i];
    c = dot_seq(r, r, n);
    if (type == 1) {
      for (int s = 0; s < nmass; s++) {
        if (convsP[s]) continue;
        for (long i = 0; i < n; i++) psi[0][i] = -bs[s] * alpha[s] * p[s][i] + psi[0][i];
      }
    } else {
      for (int s = 0; s < nmass; s++) {
        if (convsP[s]) continue;
        for (long i = 0; i < n; i++) psi[s][i] = -bs[s] * p[s][i] + psi[s][i];
      }
    }
    for (int s = 0; s < nmass; s++) {
      if (convsP[s]) continue;
      css = c * z[iz][s] * z[iz][s];
      convsP[s] = (css < rsd_sq[s]) ? 1 : 0;
      if (convsP[s]) { rsd[s] = css; converged[s] = k; }
    }
    convP = convsP[0];
    if (convP)
      for (int s = 0; s < nmass; s++)
        if (!convsP[s]) convP = 0;
  }
  for (int s = nmass - 1; s >= 0; s--) {
    if (convsP[s]) rsd[s] = sqrt(rsd[s]);
    else rsd[s] = sqrt(c * z[iz][s] * z[iz][s]);
  }
  for (int s = 0; s < nmass; s++) free(p[s]);
  free(p); free(r); free(Ap); free(convsP); free(converged); free(bs); free(z0); free(z1);
  free(rsd_sq);
  return k;
}

/* ------------------------------------------------------------------ */
/* Full-lattice solve: DiracOp*::MatInv with the source preserved      */
/* ------------------------------------------------------------------ */
/* out/in: full vectors of 2 checkerboards.  Wilson / DWF order odd half first
 * (d_op_wilson.C:257-334, d_op_dwf.C:316-507):
 *   t = kappa D(in_e, CHKB_EVEN) + in_o;  src = MatPcDag t;  CG on
 *   MatPcDagMatPc out_o = src from the guess in out_o;
 *   out_e = kappa D(out_o, CHKB_ODD) + in_e.
 * Mobius (SYM2) order even half first (d_op_mobius.C:389-640):
 *   t = kappa_b D4(M5^-1 in_e, CHKB_EVEN) + in_o;  out_o += (kappa_b/kappa_c)-weighted
 *   5th-direction hop of the guess;  src = MatPcDag t;  CG;
 *   out_o = M5^-1 out_o;  out_e = M5^-1 (kappa_b D4(out_o, CHKB_ODD)) + M5^-1 in_e;
 *   out *= 2 kappa_b.
 * Returns the CG iteration count; *true_res as InvCg reports it. */
int orc_matinv(const orc_op *op, double *out, const double *in, double stop_rsd, int max_num_iter,
               double *true_res) {
  const long n = orc_op_size(op);
  double *t = scratch(n), *src = scratch(n);
  int it;
  if (op->action != 2) {
    const double kappa = op->action == 0 ? 1.0 / (2.0 * (op->mass + 4.0))
                                         : 1.0 / (2 * (4 + op->a5_inv - op->m5));
    const double *in_o = in, *in_e = in + n;
    double *out_o = out, *out_e = out + n;
    orc_dslash(op, t, in_e, 0, 0);
    for (long i = 0; i < n; i++) t[i] = kappa * t[i] + in_o[i];   /* fTimesV1PlusV2 */
    orc_matpc(op, src, t, 1);
    it = orc_invcg(op, out_o, src, stop_rsd, max_num_iter, true_res, NULL);
    orc_dslash(op, t, out_o, 1, 0);
    for (long i = 0; i < n; i++) out_e[i] = kappa * t[i] + in_e[i];
  } else {
    orc_mobius_params p = op->mob;
    p.mass = op->mass;
    const int ls = p.ls;
    const long n4 = n / ls;
    cplx kb[64], kc[64], kr[64];
    mobius_kappas(&p, kb, kc, kr);
    const double *in_e = in, *in_o = in + n;
    double *out_e = out, *out_o = out + n;
    double *t2 = scratch(n);
    memcpy(t, in_e, n * sizeof(double));
    orc_mobius_m5inv(t, 0, op->dims, &p);
    orc_mobius_dslash_4(t2, op->u, t, 0, 0, op->dims, &p);
    for (int s = 0; s < ls; s++) {                                /* zmobius_zvectTimesV1PlusV2 */
      for (long i = 0; i < n4 / 2; i++) {
        cplx x = {t2[s * n4 + 2 * i], t2[s * n4 + 2 * i + 1]};
        cplx r = cmul(kb[s], x);
        t[s * n4 + 2 * i] = r.re + in_o[s * n4 + 2 * i];
        t[s * n4 + 2 * i + 1] = r.im + in_o[s * n4 + 2 * i + 1];
      }
    }
    if (p.pc_type == 2) {                                         /* SYM2: guess transform */
      memcpy(t2, out_o, n * sizeof(double));
      orc_zmobius_dslash_5_plus(out_o, t2, p.mass, 0, op->dims, ls, kr);
    }
    if (p.pc_type == 1) {                                         /* SYM1: source M5^-1 */
      orc_mobius_m5inv(t, 0, op->dims, &p);
    }
    orc_matpc(op, src, t, 1);
    it = orc_invcg(op, out_o, src, stop_rsd, max_num_iter, true_res, NULL);
    if (p.pc_type == 2) {
      memcpy(t, out_o, n * sizeof(double));
      orc_mobius_m5inv(t, 0, op->dims, &p);
      memcpy(out_o, t, n * sizeof(double));
    }
    orc_mobius_dslash_4(t, op->u, out_o, 1, 0, op->dims, &p);
    for (int s = 0; s < ls; s++) zscale(t + s * n4, kb[s], n4);   /* zmobius_zvectTimesEquComplex */
    memcpy(out_e, t, n * sizeof(double));
    orc_mobius_m5inv(out_e, 0, op->dims, &p);
    memcpy(t, in_e, n * sizeof(double));
    orc_mobius_m5inv(t, 0, op->dims, &p);
    for (long i = 0; i < n; i++) out_e[i] += t[i];               /* VecAddEquVec */
    const double two_kb = 2.0 * kb[0].re;
    for (long i = 0; i < 2 * n; i++) out[i] *= two_kb;
    free(t2);
  }
  free(t);
  free(src);
  return it;
}

/* DiracOpMobius::Dminus, d_op_mobius.C:745-777, on a full Mobius vector
 * (4-D-even half first) with mobius_dminus (mobius_dminus.C:29-86):
 *   out_e = D_W(odd -> even)(-c/2 in_o),  out_o = D_W(even -> odd)(-c/2 in_e)
 * on every s slice (fixed 4-D parity), then out = -((c (4 - M5) - a5_inv) in + out). */
int orc_mobius_dminus(const orc_op *op, double *out, const double *in) {
  if (op->action != 2) return -1;
  const long n = orc_op_size(op);
  const int ls = op->mob.ls;
  const long n4 = n / ls;
  const double c = op->mob.c[0][0];
  const double k = 0.5 * (2 * (c * (4 - op->m5) - op->a5_inv));
  double *t = scratch(n);
  for (int half = 0; half < 2; half++) {
    const double *src = in + (half ? 0 : n);   /* out_e from in_o, out_o from in_e */
    double *dst = out + (half ? n : 0);
    const int cb = half ? 0 : 1;               /* checkerboard of the input */
    for (long i = 0; i < n; i++) t[i] = src[i] * (-0.5 * c);
    for (int s = 0; s < ls; s++) orc_wilson_dslash(dst + s * n4, op->u, t + s * n4, cb, 0, op->dims);
  }
  for (long i = 0; i < 2 * n; i++) out[i] = -(k * in[i] + out[i]);
  free(t);
  return 0;
}

/* DiracOpZMobius::Dminus, d_op_zmobius.C:1213-1272, with zmobius_dminus
 * (d_op_zmobius/noarch/zmobius_dminus.C:44-116), on a full zMobius vector
 * (solve checkerboard -- odd -- half first): per slice s
 *   out_o = D_W(even -> odd)(-c_s/2 in_e),  out_e = D_W(odd -> even)(-c_s/2 in_o),
 * then out = -(k_s in + out), k_s = c_s (4 - M5) - a5_inv, all complex. */
int orc_zmobius_dminus(const orc_op *op, double *out, const double *in) {
  if (op->action != 2) return -1;
  const long n = orc_op_size(op);
  const int ls = op->mob.ls;
  const long n4 = n / ls;
  double *t = scratch(n);
  for (int half = 0; half < 2; half++) {
    const double *src = in + (half ? 0 : n);   /* out_o from in_e, out_e from in_o */
    double *dst = out + (half ? n : 0);
    const int cb = half ? 1 : 0;               /* checkerboard of the input */
    for (int s = 0; s < ls; s++) {
      const cplx c = {op->mob.c[s][0], op->mob.c[s][1]};
      zscale_copy(t + s * n4, src + s * n4, cscal(-0.5, c), n4);
    }
    for (int s = 0; s < ls; s++) orc_wilson_dslash(dst + s * n4, op->u, t + s * n4, cb, 0, op->dims);
  }
  for (int half = 0; half < 2; half++)
    for (int s = 0; s < ls; s++) {
      const cplx k = {op->mob.c[s][0] * (4 - op->m5) - op->a5_inv, op->mob.c[s][1] * (4 - op->m5)};
      double *o = out + half * n + s * n4;
      const double *x = in + half * n + s * n4;
      for (long i = 0; i < n4 / 2; i++) {      /* zTimesV1PlusV2: o = k x + o */
        const cplx xv = {x[2 * i], x[2 * i + 1]};
        const cplx r = cmul(k, xv);
        o[2 * i] = r.re + o[2 * i];
        o[2 * i + 1] = r.im + o[2 * i + 1];
      }
    }
  for (long i = 0; i < 2 * n; i++) out[i] = -out[i];
  free(t);
  return 0;
}

/* DiracOpZMobius::MatInv(out, in, true_res, PRESERVE_YES), d_op_zmobius.C:829-1080
 * (ZMOB_PC_SYM2 and ORIG), on full vectors with the solve checkerboard first:
 *   t = kb . D4(M5^-1 in_2, CHKB_EVEN) + in_1;  SYM2: out_1 = M5 out_1 (guess);
 *   src = MatPcDag t;  CG;  SYM2: out_1 = M5^-1 out_1;
 *   out_2 = M5^-1(kb . D4(out_1, CHKB_ODD)) + M5^-1 in_2   (no overall scale).
 * Returns the CG iteration count; *true_res as InvCg reports it. */
int orc_zmobius_matinv(const orc_op *op, double *out, const double *in, double stop_rsd, int max_num_iter,
                       double *true_res) {
  if (op->action != 2 || (op->mob.pc_type != 2 && op->mob.pc_type != 0 && op->mob.pc_type != 5)) return -1;
  const long n = orc_op_size(op);
  orc_mobius_params p = op->mob;
  p.mass = op->mass;
  const int ls = p.ls;
  const long n4 = n / ls;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(&p, kb, kc, kr);
  const double *in_1 = in, *in_2 = in + n;
  double *out_1 = out, *out_2 = out + n;
  double *t = scratch(n), *t2 = scratch(n), *src = scratch(n);
  memcpy(t, in_2, n * sizeof(double));
  orc_mobius_m5inv(t, 0, op->dims, &p);
  orc_mobius_dslash_4(t2, op->u, t, 0, 0, op->dims, &p);
  for (int s = 0; s < ls; s++)                                    /* zmobius_zvectTimesV1PlusV2 */
    for (long i = 0; i < n4 / 2; i++) {
      const cplx x = {t2[s * n4 + 2 * i], t2[s * n4 + 2 * i + 1]};
      const cplx r = cmul(kb[s], x);
      t[s * n4 + 2 * i] = r.re + in_1[s * n4 + 2 * i];
      t[s * n4 + 2 * i + 1] = r.im + in_1[s * n4 + 2 * i + 1];
    }
  const int sym23 = p.pc_type == 2 || p.pc_type == 5;
  if (sym23) {                                                    /* SYM2 / SYM3: guess transform */
    memcpy(t2, out_1, n * sizeof(double));
    orc_zmobius_dslash_5_plus(out_1, t2, p.mass, 0, op->dims, ls, kr);
  }
  orc_matpc(op, src, t, 1);
  const int it = orc_invcg(op, out_1, src, stop_rsd, max_num_iter, true_res, NULL);
  if (sym23) orc_mobius_m5inv(out_1, 0, op->dims, &p);
  orc_mobius_dslash_4(t, op->u, out_1, 1, 0, op->dims, &p);
  for (int s = 0; s < ls; s++) zscale(t + s * n4, kb[s], n4);    /* zmobius_zvectTimesEquComplex */
  memcpy(out_2, t, n * sizeof(double));
  orc_mobius_m5inv(out_2, 0, op->dims, &p);
  memcpy(t, in_2, n * sizeof(double));
  orc_mobius_m5inv(t, 0, op->dims, &p);
  for (long i = 0; i < n; i++) out_2[i] += t[i];                 /* VecAddEquVec */
  free(t);
  free(t2);
  free(src);
  return it;
}

/* Fzmobius::FmatInv's source scale (f_zmobius.C:70-130): both halves of a full
 * vector times 2 kappa_b(s) per slice (vecTimesEquComplex). */
int orc_zmobius_scale_2kb(const orc_op *op, double *v) {
  if (op->action != 2) return -1;
  const long n = orc_op_size(op);
  orc_mobius_params p = op->mob;
  p.mass = op->mass;
  const int ls = p.ls;
  const long n4 = n / ls;
  cplx kb[64], kc[64], kr[64];
  mobius_kappas(&p, kb, kc, kr);
  for (int h = 0; h < 2; h++)
    for (int s = 0; s < ls; s++) zscale(v + h * n + s * n4, cscal(2.0, kb[s]), n4);
  return 0;
}

/* ------------------------------------------------------------------ */
/* DiracOp::MinResExt, d_op_base/comsrc/minresext.C:32-156             */
/* ------------------------------------------------------------------ */
/* Chronological guess: orthonormalise the previous solutions v[0..degree)
 * in place (Gram-Schmidt with the complex dot conj(a).b), vm[i] =
 * MatPcDagMatPc v[i], G = v^dag A v (diagonal from the fused |M v|^2), solve
 * G a = v^dag phi by the reference's elimination (its pivot test compares
 * diagonal magnitudes), psi = sum a_i v_i.  Complex arithmetic uses C99
 * complex types, whose multiplication and division compile to the same
 * runtime routines as the reference's std::complex<double>.  Returns
 * |phi - A psi| / |phi|. */
static void cdot_seq(const double *a, const double *b, long len, double *re, double *im) {
  double r = 0.0, i = 0.0;
  for (long k = 0; k < len; k += 2) {
    r += a[k] * b[k] + a[k + 1] * b[k + 1];
    i += a[k] * b[k + 1] - a[k + 1] * b[k];
  }
  *re = r;
  *im = i;
}
static void caxpy_seq(double *a, double re, double im, const double *c, const double *d, long len) {
  for (long k = 0; k < len; k += 2) {
    const double c_re = c[k], c_im = c[k + 1];
    a[k] = re * c_re - im * c_im + d[k];
    a[k + 1] = re * c_im + im * c_re + d[k + 1];
  }
}
double orc_minresext(const orc_op *op, double *psi, const double *phi, double **v, double **vm, int degree) {
  const long n = orc_op_size(op);
  if (degree == 0) {
    memset(psi, 0, n * sizeof(double));
    return 1.0;
  }
  double _Complex G[16][16], a[16], b[16], xp;
  double re, im;
  for (int i = 0; i < degree; i++) {
    const double f = 1 / sqrt(dot_seq(v[i], v[i], n));
    for (long k = 0; k < n; k++) v[i][k] *= f;
    for (int j = i + 1; j < degree; j++) {
      cdot_seq(v[i], v[j], n, &re, &im);
      caxpy_seq(v[j], -re, -im, v[i], v[j], n);
    }
  }
  for (int i = 0; i < degree; i++) {
    cdot_seq(v[i], phi, n, &re, &im);
    b[i] = CMPLX(re, im);
    double dot = 0;
    orc_mdagm(op, vm[i], v[i], &dot);
    G[i][i] = CMPLX(dot, 0.0);
  }
  for (int j = 0; j < degree; j++)
    for (int k = j + 1; k < degree; k++) {
      cdot_seq(v[j], vm[k], n, &re, &im);
      G[j][k] = CMPLX(re, im);
      G[k][j] = conj(G[j][k]);
    }
  for (int i = 0; i < degree; i++) {
    int k = i;
    for (int j = i + 1; j < degree; j++)
      if (cabs(G[j][j]) > cabs(G[k][k])) k = j;
    if (k != i) {
      xp = b[k]; b[k] = b[i]; b[i] = xp;
      for (int j = 0; j < degree; j++) { xp = G[k][j]; G[k][j] = G[i][j]; G[i][j] = xp; }
    }
    for (int j = i + 1; j < degree; j++) {
      xp = G[j][i] / G[i][i];
      b[j] -= xp * b[i];
      for (int m = 0; m < degree; m++) G[j][m] -= xp * G[i][m];
    }
  }
  double *r = scratch(n);
  memset(psi, 0, n * sizeof(double));
  memcpy(r, phi, n * sizeof(double));
  for (int i = degree - 1; i >= 0; i--) {
    a[i] = CMPLX(0.0, 0.0);
    for (int j = i + 1; j < degree; j++) a[i] += G[i][j] * a[j];
    a[i] = (b[i] - a[i]) / G[i][i];
    caxpy_seq(psi, creal(a[i]), cimag(a[i]), v[i], psi, n);
    caxpy_seq(r, -creal(a[i]), -cimag(a[i]), vm[i], r, n);
  }
  const double err = sqrt(dot_seq(r, r, n) / dot_seq(phi, phi, n));
  free(r);
  return err;
}

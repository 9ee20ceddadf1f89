// blas.cu -- streaming kernels: CPS-order packing, precision conversion, the
// fused CG vector updates and generic axpby with deterministic norms.
//
// The CG updates restate DiracOp::InvCgShift (cps_pp/src/util/dirac_op/d_op_base/
// comsrc/inv_cg.C:322-360): a = |r|^2/d; x = a p + x; r = -a Ap + r; |r|^2;
// b = |r|^2_new/|r|^2_old; p = b p + r -- split over two kernels, with every
// scalar produced on the device by the last block of the reduction.
#include <math.h>
#include "cg_state.h"
#include "cpsb_kernels.h"
#include "blas.h"

namespace cpsb {

int grid_blocks(long sites_per_rhs, int nt) {
  long nb = (sites_per_rhs + nt - 1) / nt;
  const long cap = 148L * 16;  // grid-stride beyond this
  if (nb > cap) nb = cap;
  if (nb < 1) nb = 1;
  return (int)nb;
}

// ---------------------------------------------------------------- packing
// CPS order (right-hand side, then slice s, then 4-D checkerboard site x; 24
// doubles per site) <-> the column layout of cpsb_device.cuh.  Threads walk
// the device entries in order, so device chunks are read or written in whole
// 128-byte segments and each thread moves its site's 192 contiguous CPS bytes.
__device__ __forceinline__ long cps_index(const Geom &g, unsigned e) {
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  const unsigned rhs = e / per;
  const unsigned j = e - rhs * per;
  const int k = (g.ncls == 2 && j >= (unsigned)g.kb1) ? 1 : 0;
  const unsigned jj = j - (k ? (unsigned)g.kb1 : 0u);
  const unsigned c = (unsigned)g.cs[k];
  const unsigned x = jj / c, sp = jj - x * c;
  const unsigned s = g.ncls == 2 ? (unsigned)k + 2 * sp : sp;
  return (long)rhs * per + (long)s * g.n4cb + x;
}

template <int P>
__global__ void pack_kernel(SpinorPtr dst, const double *src, Geom g) {
  typedef typename PrecTraits<P>::real T;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < g.nsites; e += (long)gridDim.x * blockDim.x) {
    Spinor<T> s;
    const double2 *p = (const double2 *)(src + 24 * cps_index(g, (unsigned)e));
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 v = p[k];
      s.c[k / 3][k % 3] = mk((T)v.x, (T)v.y);
    }
    store_spinor<P>(dst, e, s);
  }
}

template <int P>
__global__ void unpack_kernel(double *dst, SpinorPtr src, Geom g) {
  typedef typename PrecTraits<P>::real T;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < g.nsites; e += (long)gridDim.x * blockDim.x) {
    Spinor<T> s = load_spinor<P>(src, e);
    double2 *p = (double2 *)(dst + 24 * cps_index(g, (unsigned)e));
#pragma unroll
    for (int k = 0; k < 12; k++) p[k] = make_double2((double)s.c[k / 3][k % 3].re, (double)s.c[k / 3][k % 3].im);
  }
}

template <int PD, int PS>
__global__ void convert_kernel(SpinorPtr dst, SpinorPtr src, long n) {
  typedef typename PrecTraits<PD>::real TD;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    store_spinor<PD>(dst, i, convert<TD>(load_spinor<PS>(src, i)));
  }
}

static int flat_grid(long n) {
  long nb = (n + 255) / 256;
  if (nb > 148L * 32) nb = 148L * 32;
  return (int)(nb < 1 ? 1 : nb);
}

cudaError_t launch_pack(int prec, SpinorPtr dst, const double *src, const Geom &g, cudaStream_t st) {
  const long n = g.nsites;
  if (prec == P64) pack_kernel<P64><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  else if (prec == P32) pack_kernel<P32><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  else pack_kernel<P16><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  return launched();
}

cudaError_t launch_unpack(int prec, double *dst, SpinorPtr src, const Geom &g, cudaStream_t st) {
  const long n = g.nsites;
  if (prec == P64) unpack_kernel<P64><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  else if (prec == P32) unpack_kernel<P32><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  else unpack_kernel<P16><<<flat_grid(n), 256, 0, st>>>(dst, src, g);
  return launched();
}

cudaError_t launch_convert(int pd, SpinorPtr dst, int ps, SpinorPtr src, long n, cudaStream_t st) {
  const int g = flat_grid(n);
#define CV(A, B) if (pd == A && ps == B) { convert_kernel<A, B><<<g, 256, 0, st>>>(dst, src, n); return launched(); }
  CV(P64, P64) CV(P64, P32) CV(P64, P16) CV(P32, P64) CV(P32, P32) CV(P32, P16) CV(P16, P64) CV(P16, P32) CV(P16, P16)
#undef CV
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------- gauge packing
// u: CANONICAL order (site x+lx*(y+ly*(z+lz*t)), link mu, row-major 3x3), as
// Lattice::GaugeField() holds it (lattice/convert/convert_func.C:397-405).
// FP64 keeps all 18 reals and folds the antiperiodic time sign into the links
// on the last time slice, as Lattice::BondCond does (lattice_base.C:5313-5370);
// FP32/FP16 keep rows 0 and 1 without the sign (the kernels apply it).
template <int P>
__global__ void gauge_pack_kernel(void *dst, const double *u, int lx, int ly, int lz, int lt, int bc_t) {
  const long vol = (long)lx * ly * lz * lt;
  const long n4cb = vol / 2;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < vol * 4; i += (long)gridDim.x * blockDim.x) {
    const long site = i >> 2;
    const int mu = (int)(i & 3);
    const int x = (int)(site % lx), y = (int)((site / lx) % ly), z = (int)((site / ((long)lx * ly)) % lz),
              t = (int)(site / ((long)lx * ly * lz));
    const int par = (x + y + z + t) & 1;
    const long cbi = x / 2 + (long)(lx / 2) * (y + (long)ly * (z + (long)lz * t));
    const double *m = u + 72 * site + 18 * mu;
    const double sg = (P == P64 && bc_t && mu == 3 && t == lt - 1) ? -1.0 : 1.0;
    if (P == P64) {
      double2 *d = (double2 *)dst;
      for (int k = 0; k < 9; k++) d[((long)(par * 4 + mu) * 9 + k) * n4cb + cbi] = make_double2(sg * m[2 * k], sg * m[2 * k + 1]);
    } else if (P == P32) {
      float4 *d = (float4 *)dst;
      for (int k = 0; k < 3; k++)
        d[((long)(par * 4 + mu) * 3 + k) * n4cb + cbi] =
            make_float4((float)m[4 * k], (float)m[4 * k + 1], (float)m[4 * k + 2], (float)m[4 * k + 3]);
    } else {
      uint2 *d = (uint2 *)dst;
      for (int k = 0; k < 3; k++) {
        uint2 v;
        v.x = enc16x2((float)m[4 * k], (float)m[4 * k + 1], 32767.0f);
        v.y = enc16x2((float)m[4 * k + 2], (float)m[4 * k + 3], 32767.0f);
        d[((long)(par * 4 + mu) * 3 + k) * n4cb + cbi] = v;
      }
    }
  }
}

// Lattice::Fconvert between CANONICAL and the checkerboarded fermion orders
// (lattice/convert/convert_func.C:429-495, convert.C:635-1010): a permutation
// of 24-real sites.  One thread moves one site (12 double2).  order 0: [odd |
// even] per 4-D slice, or for ls > 1 the 5-D checkerboard (sites with
// x+y+z+t+s odd first); order 1: DWF_4D_EOPREC_EE (4-D even half of every
// slice, then the odd half).  direction 0: CANONICAL -> order, 1: back.
__global__ void fconvert_kernel(double2 *out, const double2 *in, int lx, int ly, int lz, int lt, int ls, int order,
                                int direction) {
  const long vol = (long)lx * ly * lz * lt, h = vol / 2, n = vol * ls;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long s = i / vol, site = i - s * vol;
    const int x = (int)(site % lx), y = (int)((site / lx) % ly), z = (int)((site / ((long)lx * ly)) % lz),
              t = (int)(site / ((long)lx * ly * lz));
    const int par = (x + y + z + t) & 1;
    const long cbi = x / 2 + (long)(lx / 2) * (y + (long)ly * (z + (long)lz * t));
    int second;  // 1: the site goes to the second half
    if (order == 0) second = ls > 1 ? 1 - ((par + (int)s) & 1) : 1 - par;  // even (5-D / 4-D) sites second
    else second = par;                                                       // 4-D odd sites second
    const long j = second * ls * h + s * h + cbi;
    const double2 *src = in + 12 * (direction == 0 ? i : j);
    double2 *dst = out + 12 * (direction == 0 ? j : i);
#pragma unroll
    for (int k = 0; k < 12; k++) dst[k] = src[k];
  }
}

cudaError_t launch_fconvert(double *out, const double *in, const int dims[4], int ls, int order, int direction,
                            cudaStream_t st) {
  const long n = (long)dims[0] * dims[1] * dims[2] * dims[3] * ls;
  fconvert_kernel<<<flat_grid(n), 256, 0, st>>>((double2 *)out, (const double2 *)in, dims[0], dims[1], dims[2],
                                                dims[3], ls, order, direction);
  return launched();
}

cudaError_t launch_gauge_pack(int prec, void *dst, const double *u, const int dims[4], int bc_t, cudaStream_t st) {
  const long n = (long)dims[0] * dims[1] * dims[2] * dims[3] * 4;
  const int g = flat_grid(n);
  if (prec == P64) gauge_pack_kernel<P64><<<g, 256, 0, st>>>(dst, u, dims[0], dims[1], dims[2], dims[3], bc_t);
  else if (prec == P32) gauge_pack_kernel<P32><<<g, 256, 0, st>>>(dst, u, dims[0], dims[1], dims[2], dims[3], bc_t);
  else gauge_pack_kernel<P16><<<g, 256, 0, st>>>(dst, u, dims[0], dims[1], dims[2], dims[3], bc_t);
  return launched();
}

// Max deviation of row 2 from conj(row0 x row1) over all links with the
// antiperiodic sign removed: decides whether recon-12 storage is exact enough.
__global__ void unitarity_kernel(const double *u, long nlinks, int lx, int ly, int lz, int lt, int bc_t,
                                 unsigned long long *out_bits) {
  double worst = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nlinks; i += (long)gridDim.x * blockDim.x) {
    const double *m = u + 18 * i;
    for (int j = 0; j < 3; j++) {
      const int k = (j + 1) % 3, l = (j + 2) % 3;
      double ar = m[2 * k] * m[6 + 2 * l] - m[2 * k + 1] * m[6 + 2 * l + 1] - (m[2 * l] * m[6 + 2 * k] - m[2 * l + 1] * m[6 + 2 * k + 1]);
      double ai = m[2 * k] * m[6 + 2 * l + 1] + m[2 * k + 1] * m[6 + 2 * l] - (m[2 * l] * m[6 + 2 * k + 1] + m[2 * l + 1] * m[6 + 2 * k]);
      worst = fmax(worst, fabs(m[12 + 2 * j] - ar));
      worst = fmax(worst, fabs(m[12 + 2 * j + 1] + ai));
    }
  }
  atomicMax(out_bits, __double_as_longlong(worst));
}

cudaError_t launch_unitarity(const double *u, long nlinks, const int dims[4], int bc_t, unsigned long long *out,
                             cudaStream_t st) {
  unitarity_kernel<<<flat_grid(nlinks), 256, 0, st>>>(u, nlinks, dims[0], dims[1], dims[2], dims[3], bc_t, out);
  return launched();
}

// ---------------------------------------------------------------- CG updates
// r = r - alpha*Ap (alpha = rr/d from the device state), |r|^2 per RHS; the last
// block advances the recurrence scalars and decides whether this RHS halts.
template <int P, int NT>
__global__ void __launch_bounds__(NT) cg_r_update_kernel(Geom g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p, CgState *S, Reduce red) {
  typedef typename PrecTraits<P>::real T;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * g.ls;
  double acc = 0;
  if (!S->halt[rhs]) {
    const double sigma = S->shift;
    const double alpha = S->rr[rhs] / (S->d[rhs] + sigma * S->pp[rhs]);
    const T a = (T)alpha, ts = (T)sigma;
    for (long j = (long)blockIdx.x * NT + threadIdx.x; j < per; j += (long)gridDim.x * NT) {
      const long i = rhs * per + j;
      Spinor<T> rv = load_spinor<P>(r, i);
      Spinor<T> av = load_spinor<P>(Ap, i);
      if (sigma != 0.0) {
        const Spinor<T> pv = load_spinor<P>(p, i);
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) av.c[s][c] = av.c[s][c] + cscale(ts, pv.c[s][c]);
      }
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) rv.c[s][c] = rv.c[s][c] - cscale(a, av.c[s][c]);
      store_spinor<P>(r, i, rv);
      acc += norm2(rounded<P>(rv));
    }
  }
  double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[rhs * gridDim.x + blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int q = 0; q < g.nrhs; q++) {
      double c = ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0 && !S->halt[q]) {
        const double rprev = S->rr[q];
        const double d = S->d[q] + S->shift * S->pp[q];
        S->alpha[q] = rprev / d;
        S->rr_prev[q] = rprev;
        S->rr[q] = c;
        S->beta[q] = c / rprev;
        S->iters[q] += 1;
        int reason = HALT_NONE;
        const double rn = sqrt(c);
        if (!(d != 0.0) || !isfinite(c)) reason = HALT_BREAKDOWN;
        else if (c <= S->stp[q]) reason = HALT_CONVERGED;
        else if (S->iters[q] >= S->max_iter - 1) reason = HALT_MAXITER;
        else if (S->delta > 0 && rn < S->delta * S->maxr[q]) reason = HALT_RELIABLE;
        if (rn > S->maxr[q]) S->maxr[q] = rn;
        if (reason) { S->halt[q] = 1; S->reason[q] = reason; }
        if (red.result) red.result[q] = c;
      }
      __syncthreads();
    }
  }
}

// x = x + alpha p ; p = r + beta p (skipped in the iteration that halts).
template <int PX, int P, int NT>
__global__ void __launch_bounds__(NT) cg_xp_update_kernel(Geom g, SpinorPtr x, SpinorPtr p, SpinorPtr r, CgState *S,
                                                          Reduce red) {
  typedef typename PrecTraits<P>::real T;
  typedef typename PrecTraits<PX>::real TX;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * g.ls;
  const bool want_pp = S->shift != 0.0;
  double acc = 0;
  if (!S->halt_done[rhs]) {
    const double alpha = S->alpha[rhs], beta = S->beta[rhs];
    const bool upd_p = !S->halt[rhs];
    for (long j = (long)blockIdx.x * NT + threadIdx.x; j < per; j += (long)gridDim.x * NT) {
      const long i = rhs * per + j;
      Spinor<T> pv = load_spinor<P>(p, i);
      if (x.data) {  // x == null: the residual-update hop has made this update
        Spinor<TX> xv = load_spinor<PX>(x, i);
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            xv.c[s][c].re = (TX)(alpha * (double)pv.c[s][c].re) + xv.c[s][c].re;
            xv.c[s][c].im = (TX)(alpha * (double)pv.c[s][c].im) + xv.c[s][c].im;
          }
        store_spinor<PX>(x, i, xv);
      }
      if (upd_p) {
        Spinor<T> rv = load_spinor<P>(r, i);
        const T b = (T)beta;
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) pv.c[s][c] = cscale(b, pv.c[s][c]) + rv.c[s][c];
        store_spinor<P>(p, i, pv);
        if (want_pp) acc += norm2(rounded<P>(pv));
      }
    }
  }
  const double bsum = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[rhs * gridDim.x + blockIdx.x] = bsum;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int q = 0; q < g.nrhs; q++) {
      const double t = want_pp ? ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh) : 0.0;
      if (threadIdx.x == 0) {
        if (want_pp && !S->halt_done[q] && !S->halt[q]) S->pp[q] = t;
        S->halt_done[q] = S->halt[q];
      }
      __syncthreads();
    }
  }
}

cudaError_t launch_cg_r_update(int prec, const Geom &g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p, CgState *S, Reduce red,
                               cudaStream_t st) {
  dim3 grid(grid_blocks((long)g.n4cb * g.ls, 256), g.nrhs);
  if (prec == P64) cg_r_update_kernel<P64, 256><<<grid, 256, 0, st>>>(g, r, Ap, p, S, red);
  else if (prec == P32) cg_r_update_kernel<P32, 256><<<grid, 256, 0, st>>>(g, r, Ap, p, S, red);
  else cg_r_update_kernel<P16, 256><<<grid, 256, 0, st>>>(g, r, Ap, p, S, red);
  return launched();
}

cudaError_t launch_cg_xp_update(int px, int prec, const Geom &g, SpinorPtr x, SpinorPtr p, SpinorPtr r, CgState *S,
                                Reduce red, cudaStream_t st) {
  dim3 grid(grid_blocks((long)g.n4cb * g.ls, 256), g.nrhs);
  if (px == P64 && prec == P64) cg_xp_update_kernel<P64, P64, 256><<<grid, 256, 0, st>>>(g, x, p, r, S, red);
  else if (px == P32 && prec == P32) cg_xp_update_kernel<P32, P32, 256><<<grid, 256, 0, st>>>(g, x, p, r, S, red);
  else if (px == P32 && prec == P16) cg_xp_update_kernel<P32, P16, 256><<<grid, 256, 0, st>>>(g, x, p, r, S, red);
  else return cudaErrorInvalidValue;
  return launched();
}

// ---------------------------------------------------------------- axpby
// out = a[rhs]*X + b[rhs]*Y (Y optional), optional |out|^2 per RHS, optional
// per-RHS skip mask.  Precisions may differ; arithmetic in the wider type.
template <int PO, int PX, int PY, int NT>
__global__ void __launch_bounds__(NT) axpby_kernel(Geom g, SpinorPtr out, SpinorPtr X, SpinorPtr Y, Scal2 sc,
                                                   const int *skip, Reduce red, int norm) {
  typedef typename PrecTraits<PO>::real TO;
  typedef double TA;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * g.ls;
  double acc = 0;
  if (!(skip && skip[rhs])) {
    const TA a = sc.a[rhs], b = sc.b[rhs];
    for (long j = (long)blockIdx.x * NT + threadIdx.x; j < per; j += (long)gridDim.x * NT) {
      const long i = rhs * per + j;
      Spinor<TA> xv = convert<TA>(load_spinor<PX>(X, i));
      Spinor<TA> o;
      if (Y.data) {
        Spinor<TA> yv = convert<TA>(load_spinor<PY>(Y, i));
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) o.c[s][c] = cscale(a, xv.c[s][c]) + cscale(b, yv.c[s][c]);
      } else {
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int c = 0; c < 3; c++) o.c[s][c] = cscale(a, xv.c[s][c]);
      }
      Spinor<TO> ov = convert<TO>(o);
      store_spinor<PO>(out, i, ov);
      if (norm) acc += norm2(rounded<PO>(ov));
    }
  }
  if (norm) {
    double bs = block_sum<NT>(acc, sh);
    if (threadIdx.x == 0) red.partial[rhs * gridDim.x + blockIdx.x] = bs;
    if (last_block(red.ticket, gridDim.x * gridDim.y)) {
      for (int q = 0; q < g.nrhs; q++) {
        double c = ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh);
        if (threadIdx.x == 0 && !(skip && skip[q])) red.result[q] = c;
        __syncthreads();
      }
    }
  }
}

cudaError_t launch_axpby(int po, SpinorPtr out, int px, SpinorPtr X, int py, SpinorPtr Y, const Geom &g, Scal2 sc,
                         const int *skip, Reduce red, int norm, cudaStream_t st) {
  dim3 grid(grid_blocks((long)g.n4cb * g.ls, 256), g.nrhs);
#define AX(A, B, C)                                                                               \
  if (po == A && px == B && py == C) {                                                          \
    axpby_kernel<A, B, C, 256><<<grid, 256, 0, st>>>(g, out, X, Y, sc, skip, red, norm);        \
    return launched();                                                                  \
  }
  AX(P64, P64, P64) AX(P64, P64, P32) AX(P64, P32, P64) AX(P64, P16, P64) AX(P64, P64, P16)
  AX(P32, P32, P32) AX(P32, P64, P32) AX(P32, P32, P64) AX(P32, P16, P32) AX(P32, P32, P16)
  AX(P16, P16, P16) AX(P16, P64, P16) AX(P16, P16, P64) AX(P16, P32, P16) AX(P16, P64, P64)
  AX(P32, P64, P64) AX(P16, P32, P32) AX(P16, P16, P32)
#undef AX
  return cudaErrorInvalidValue;
}

// <X, Y> (real part) per RHS.
template <int P, int NT>
__global__ void __launch_bounds__(NT) redot_kernel(Geom g, SpinorPtr X, SpinorPtr Y, Reduce red) {
  typedef typename PrecTraits<P>::real T;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * g.ls;
  double acc = 0;
  for (long j = (long)blockIdx.x * NT + threadIdx.x; j < per; j += (long)gridDim.x * NT) {
    const long i = rhs * per + j;
    acc += redot(load_spinor<P>(X, i), load_spinor<P>(Y, i));
  }
  double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[rhs * gridDim.x + blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int q = 0; q < g.nrhs; q++) {
      double c = ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0) red.result[q] = c;
      __syncthreads();
    }
  }
}

// conj(X).Y of FP64 fields (one RHS): result[0] = real part, result[1] =
// imaginary part (Vector::CompDotProductGlbSum, vector/comsrc/vector.C:196);
// every double2 chunk is one complex number.
template <int NT>
__global__ void __launch_bounds__(NT) cdot_kernel(long nchunks, const double2 *X, const double2 *Y, Reduce red) {
  __shared__ double sh[NT / 32];
  double re = 0, im = 0;
  for (long j = (long)blockIdx.x * NT + threadIdx.x; j < nchunks; j += (long)gridDim.x * NT) {
    const double2 a = X[j], b = Y[j];
    re += a.x * b.x + a.y * b.y;
    im += a.x * b.y - a.y * b.x;
  }
  const double br = block_sum<NT>(re, sh);
  const double bi = block_sum<NT>(im, sh);
  if (threadIdx.x == 0) {
    red.partial[blockIdx.x] = br;
    red.partial[gridDim.x + blockIdx.x] = bi;
  }
  if (last_block(red.ticket, gridDim.x)) {
    for (int q = 0; q < 2; q++) {
      const double c = ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0) red.result[q] = c;
      __syncthreads();
    }
  }
}

cudaError_t launch_cdot(SpinorPtr X, SpinorPtr Y, long nsites, Reduce red, cudaStream_t st) {
  const long nch = nsites * 12;  // FP64 chunked layout: 12 complex chunks per site, contiguous per chunk array
  if (X.stride != nsites || Y.stride != nsites) return cudaErrorInvalidValue;
  cdot_kernel<256><<<grid_blocks(nch, 256), 256, 0, st>>>(nch, (const double2 *)X.data, (const double2 *)Y.data,
                                                            red);
  return launched();
}

// out = c X + Y on FP64 fields (Vector::CTimesV1PlusV2, vector_util.C:910).
__global__ void caxpy_kernel(long nchunks, double2 *out, double cr, double ci, const double2 *X, const double2 *Y) {
  for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < nchunks; j += (long)gridDim.x * blockDim.x) {
    const double2 x = X[j], y = Y[j];
    out[j] = make_double2(cr * x.x - ci * x.y + y.x, cr * x.y + ci * x.x + y.y);
  }
}

cudaError_t launch_caxpy(SpinorPtr out, double cr, double ci, SpinorPtr X, SpinorPtr Y, long nsites, cudaStream_t st) {
  const long nch = nsites * 12;
  if (out.stride != nsites || X.stride != nsites || Y.stride != nsites) return cudaErrorInvalidValue;
  caxpy_kernel<<<flat_grid(nch), 256, 0, st>>>(nch, (double2 *)out.data, cr, ci, (const double2 *)X.data,
                                               (const double2 *)Y.data);
  return launched();
}

cudaError_t launch_redot(int prec, const Geom &g, SpinorPtr X, SpinorPtr Y, Reduce red, cudaStream_t st) {
  dim3 grid(grid_blocks((long)g.n4cb * g.ls, 256), g.nrhs);
  if (prec == P64) redot_kernel<P64, 256><<<grid, 256, 0, st>>>(g, X, Y, red);
  else if (prec == P32) redot_kernel<P32, 256><<<grid, 256, 0, st>>>(g, X, Y, red);
  else redot_kernel<P16, 256><<<grid, 256, 0, st>>>(g, X, Y, red);
  return launched();
}

}  // namespace cpsb

// dslash.cu -- checkerboarded Wilson / domain-wall hopping kernels for sm_100a.
//
// One thread per output site of a (possibly 5-D, possibly multi-RHS) checkerboard
// field.  The 4-D hop restates CPS's wilson_dslash (cps_pp/src/util/dirac_op/
// d_op_wilson/noarch/wilson_dslash.C:173-516) with spin projection: each of the
// 8 neighbours is projected to a half spinor, multiplied by the link (or its
// adjoint) and re-expanded into the accumulator.  For Shamir DWF the slices use
// 5-D checkerboarding (dwf_dslash_4.C:107-112: slice s holds 4-D parity
// (s+cb)%2) and the 5th-direction hop of dwf_dslash_5_plus.C:111-340 is fused
// into the same kernel.  For Mobius every slice carries the same 4-D parity
// (the DWF_4D_EOPREC_EE layout, d_op_mobius/d_op_mobius.C:75).
//
// Epilogues (fused, no extra pass over memory):
//   out = a * D in                         (EPI_SCALE)
//   out = x + a * D in                     (EPI_XPAY)   e.g. M = 1 - kappa^2 D D
// each optionally accumulating |out|^2 per right-hand side with a
// deterministic two-level reduction.
#include "cpsb_device.cuh"
#include "cpsb_kernels.h"

namespace cpsb {

template <int P, int NT, bool XPAY, bool NORM>
__global__ void __launch_bounds__(NT) dslash_kernel(DslashArgs A) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  __shared__ double red[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * g.ls;
  double nrm = 0;
  const bool skip = A.skip && A.skip[rhs];
  const T sdag = A.dag ? T(-1) : T(1);
  const int L[4] = {g.lx, g.ly, g.lz, g.lt};
  for (long j = (long)blockIdx.x * NT + threadIdx.x; !skip && j < per; j += (long)gridDim.x * NT) {
    const long i = rhs * per + j;
    const int x = (int)(j % g.n4cb);
    const int s = (int)(j / g.n4cb);
    const long sbase = i - x;                       // first site of this slice
    const int par_out = A.five_d ? ((1 - A.cb + s) & 1) : (1 - A.cb);
    const int par_in = 1 - par_out;
    const Coord c = decode(g, x, par_out);
    Spinor<T> acc;
    zero(acc);
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      int p[4] = {c.x, c.y, c.z, c.t};
      p[mu] = (p[mu] + 1 == L[mu]) ? 0 : p[mu] + 1;
      const int xf = cbindex(g, p[0], p[1], p[2], p[3]);
      Spinor<T> nb = load_spinor<P>(A.in, sbase + xf);
      Half<T> h = project(nb, mu, -sdag);
      Link<T> l = load_link<P>(A.U, par_out, mu, x);
      Half<T> uh = umul(l, h);
      if (mu == 3 && A.bc_t_sign < 0 && c.t == g.lt - 1) {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) uh.c[a][r] = cscale(T(-1), uh.c[a][r]);
      }
      accum_reconstruct(acc, uh, mu, -sdag);
    }
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      int p[4] = {c.x, c.y, c.z, c.t};
      p[mu] = (p[mu] == 0) ? L[mu] - 1 : p[mu] - 1;
      const int xb = cbindex(g, p[0], p[1], p[2], p[3]);
      Spinor<T> nb = load_spinor<P>(A.in, sbase + xb);
      Half<T> h = project(nb, mu, sdag);
      Link<T> l = load_link<P>(A.U, par_in, mu, xb);
      Half<T> uh = umul_dag(l, h);
      if (mu == 3 && A.bc_t_sign < 0 && c.t == 0) {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) uh.c[a][r] = cscale(T(-1), uh.c[a][r]);
      }
      accum_reconstruct(acc, uh, mu, sdag);
    }
    if (A.hop5) {
      // 5th-direction hop: upper (lower) chirality from s-1 (s+1) for dag=0,
      // swapped for dag=1; -m_f times the factor across the walls.
      const int ls = g.ls;
      const long rbase = rhs * per;  // slice 0 of this RHS
      const int sm = (s == 0) ? ls - 1 : s - 1;
      const int sp = (s == ls - 1) ? 0 : s + 1;
      const T fm = (T)((s == 0) ? A.hop5_wall : A.hop5_fact);
      const T fp = (T)((s == ls - 1) ? A.hop5_wall : A.hop5_fact);
      Spinor<T> vm = load_spinor<P>(A.in, rbase + (long)sm * g.n4cb + x);
      Spinor<T> vp = load_spinor<P>(A.in, rbase + (long)sp * g.n4cb + x);
      if (!A.dag) {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) {
            acc.c[a][r] = acc.c[a][r] + cscale(fm, vm.c[a][r]);
            acc.c[2 + a][r] = acc.c[2 + a][r] + cscale(fp, vp.c[2 + a][r]);
          }
      } else {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) {
            acc.c[2 + a][r] = acc.c[2 + a][r] + cscale(fm, vm.c[2 + a][r]);
            acc.c[a][r] = acc.c[a][r] + cscale(fp, vp.c[a][r]);
          }
      }
    }
    const T a = (T)A.a;
    if (XPAY) {
      Spinor<T> xv = load_spinor<P>(A.x, i);
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = xv.c[s2][r] + cscale(a, acc.c[s2][r]);
    } else if (A.a != 1.0) {
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = cscale(a, acc.c[s2][r]);
    }
    store_spinor<P>(A.out, i, acc);
    if (NORM) nrm += norm2(rounded<P>(acc));
  }
  if (NORM) {
    double bs = block_sum<NT>(nrm, red);
    if (threadIdx.x == 0) A.red.partial[rhs * gridDim.x + blockIdx.x] = bs;
    if (last_block(A.red.ticket, gridDim.x * gridDim.y)) {
      for (int q = 0; q < g.nrhs; q++) {
        double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) A.red.result[q] = t;
        __syncthreads();
      }
    }
  }
}

template <int P, int NT>
static cudaError_t launch_nt(const DslashArgs &A, int xpay, int norm, cudaStream_t st) {
  dim3 grid(grid_blocks((long)A.g.n4cb * A.g.ls, NT), A.g.nrhs);
  if (xpay && norm) dslash_kernel<P, NT, true, true><<<grid, NT, 0, st>>>(A);
  else if (xpay) dslash_kernel<P, NT, true, false><<<grid, NT, 0, st>>>(A);
  else if (norm) dslash_kernel<P, NT, false, true><<<grid, NT, 0, st>>>(A);
  else dslash_kernel<P, NT, false, false><<<grid, NT, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_dslash(int prec, const DslashArgs &A, int xpay, int norm, int nt, cudaStream_t st) {
  if (prec == P64) {
    if (nt == 64) return launch_nt<P64, 64>(A, xpay, norm, st);
    if (nt == 256) return launch_nt<P64, 256>(A, xpay, norm, st);
    return launch_nt<P64, 128>(A, xpay, norm, st);
  }
  if (prec == P32) {
    if (nt == 64) return launch_nt<P32, 64>(A, xpay, norm, st);
    if (nt == 256) return launch_nt<P32, 256>(A, xpay, norm, st);
    return launch_nt<P32, 128>(A, xpay, norm, st);
  }
  if (nt == 64) return launch_nt<P16, 64>(A, xpay, norm, st);
  if (nt == 256) return launch_nt<P16, 256>(A, xpay, norm, st);
  return launch_nt<P16, 128>(A, xpay, norm, st);
}

}  // namespace cpsb

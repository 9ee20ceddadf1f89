// dslash_impl.cuh -- checkerboarded Wilson / domain-wall hopping kernels for sm_100a.
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
#pragma once
#include "cpsb_device.cuh"
#include "cg_state.h"
#include "cpsb_kernels.h"

namespace cpsb {

// Thread mapping: a block owns a tile of TX consecutive checkerboard sites x
// and sweeps every slice (and right-hand side) of that tile, so each link is
// fetched from DRAM once per tile and served from L1 to all slices.  Threads
// of a block are TX x SL (x fastest, so a warp reads 32 consecutive sites);
// a thread handles SPT slices s, s+SL, ... that share the 4-D parity (SL even
// or 4-D checkerboarding), loading and unpacking each link once for all of them.
template <int P, int SPT>
__device__ __forceinline__ void hop_slices(const DslashArgs &A, int x, int par_out, const long *sbase,
                                           Spinor<typename PrecTraits<P>::real> *acc) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  const int par_in = 1 - par_out;
  const T sdag = A.dag ? T(-1) : T(1);
  const Coord c = decode(g, x, par_out);
  const int L[4] = {g.lx, g.ly, g.lz, g.lt};
#pragma unroll
  for (int k = 0; k < SPT; k++) zero(acc[k]);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    int p[4] = {c.x, c.y, c.z, c.t};
    p[mu] = (p[mu] + 1 == L[mu]) ? 0 : p[mu] + 1;
    const int xf = cbindex(g, p[0], p[1], p[2], p[3]);
    const Link<T> l = load_link<P>(A.U, par_out, mu, x);
    const bool flip = (mu == 3 && A.bc_t_sign < 0 && c.t == g.lt - 1);
#pragma unroll
    for (int k = 0; k < SPT; k++) {
      Half<T> h = project(load_spinor<P>(A.in, sbase[k] + xf), mu, -sdag);
      Half<T> uh = umul(l, h);
      if (flip) {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) uh.c[a][r] = cscale(T(-1), uh.c[a][r]);
      }
      accum_reconstruct(acc[k], uh, mu, -sdag);
    }
  }
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    int p[4] = {c.x, c.y, c.z, c.t};
    p[mu] = (p[mu] == 0) ? L[mu] - 1 : p[mu] - 1;
    const int xb = cbindex(g, p[0], p[1], p[2], p[3]);
    const Link<T> l = load_link<P>(A.U, par_in, mu, xb);
    const bool flip = (mu == 3 && A.bc_t_sign < 0 && c.t == 0);
#pragma unroll
    for (int k = 0; k < SPT; k++) {
      Half<T> h = project(load_spinor<P>(A.in, sbase[k] + xb), mu, sdag);
      Half<T> uh = umul_dag(l, h);
      if (flip) {
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int r = 0; r < 3; r++) uh.c[a][r] = cscale(T(-1), uh.c[a][r]);
      }
      accum_reconstruct(acc[k], uh, mu, sdag);
    }
  }
}

// 5th-direction hop of dwf_dslash_5_plus: upper (lower) chirality from s-1
// (s+1) for dag=0, swapped for dag=1; -m_f times the factor across the walls.
template <int P>
__device__ __forceinline__ void hop5_add(const DslashArgs &A, int x, int s, long rbase,
                                         Spinor<typename PrecTraits<P>::real> &acc) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  const int ls = g.ls;
  const int sm = (s == 0) ? ls - 1 : s - 1;
  const int sp = (s == ls - 1) ? 0 : s + 1;
  const T fm = (T)((s == 0) ? A.hop5_wall : A.hop5_fact);
  const T fp = (T)((s == ls - 1) ? A.hop5_wall : A.hop5_fact);
  const Spinor<T> vm = load_spinor<P>(A.in, rbase + (long)sm * g.n4cb + x);
  const Spinor<T> vp = load_spinor<P>(A.in, rbase + (long)sp * g.n4cb + x);
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

template <int P, int NT, int MINB, int SPT, bool XPAY, bool NORM>
__global__ void __launch_bounds__(NT, MINB) dslash_kernel(DslashArgs A) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  __shared__ double red[NT / 32];
  const int SL = A.sl;          // slice lanes per block (host: SL*SPT divides ls)
  const int TX = NT / SL;
  const int tx = threadIdx.x % TX, sl = threadIdx.x / TX;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int per = g.n4cb * g.ls;
  // Per-thread, per-RHS norm accumulators in shared memory (deterministic:
  // every slot has one owner; the block then reduces the slots in order).
  extern __shared__ double nrm_sh[];
  if (NORM)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const T a = (T)A.a;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x = tile * TX + tx;
    if (x >= g.n4cb) continue;
    for (int rhs = 0; rhs < g.nrhs; rhs++) {
      if (A.skip && A.skip[rhs]) continue;
      const long rbase = (long)rhs * per;
      for (int s0 = sl; s0 < g.ls; s0 += SL * SPT) {
        const int par_out = A.five_d ? ((1 - A.cb + s0) & 1) : (1 - A.cb);
        long sbase[SPT];
#pragma unroll
        for (int k = 0; k < SPT; k++) sbase[k] = rbase + (long)(s0 + k * SL) * g.n4cb;
        Spinor<T> acc[SPT];
        hop_slices<P, SPT>(A, x, par_out, sbase, acc);
#pragma unroll
        for (int k = 0; k < SPT; k++) {
          const int s = s0 + k * SL;
          const long i = sbase[k] + x;
          if (A.hop5) hop5_add<P>(A, x, s, rbase, acc[k]);
          if (XPAY) {
            const Spinor<T> xv = load_spinor<P>(A.x, i);
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
              for (int r = 0; r < 3; r++) acc[k].c[s2][r] = xv.c[s2][r] + cscale(a, acc[k].c[s2][r]);
          } else if (A.a != 1.0) {
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
              for (int r = 0; r < 3; r++) acc[k].c[s2][r] = cscale(a, acc[k].c[s2][r]);
          }
          store_spinor<P>(A.out, i, acc[k]);
          if (NORM) {
            nrm_sh[rhs * NT + threadIdx.x] += norm2(rounded<P>(acc[k]));
          }
        }
      }
    }
  }
  if (NORM) {
    for (int q = 0; q < g.nrhs; q++) {
      const double bs = block_sum<NT>(nrm_sh[q * NT + threadIdx.x], red);
      if (threadIdx.x == 0) A.red.partial[q * gridDim.x + blockIdx.x] = bs;
    }
    if (last_block(A.red.ticket, gridDim.x)) {
      for (int q = 0; q < g.nrhs; q++) {
        double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) A.red.result[q] = t;
        __syncthreads();
      }
    }
  }
}

// Largest power-of-two slice-lane count <= NT/32 with SL*SPT dividing ls.
static inline int slice_lanes(int nt, int spt, int ls) {
  int sl = 1;
  for (int c = 2; c <= nt / 32; c *= 2)
    if (ls % (c * spt) == 0) sl = c;
  return sl;
}

template <int P, int NT, int MINB, int SPT>
static cudaError_t dslash_launch_v(DslashArgs A, int xpay, int norm, cudaStream_t st) {
  // Shapes that do not fit this lattice report cudaErrorNotSupported without launching.
  if (A.g.ls % SPT) return cudaErrorNotSupported;
  A.sl = slice_lanes(NT, SPT, A.g.ls);
  if (SPT > 1 && A.five_d && (A.sl % 2)) return cudaErrorNotSupported;  // a thread's slices must share parity
  const int tx = NT / A.sl;
  const long ntiles = (A.g.n4cb + tx - 1) / tx;
  long nb = ntiles < 148L * 16 ? ntiles : 148L * 16;
  dim3 grid((unsigned)nb, 1);
  const size_t shm = norm ? sizeof(double) * NT * A.g.nrhs : 0;
  if (xpay && norm) dslash_kernel<P, NT, MINB, SPT, true, true><<<grid, NT, shm, st>>>(A);
  else if (xpay) dslash_kernel<P, NT, MINB, SPT, true, false><<<grid, NT, 0, st>>>(A);
  else if (norm) dslash_kernel<P, NT, MINB, SPT, false, true><<<grid, NT, shm, st>>>(A);
  else dslash_kernel<P, NT, MINB, SPT, false, false><<<grid, NT, 0, st>>>(A);
  return launched();
}

// Launch shapes the autotuner chooses from: (threads, min blocks/SM, slices per thread).
template <int P>
static cudaError_t dslash_launch_p(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  switch (variant) {
    case 1: return dslash_launch_v<P, 128, 3, 1>(A, xpay, norm, st);
    case 2: return dslash_launch_v<P, 256, 2, 1>(A, xpay, norm, st);
    case 3: return dslash_launch_v<P, 128, 4, 1>(A, xpay, norm, st);
    case 4: return dslash_launch_v<P, 128, 2, 2>(A, xpay, norm, st);
    case 5: return dslash_launch_v<P, 256, 1, 2>(A, xpay, norm, st);
    default: return dslash_launch_v<P, 128, 1, 1>(A, xpay, norm, st);
  }
}

}  // namespace cpsb

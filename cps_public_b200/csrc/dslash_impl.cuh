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
// and sweeps every slice (and right-hand side) of that tile.  Threads of a
// block are TX x SL (x fastest, so a warp reads 32 consecutive sites).
// With the link cache (LC) the block first unpacks the 8 links of every site
// of the tile (forward links at x, backward links at x-mu), for each 4-D parity
// its slices need, into shared memory; every slice then reads them from there,
// so a link is fetched, decoded and reconstructed once per tile instead of once
// per slice.  Without it each slice loads its links through L1.
template <typename T> struct LinkCache {
  cplx<T> *sh;  // [(pidx*8 + j)*9 + k][TX]
  int TX;
  __device__ __forceinline__ void put(int pidx, int j, int xi, const Link<T> &l) {
#pragma unroll
    for (int k = 0; k < 9; k++) sh[((pidx * 8 + j) * 9 + k) * TX + xi] = l.u[k / 3][k % 3];
  }
  __device__ __forceinline__ Link<T> get(int pidx, int j, int xi) const {
    Link<T> l;
#pragma unroll
    for (int k = 0; k < 9; k++) l.u[k / 3][k % 3] = sh[((pidx * 8 + j) * 9 + k) * TX + xi];
    return l;
  }
};

template <int P, bool LC>
__device__ __forceinline__ void hop_site(const DslashArgs &A, int x, int xi, int par_out, int pidx, long sbase,
                                         const LinkCache<typename PrecTraits<P>::real> &lc,
                                         Spinor<typename PrecTraits<P>::real> &acc) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  const int par_in = 1 - par_out;
  const T sdag = A.dag ? T(-1) : T(1);
  const Coord c = decode(g, x, par_out);
  const int L[4] = {g.lx, g.ly, g.lz, g.lt};
  zero(acc);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    int p[4] = {c.x, c.y, c.z, c.t};
    p[mu] = (p[mu] + 1 == L[mu]) ? 0 : p[mu] + 1;
    const int xf = cbindex(g, p[0], p[1], p[2], p[3]);
    Half<T> h = project(load_spinor<P>(A.in, sbase + xf), mu, -sdag);
    const Link<T> l = LC ? lc.get(pidx, mu, xi) : load_link<P>(A.U, par_out, mu, x);
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
    Half<T> h = project(load_spinor<P>(A.in, sbase + xb), mu, sdag);
    const Link<T> l = LC ? lc.get(pidx, 4 + mu, xi) : load_link<P>(A.U, par_in, mu, xb);
    Half<T> uh = umul_dag(l, h);
    if (mu == 3 && A.bc_t_sign < 0 && c.t == 0) {
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int r = 0; r < 3; r++) uh.c[a][r] = cscale(T(-1), uh.c[a][r]);
    }
    accum_reconstruct(acc, uh, mu, sdag);
  }
}

// 5th-direction hop of dwf_dslash_5_plus: upper (lower) chirality from s-1
// (s+1) for dag=0, swapped for dag=1; -m_f times the factor across the walls.
// Only the chiral half that is used is loaded.
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

template <int P, int NT, int MINB, bool LC, bool XPAY, bool NORM>
__global__ void __launch_bounds__(NT, MINB) dslash_kernel(DslashArgs A) {
  typedef typename PrecTraits<P>::real T;
  const Geom &g = A.g;
  __shared__ double red[NT / 32];
  extern __shared__ double dyn_sh[];
  const int SL = A.sl;          // slice lanes per block (host: SL divides ls)
  const int TX = NT / SL;
  const int tx = threadIdx.x % TX, sl = threadIdx.x / TX;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int per = g.n4cb * g.ls;
  const int npar = A.five_d ? 2 : 1;
  // dynamic shared memory: [link cache][per-thread, per-RHS norm slots]
  LinkCache<T> lc;
  lc.sh = (cplx<T> *)dyn_sh;
  lc.TX = TX;
  double *nrm_sh = dyn_sh + (LC ? (size_t)npar * 8 * 9 * TX * sizeof(cplx<T>) / sizeof(double) : 0);
  if (NORM)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const T a = (T)A.a;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (LC) {
      __syncthreads();  // the previous tile is done with the cache
      const int items = TX * npar * 8;
      for (int it = threadIdx.x; it < items; it += NT) {
        const int xi = it % TX;
        const int j = (it / TX) % 8;
        const int pidx = it / (TX * 8);
        const int xx = tile * TX + xi;
        if (xx >= g.n4cb) continue;
        const int po = A.five_d ? pidx : 1 - A.cb;
        Link<T> l;
        if (j < 4) {
          l = load_link<P>(A.U, po, j, xx);
        } else {
          const int mu = j - 4;
          const Coord c = decode(g, xx, po);
          int p[4] = {c.x, c.y, c.z, c.t};
          const int L[4] = {g.lx, g.ly, g.lz, g.lt};
          p[mu] = (p[mu] == 0) ? L[mu] - 1 : p[mu] - 1;
          l = load_link<P>(A.U, 1 - po, mu, cbindex(g, p[0], p[1], p[2], p[3]));
        }
        lc.put(pidx, j, xi, l);
      }
      __syncthreads();
    }
    const int x = tile * TX + tx;
    if (x >= g.n4cb) continue;
    for (int rhs = 0; rhs < g.nrhs; rhs++) {
      if (A.skip && A.skip[rhs]) continue;
      const long rbase = (long)rhs * per;
      for (int s = sl; s < g.ls; s += SL) {
        const int par_out = A.five_d ? ((1 - A.cb + s) & 1) : (1 - A.cb);
        const int pidx = A.five_d ? par_out : 0;
        const long sbase = rbase + (long)s * g.n4cb;
        Spinor<T> acc;
        hop_site<P, LC>(A, x, tx, par_out, pidx, sbase, lc, acc);
        const long i = sbase + x;
        if (A.hop5) hop5_add<P>(A, x, s, rbase, acc);
        if (XPAY) {
          const Spinor<T> xv = load_spinor<P>(A.x, i);
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
        if (NORM) nrm_sh[rhs * NT + threadIdx.x] += norm2(rounded<P>(acc));
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

// Largest power-of-two slice-lane count <= NT/32 that divides ls.
static inline int slice_lanes(int nt, int ls) {
  int sl = 1;
  for (int c = 2; c <= nt / 32; c *= 2)
    if (ls % c == 0) sl = c;
  return sl;
}

template <int P, int NT, int MINB, bool LC>
static cudaError_t dslash_launch_v(DslashArgs A, int xpay, int norm, cudaStream_t st) {
  typedef typename PrecTraits<P>::real T;
  A.sl = slice_lanes(NT, A.g.ls);
  // The link cache pays off only when several slices share a tile's links.
  if (LC && A.g.ls * A.g.nrhs < 4) return cudaErrorNotSupported;
  const int tx = NT / A.sl;
  const long ntiles = (A.g.n4cb + tx - 1) / tx;
  long nb = ntiles < 148L * 16 ? ntiles : 148L * 16;
  const int npar = A.five_d ? 2 : 1;
  size_t shm = LC ? (size_t)npar * 8 * 9 * tx * sizeof(cplx<T>) : 0;
  if (norm) shm += sizeof(double) * NT * A.g.nrhs;
  if (shm > 200 * 1024) return cudaErrorNotSupported;  // above the opt-in set below
  static bool attr_set[2][2] = {{false, false}, {false, false}};
  if (shm + 1024 > 48 * 1024) {  // the 48 KB default counts static shared memory too
    auto set = [&](const void *f) { return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); };
    cudaError_t e = cudaSuccess;
    if (!attr_set[xpay][norm]) {
      if (xpay && norm) e = set((const void *)dslash_kernel<P, NT, MINB, LC, true, true>);
      else if (xpay) e = set((const void *)dslash_kernel<P, NT, MINB, LC, true, false>);
      else if (norm) e = set((const void *)dslash_kernel<P, NT, MINB, LC, false, true>);
      else e = set((const void *)dslash_kernel<P, NT, MINB, LC, false, false>);
      if (e != cudaSuccess) return e;
      attr_set[xpay][norm] = true;
    }
  }
  dim3 grid((unsigned)nb, 1);
  if (xpay && norm) dslash_kernel<P, NT, MINB, LC, true, true><<<grid, NT, shm, st>>>(A);
  else if (xpay) dslash_kernel<P, NT, MINB, LC, true, false><<<grid, NT, shm, st>>>(A);
  else if (norm) dslash_kernel<P, NT, MINB, LC, false, true><<<grid, NT, shm, st>>>(A);
  else dslash_kernel<P, NT, MINB, LC, false, false><<<grid, NT, shm, st>>>(A);
  return launched();
}

// Launch shapes the autotuner chooses from: (threads, min blocks/SM, link cache).
template <int P>
static cudaError_t dslash_launch_p(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  if (A.cg) return cudaErrorNotSupported;  // the fused residual update is FP32 / 16-bit only
  switch (variant) {
    case 1: return dslash_launch_v<P, 128, 4, false>(A, xpay, norm, st);
    case 2: return dslash_launch_v<P, 256, 2, false>(A, xpay, norm, st);
    case 3: return dslash_launch_v<P, 128, 1, true>(A, xpay, norm, st);
    case 4: return dslash_launch_v<P, 256, 1, true>(A, xpay, norm, st);
    case 5: return dslash_launch_v<P, 256, 2, true>(A, xpay, norm, st);
    case 6: return dslash_launch_v<P, 128, 4, true>(A, xpay, norm, st);
    case 0: return dslash_launch_v<P, 128, 1, false>(A, xpay, norm, st);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace cpsb

// cg_persistent.cu -- every iteration of an FP64 CG solve on a small lattice in
// one cooperative kernel.
//
// On lattices where one CG iteration is a few microseconds of device work (the
// Wilson 8^4 workload has 2048 sites per checkerboard), the launch-per-step
// loop of solver.cu is bound by launch and scheduling latency, not bandwidth.
// Here a single cooperative launch runs the iterations of DiracOp::InvCg
// (cps_pp/src/util/dirac_op/d_op_base/comsrc/inv_cg.C:293-364) until every
// right-hand side halts: the four hops of MatPcDagMatPc (the residual update
// r -= alpha A p, |r|^2 and x += alpha p fused into the last one, as in the
// launch-per-step loop), then p = r + beta p, separated by grid barriers.
// Every block keeps its own copy of the recurrence scalars (CgState) in shared
// memory and sums the per-block partials of each reduction in block order, so
// all blocks hold identical scalars and take the same branches; block 0
// writes the state back when the loop ends.  Fields written inside the launch
// are read through L2 (ld.global.cg), never through the read-only cache.
//
// Two forms.  On fields of at most PCG_DP_SITES entries (all right-hand sides)
// the hops run with eight lanes per entry and the direction update rides on the
// next iteration's first two hops, so an iteration is four hops and four grid
// barriers; measured on B200 this beats the device-side graph loop of
// solver.cu for Wilson (8^4 FP64: 506 against 482 solves/s) and is the default
// there.  It does not suit DWF, whose columns of slices share each link (DWF
// 8^4 x Ls 16 with this form: 39 against 10.4 ms per solve).  Larger fields run
// the column hop of hop_kernel plus a p-update phase (five barriers), which is
// slower than the graph loop (DWF 8^4 x Ls 16: 11.3 against 10.3 ms per solve);
// both run for DWF and for larger fields only when asked for.
//
// Grid barriers spin on a generation counter with a time limit: a wait that
// runs out sets the error flag, every other block leaves at its next wait, and
// the host reports the error.  The cooperative launch keeps all blocks
// resident, so the barriers complete in normal operation.
#include <string.h>

#include "host.h"
#include "hop.cuh"

namespace cpsb {

// Threads per block: 128, or 32 for single-slice columns (Wilson), so that a
// unit is 32 columns whose link table fits shared memory and a small lattice
// still spreads over many SMs.
constexpr int PCG_NT_MAX = 128;
// Fields (all right-hand sides) of at most this many entries use the
// direction-parallel hop phases (the same bound as the automatic mode).
constexpr long PCG_DP_SITES = PCG_AUTO_SITES;
// Longest barrier wait before it gives up (ns of the global timer): far above a
// phase of any lattice the loop takes, and above kernels of other streams that
// may hold SMs while the launch's blocks become resident.
constexpr unsigned long long PCG_WAIT_NS = 5000000000ull;

__device__ __forceinline__ unsigned long long pcg_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct PcgArgs {
  // the four hops of one iteration (in, out, x, cb, dag, a set per phase):
  // [0] t1 = D p, [1] t2 = p - kappa^2 D t1 with |t2|^2, [2] t1 = D^dag t2,
  // [3] A p = t2 - kappa^2 D^dag t1 consumed by the residual update
  DslashArgs ph[4];
  SpinorPtr r, p, x;
  CgState *S;
  double *partial;  // [nrhs][gridDim.x] block partials
  unsigned *bar;    // [0] arrivals, [1] generation
  int *err;         // set when a barrier wait ran out
};

// Grid barrier with a bounded wait; false (in every thread) when this block's
// wait ran out or another block has already reported one.
__device__ __forceinline__ bool pcg_sync(const PcgArgs &P) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = P.bar + 1;
    volatile int *err = P.err;
    const unsigned g0 = *gen;
    __threadfence();
    ok = 1;
    if (atomicAdd(P.bar, 1u) == gridDim.x - 1) {
      atomicExch(P.bar, 0u);
      __threadfence();
      atomicAdd(P.bar + 1, 1u);
    } else {
      const unsigned long long t0 = pcg_now();
      while (*gen == g0) {
        if (*err || pcg_now() - t0 > PCG_WAIT_NS) {
          atomicExch(P.err, 1);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// One hop over every unit of the lattice (the FP64 branch of hop_kernel with one
// right-hand side per thread at a time).  MODE 0: out = D in; 1: out = x + a D in
// with |out|^2 into nrm; 2: A p = x + a D in, then r -= alpha A p, x_sol += alpha p
// and |r|^2 into nrm.
template <int NT, bool LC, bool DAG, int MODE>
__device__ __forceinline__ void pcg_hop(const DslashArgs &A, const PcgArgs &P, unsigned char *dsh, double *nrm,
                                        const int *skip, const double *alpha) {
  const Geom &g = A.g;
  const int C0 = g.cs[0];
  const int TX = NT / C0;
  const HopShm L = hop_shm(TX, NT, g.nrhs, true, LC);
  const int sp = threadIdx.x % C0;
  const int xl = threadIdx.x / C0;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int nunits = ntiles * g.ncls;
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    const int k = unit % g.ncls, tile = unit / g.ncls;
    const int par_out = A.five_d ? ((1 - A.cb + k) & 1) : 1 - A.cb;
    __syncthreads();  // the previous unit is done with the tables
    load_unit<P64, LC>(A, tile, k, par_out, TX, NT, dsh);
    __syncthreads();
    const int xs = tile * TX + xl;
    const int C = g.cs[k];
    if (xl >= TX || xs >= g.n4cb || sp >= C) continue;
    HopCtx hc;
    entry_ctx<P64, LC>(hc, A, dsh, L, xl, xs, k, sp, par_out);
    const unsigned own = (k ? (unsigned)g.kb1 : 0u) + (unsigned)xs * (unsigned)C + (unsigned)sp;
    for (int q = 0; q < g.nrhs; q++) {
      if (skip[q]) continue;
      const unsigned rb = (unsigned)q * per;
      const unsigned i = rb + own;
      Spinor<double> acc = hop_entry_64<P64, LC, DAG, 1, true>(A, hc, rb);
      if (MODE == 0) {
        store_spinor<P64>(A.out, i, acc);
        continue;
      }
      const double a = A.a;
      const Spinor<double> xv = unpack64(load_raw64_l2(A.x, i));
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = xv.c[s2][r] + cscale(a, acc.c[s2][r]);
      if (MODE == 1) {
        store_spinor<P64>(A.out, i, acc);
        nrm[q * NT + threadIdx.x] += norm2(acc);
        continue;
      }
      const double al = alpha[q];
      Spinor<double> rv = unpack64(load_raw64_l2(P.r, i));
      const Spinor<double> pv = unpack64(load_raw64_l2(P.p, i));
      Spinor<double> sv = unpack64(load_raw64_l2(P.x, i));
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) sv.c[s2][r] = cscale(al, pv.c[s2][r]) + sv.c[s2][r];
      store_spinor<P64>(P.x, i, sv);
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) rv.c[s2][r] = rv.c[s2][r] - cscale(al, acc.c[s2][r]);
      store_spinor<P64>(P.r, i, rv);
      nrm[q * NT + threadIdx.x] += norm2(rv);
    }
  }
}

// The same phase with eight lanes per entry (hop8_kernel of hop.cuh): lane d
// loads neighbour d and its link, lanes 0 and 1 the 5th-direction terms, lane
// 0 sums the partial spinors in direction order through the shared-memory
// slots gsh (12 x NT double2) and runs the epilogue; all loads through L2.
// PUPD folds the direction update p = r + beta p of the previous iteration in:
// MODE 0 forms each neighbour's r + beta p from r and the old p as it loads
// them, and MODE 1 forms its own entry's, stores it as the new p and uses it as
// the xpay input (one fused multiply-add per real in both, so the two agree).
__device__ __forceinline__ Raw<P64> p_next(const Raw<P64> &r, const Raw<P64> &p, double b) {
  Raw<P64> o;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k] = make_double2(__fma_rn(b, p.c[k].x, r.c[k].x), __fma_rn(b, p.c[k].y, r.c[k].y));
  return o;
}

template <int NT, bool DAG, int MODE, bool PUPD>
__device__ __forceinline__ void pcg8_hop(const DslashArgs &A, const PcgArgs &P, double2 *gsh, double *nrm,
                                         const int *skip, const double *alpha, const double *beta) {
  const Geom &g = A.g;
  constexpr double sdag = DAG ? -1.0 : 1.0;
  const int d = threadIdx.x & 7;
  const int lane = threadIdx.x & 31;
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  const long wstride = (long)gridDim.x * (NT / 32) * 4;
  for (int q = 0; q < g.nrhs; q++) {
    if (skip[q]) continue;
    for (long e0 = ((long)blockIdx.x * (NT / 32) + threadIdx.x / 32) * 4; e0 < (long)per; e0 += wstride) {
      const long e = e0 + (lane >> 3);
      const bool valid = e < (long)per;
      Spinor<double> acc;
      zero(acc);
      double2 v5[6];
#pragma unroll
      for (int qq = 0; qq < 6; qq++) v5[qq] = make_double2(0.0, 0.0);
      unsigned i = 0;
      double f5m = 0.0, f5p = 0.0;
      if (valid) {
        const unsigned own = (unsigned)e;
        const int k = (g.ncls == 2 && own >= (unsigned)g.kb1) ? 1 : 0;
        const int C = g.cs[k];
        const unsigned rem = own - (k ? (unsigned)g.kb1 : 0u);
        const int x = (int)(rem / (unsigned)C);
        const int sp = (int)(rem - (unsigned)x * (unsigned)C);
        const int s = g.ncls == 2 ? k + 2 * sp : sp;
        const int par_out = A.five_d ? ((1 - A.cb + k) & 1) : 1 - A.cb;
        const unsigned rb = (unsigned)q * per;
        i = rb + own;
        const int mu = d & 3;
        const double sg = d < 4 ? -sdag : sdag;
        Coord c = decode(g, x, par_out);
        auto step = [&](int v, int n) { return d < 4 ? (v + 1 == n ? 0 : v + 1) : (v == 0 ? n - 1 : v - 1); };
        switch (mu) {
          case 0: c.x = step(c.x, g.lx); break;
          case 1: c.y = step(c.y, g.ly); break;
          case 2: c.z = step(c.z, g.lz); break;
          default: c.t = step(c.t, g.lt); break;
        }
        const int xn = cbindex(g, c.x, c.y, c.z, c.t);
        const unsigned ni = rb + (k ? (unsigned)g.kb1 : 0u) + (unsigned)xn * (unsigned)C + (unsigned)sp;
        Raw<P64> nr = load_raw64_l2(A.in, ni);
        if (PUPD && MODE == 0) nr = p_next(load_raw64_l2(P.r, ni), nr, beta[q]);
        if (A.hop5 && d < 2) {
          const int sn = d == 0 ? (s == 0 ? g.ls - 1 : s - 1) : (s == g.ls - 1 ? 0 : s + 1);
          const int chunk0 = (d == 0) != DAG ? 0 : 6;
          const unsigned i5 = rb + site_entry(g, sn, x);
          const double2 *b = entry_ptr<12, const double2>(A.in.data, i5);
          if (PUPD && MODE == 0) {
            const double2 *br = entry_ptr<12, const double2>(P.r.data, i5);
#pragma unroll
            for (int qq = 0; qq < 6; qq++) {
              const double2 pv = __ldcg(b + 8 * (chunk0 + qq)), rv = __ldcg(br + 8 * (chunk0 + qq));
              v5[qq] = make_double2(__fma_rn(beta[q], pv.x, rv.x), __fma_rn(beta[q], pv.y, rv.y));
            }
          } else {
#pragma unroll
            for (int qq = 0; qq < 6; qq++) v5[qq] = __ldcg(b + 8 * (chunk0 + qq));
          }
          f5m = s == 0 ? A.hop5_wall : A.hop5_fact;
          f5p = s == g.ls - 1 ? A.hop5_wall : A.hop5_fact;
        }
        const Link<double> l = d < 4 ? load_link<P64>(A.U, par_out, mu, x) : load_link<P64>(A.U, 1 - par_out, mu, xn);
        const Half<double> h = project(unpack64(nr), mu, sg);
        switch (mu) {
          case 0: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 0, sg); break;
          case 1: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 1, sg); break;
          case 2: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 2, sg); break;
          default: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 3, sg); break;
        }
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int r = 0; r < 3; r++) gsh[(3 * a + r) * NT + threadIdx.x] = make_double2(acc.c[a][r].re, acc.c[a][r].im);
      __syncwarp();
      if (d == 0) {
#pragma unroll
        for (int j = 1; j < 8; j++)
#pragma unroll
          for (int a = 0; a < 4; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
              const double2 v = gsh[(3 * a + r) * NT + threadIdx.x + j];
              acc.c[a][r] = acc.c[a][r] + mk(v.x, v.y);
            }
      }
      __syncwarp();
      const int base = lane & ~7;
      double2 vp[6];
#pragma unroll
      for (int qq = 0; qq < 6; qq++)
        vp[qq] = make_double2(__shfl_sync(0xffffffffu, v5[qq].x, base + 1), __shfl_sync(0xffffffffu, v5[qq].y, base + 1));
      if (!valid || d != 0) continue;
      if (A.hop5) {
#pragma unroll
        for (int qq = 0; qq < 6; qq++) {
          const cplx<double> lo = cscale(f5m, mk(v5[qq].x, v5[qq].y)), hi = cscale(f5p, mk(vp[qq].x, vp[qq].y));
          cplx<double> &u = acc.c[qq / 3][qq % 3], &w = acc.c[2 + qq / 3][qq % 3];
          if (!DAG) {
            u = u + lo;
            w = w + hi;
          } else {
            w = w + lo;
            u = u + hi;
          }
        }
      }
      if (MODE == 0) {
        store_spinor<P64>(A.out, i, acc);
        continue;
      }
      const double a = A.a;
      Spinor<double> xv;
      if (PUPD && MODE == 1) {
        // the new direction p = r + beta p at this entry: stored, and the xpay input
        xv = unpack64(p_next(load_raw64_l2(P.r, i), load_raw64_l2(A.x, i), beta[q]));
        store_spinor<P64>(A.x, i, xv);
      } else {
        xv = unpack64(load_raw64_l2(A.x, i));
      }
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = xv.c[s2][r] + cscale(a, acc.c[s2][r]);
      if (MODE == 1) {
        store_spinor<P64>(A.out, i, acc);
        nrm[q * NT + threadIdx.x] += norm2(acc);
        continue;
      }
      const double al = alpha[q];
      Spinor<double> rv = unpack64(load_raw64_l2(P.r, i));
      const Spinor<double> pv = unpack64(load_raw64_l2(P.p, i));
      Spinor<double> sv = unpack64(load_raw64_l2(P.x, i));
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) sv.c[s2][r] = cscale(al, pv.c[s2][r]) + sv.c[s2][r];
      store_spinor<P64>(P.x, i, sv);
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) rv.c[s2][r] = rv.c[s2][r] - cscale(al, acc.c[s2][r]);
      store_spinor<P64>(P.r, i, rv);
      nrm[q * NT + threadIdx.x] += norm2(rv);
    }
  }
}

// Per-right-hand-side sums of nrm over the grid, left in out[] of every block
// (the block partials summed in block order, the same order in every block).
template <int NT>
__device__ __forceinline__ bool pcg_reduce(const PcgArgs &P, int nrhs, double *nrm, double *red, double *out) {
  for (int q = 0; q < nrhs; q++) {
    const double bs = block_sum<NT>(nrm[q * NT + threadIdx.x], red);
    nrm[q * NT + threadIdx.x] = 0;
    if (threadIdx.x == 0) P.partial[q * gridDim.x + blockIdx.x] = bs;
  }
  if (!pcg_sync(P)) return false;
  for (int q = 0; q < nrhs; q++) {
    const double t = ordered_sum<NT>(P.partial + q * gridDim.x, gridDim.x, red);
    if (threadIdx.x == 0) out[q] = t;
    __syncthreads();
  }
  return true;
}

// DP: the hop phases with eight lanes per entry (pcg8_hop), for the smallest lattices.
template <int NT, bool LC, bool DP>
__global__ void __launch_bounds__(NT, 1) pcg_kernel(PcgArgs P) {
  extern __shared__ __align__(16) unsigned char dsh[];
  __shared__ CgState S;
  __shared__ double red[NT / 32];
  __shared__ double sums[MAX_RHS], alpha[MAX_RHS], beta[MAX_RHS];
  __shared__ int skip[MAX_RHS];
  const Geom &g = P.ph[0].g;
  const int nrhs = g.nrhs;
  const int C0 = g.cs[0];
  const HopShm L = hop_shm(NT / C0, NT, nrhs, true, LC);
  double2 *gsh = (double2 *)dsh;  // DP: 12 x NT partial-spinor slots
  double *nrm = (double *)(dsh + (DP ? (size_t)12 * NT * sizeof(double2) : L.norm));
  if (threadIdx.x == 0) S = *P.S;
  for (int q = 0; q < nrhs; q++) nrm[q * NT + threadIdx.x] = 0;
  __syncthreads();
  const long per = (long)g.n4cb * g.ls;
  for (int guard = 0; guard <= S.max_iter + 1; guard++) {
    bool all = true;
    for (int q = 0; q < nrhs; q++) all = all && S.halt_done[q];
    if (all) break;
    if (threadIdx.x < nrhs) {
      skip[threadIdx.x] = S.halt[threadIdx.x];
      // DP: the direction update of the previous iteration rides on this one's
      // first two hops (p = r on entry: beta 0 in the first iteration)
      beta[threadIdx.x] = guard == 0 ? 0.0 : S.beta[threadIdx.x];
    }
    __syncthreads();
    // t1 = D p
    if constexpr (DP) pcg8_hop<NT, false, 0, true>(P.ph[0], P, gsh, nrm, skip, alpha, beta);
    else pcg_hop<NT, LC, false, 0>(P.ph[0], P, dsh, nrm, skip, alpha);
    if (!pcg_sync(P)) break;
    // t2 = MatPc p, d = |t2|^2
    if constexpr (DP) pcg8_hop<NT, false, 1, true>(P.ph[1], P, gsh, nrm, skip, alpha, beta);
    else pcg_hop<NT, LC, false, 1>(P.ph[1], P, dsh, nrm, skip, alpha);
    if (!pcg_reduce<NT>(P, nrhs, nrm, red, sums)) break;
    if (threadIdx.x < nrhs && !skip[threadIdx.x]) S.d[threadIdx.x] = sums[threadIdx.x];
    __syncthreads();
    // t1 = D^dag t2
    if constexpr (DP) pcg8_hop<NT, true, 0, false>(P.ph[2], P, gsh, nrm, skip, alpha, beta);
    else pcg_hop<NT, LC, true, 0>(P.ph[2], P, dsh, nrm, skip, alpha);
    if (!pcg_sync(P)) break;
    // A p = MatPcDag t2: r -= alpha A p, x += alpha p, |r|^2
    if (threadIdx.x < nrhs) {
      const int q = threadIdx.x;
      alpha[q] = S.rr[q] / (S.d[q] + S.shift * S.pp[q]);
    }
    __syncthreads();
    if constexpr (DP) pcg8_hop<NT, true, 2, false>(P.ph[3], P, gsh, nrm, skip, alpha, beta);
    else pcg_hop<NT, LC, true, 2>(P.ph[3], P, dsh, nrm, skip, alpha);
    if (!pcg_reduce<NT>(P, nrhs, nrm, red, sums)) break;
    if (threadIdx.x == 0)
      for (int q = 0; q < nrhs; q++)
        if (!skip[q]) cg_advance(&S, q, sums[q]);
    __syncthreads();
    if constexpr (DP) {
      // p is updated by the next iteration's first two hops; a right-hand side
      // that halted here is skipped from then on
      if (threadIdx.x == 0)
        for (int q = 0; q < nrhs; q++) S.halt_done[q] = S.halt[q];
      __syncthreads();
      continue;
    }
    // p = r + beta p for the right-hand sides still iterating (cg_xp_update, blas.cu)
    for (int q = 0; q < nrhs; q++) {
      if (S.halt_done[q] || S.halt[q]) continue;
      const double b = S.beta[q];
      for (long j = (long)blockIdx.x * NT + threadIdx.x; j < per; j += (long)gridDim.x * NT) {
        const unsigned i = (unsigned)(q * per + j);
        Spinor<double> pv = unpack64(load_raw64_l2(P.p, i));
        const Spinor<double> rv = unpack64(load_raw64_l2(P.r, i));
#pragma unroll
        for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
          for (int r = 0; r < 3; r++) pv.c[s2][r] = cscale(b, pv.c[s2][r]) + rv.c[s2][r];
        store_spinor<P64>(P.p, i, pv);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int q = 0; q < nrhs; q++) S.halt_done[q] = S.halt[q];
    if (!pcg_sync(P)) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *P.S = S;
}

// Largest grid of a persistent solve on this device: all blocks resident.
static int pcg_max_blocks(const void *fn, int nt, size_t shm) {
  int dev = 0, nsm = 0, per_sm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, shm) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nsm * per_sm;
}

int persistent_cg_mode() {
  const char *e = getenv("CPSB_PERSISTENT_CG");
  return e ? atoi(e) : 1;
}

// Runs the iterations of an FP64 CG solve whose state (r, p, x, CgState) the
// caller has set up.  Returns cudaErrorNotSupported, launching nothing, where
// the persistent form does not apply (the caller then runs its own loop).
cudaError_t launch_persistent_cg(const DslashArgs &base, double mkappa2, SpinorPtr t1, SpinorPtr t2, SpinorPtr r,
                                 SpinorPtr p, SpinorPtr x, CgState *S, double *partial, size_t partial_slots,
                                 unsigned *bar_err, cudaStream_t st) {
  const Geom &g = base.g;
  const int C0 = g.cs[0];
  if (C0 < 1 || C0 > PCG_NT_MAX) return cudaErrorNotSupported;
  const long per = (long)g.n4cb * g.ls;
  // eight lanes per entry where even that leaves blocks for every SM to spare
  const bool dp = per * g.nrhs <= PCG_DP_SITES;
  const int nt = dp ? PCG_NT_MAX : C0 == 1 ? 32 : PCG_NT_MAX;
  const int TX = nt / C0;
  const bool lc = TX <= 32;
  const size_t shm = dp ? (size_t)12 * nt * sizeof(double2) + (size_t)nt * g.nrhs * sizeof(double)
                        : hop_shm(TX, nt, g.nrhs, true, lc).total;
  if (shm > 48 * 1024) return cudaErrorNotSupported;
  const void *fn = dp ? (const void *)pcg_kernel<PCG_NT_MAX, false, true>
                      : nt == 32 ? (const void *)pcg_kernel<32, true, false>
                      : lc ? (const void *)pcg_kernel<PCG_NT_MAX, true, false>
                           : (const void *)pcg_kernel<PCG_NT_MAX, false, false>;
  const long units = dp ? (per + nt / 8 - 1) / (nt / 8) : (long)((g.n4cb + TX - 1) / TX) * g.ncls;
  const int grid = (int)std::min(units, (long)pcg_max_blocks(fn, nt, shm));
  if (grid < 1 || (size_t)grid * g.nrhs > partial_slots) return cudaErrorNotSupported;
  PcgArgs P;
  memset(&P, 0, sizeof(P));
  for (int k = 0; k < 4; k++) {
    P.ph[k] = base;
    P.ph[k].rg = 1;
    P.ph[k].rgroup = g.nrhs;
    P.ph[k].torder = 0;
    P.ph[k].skip = nullptr;
    memset(&P.ph[k].red, 0, sizeof(Reduce));
    P.ph[k].cg = nullptr;
  }
  P.ph[0].in = p, P.ph[0].out = t1, P.ph[0].cb = 1, P.ph[0].dag = 0, P.ph[0].a = 1.0;
  P.ph[1].in = t1, P.ph[1].out = t2, P.ph[1].x = p, P.ph[1].cb = 0, P.ph[1].dag = 0, P.ph[1].a = mkappa2;
  P.ph[2].in = t2, P.ph[2].out = t1, P.ph[2].cb = 1, P.ph[2].dag = 1, P.ph[2].a = 1.0;
  P.ph[3].in = t1, P.ph[3].x = t2, P.ph[3].cb = 0, P.ph[3].dag = 1, P.ph[3].a = mkappa2;
  P.r = r;
  P.p = p;
  P.x = x;
  P.S = S;
  P.partial = partial;
  P.bar = bar_err;
  P.err = (int *)(bar_err + 2);
  cudaError_t e = cudaMemsetAsync(bar_err, 0, 4 * sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  void *args[] = {&P};
  e = cudaLaunchCooperativeKernel(fn, dim3((unsigned)grid), dim3(nt), args, shm, st);
  count_launch();
  return e;
}

}  // namespace cpsb

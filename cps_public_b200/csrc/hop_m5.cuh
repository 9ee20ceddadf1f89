// hop_m5.cuh -- the Mobius 4-D hop with the M5 column operations of its output
// fused in: one pass over memory where the operator otherwise runs the hop,
// stores its output, and reads it back in a separate M5 kernel.
//
//   dag 0:  out = a * mix(M5^-1 (D in))                  (zmobius_m-sym2.h: the
//           M5^-1 that follows the first kappa_b D4 of MatPc, dag 0)
//   dag 1:  out = [x +] a * M5^-dag(mix^dag(D^dag in))  [, |out|^2]
//           (zmobius_mdag-sym2.h: the M5^-dag after each D4^dag of MatPcDag)
//
// With 4-D checkerboarding (DWF_4D_EOPREC_EE) every slice of a site has the
// same parity, so the column of a site holds all Ls slices and the block that
// computes a tile's hop owns whole columns: the Ls hop outputs of a column are
// written to a shared-memory tile, one thread per (column, complex component)
// runs the sweeps of m5_sweep.cuh over its Ls values in registers, and every
// thread reads its own entry back for the epilogue and the store.  The hop
// itself is hop.cuh's (links of the unit in shared memory, neighbour tables).
#pragma once
#include "hop.cuh"
#include "m5_sweep.cuh"

namespace cpsb {

// Element of the sweep tile: one complex component in the arithmetic type.
template <int P> struct SweepT { typedef float2 T; typedef float R; };
template <> struct SweepT<P64> { typedef double2 T; typedef double R; };

// Dynamic shared memory: hop.cuh's tables, then the sweep tile of TX columns
// x 12 components x (LS + 1) slots (the pad spreads the columns that one warp
// sweeps over the banks).
template <int P, int LS>
__host__ __device__ inline size_t hop_m5_tile_off(int TX, int NT, int nrhs, bool norm) {
  return (hop_shm(TX, NT, nrhs, norm, true).total + 15) & ~(size_t)15;
}
template <int P, int LS>
__host__ __device__ inline size_t hop_m5_shm(int TX, int NT, int nrhs, bool norm) {
  return hop_m5_tile_off<P, LS>(TX, NT, nrhs, norm) + (size_t)TX * 12 * (LS + 1) * sizeof(typename SweepT<P>::T);
}

// Thread t owns slice t % LS of tile column t / LS for every right-hand side
// in turn; the skip mask is read per right-hand side, uniformly over the block,
// so every thread reaches every barrier.
template <int P, int NT, int MINB, bool DAG, bool XPAY, bool NORM, int LS, int DEPTH>
__global__ void __launch_bounds__(NT, MINB) hop_m5_kernel(DslashArgs A, M5Coef cf) {
  typedef typename SweepT<P>::T BT;
  typedef typename SweepT<P>::R R;
  constexpr int TX = NT / LS;
  constexpr int CST = LS + 1;
  const Geom &g = A.g;
  extern __shared__ __align__(16) unsigned char dsh[];
  __shared__ double red[NT / 32];
  const HopShm L = hop_shm(TX, NT, g.nrhs, NORM, true);
  BT *tile_buf = (BT *)(dsh + hop_m5_tile_off<P, LS>(TX, NT, g.nrhs, NORM));
  double *nrm_sh = (double *)(dsh + L.norm);
  if (NORM)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const int sp = threadIdx.x % LS;
  const int xl = threadIdx.x / LS;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const unsigned per = (unsigned)g.n4cb * (unsigned)LS;
  const int par_out = 1 - A.cb;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    __syncthreads();  // the previous tile is done with the tables and the sweep tile
    load_unit<P, true>(A, tile, 0, par_out, TX, NT, dsh);
    __syncthreads();
    const int x = tile * TX + xl;
    const bool act = xl < TX && x < g.n4cb;
    const int nx = min(TX, g.n4cb - tile * TX);
    HopCtx hc;
    if (act) entry_ctx<P, true>(hc, A, dsh, L, xl, x, 0, sp, par_out);
    const unsigned own = (unsigned)x * (unsigned)LS + (unsigned)sp;
    BT *mine = tile_buf + (size_t)xl * 12 * CST + sp;  // component q of this entry at mine[q * CST]
    for (int rhs = 0; rhs < g.nrhs; rhs++) {
      if (A.skip && A.skip[rhs]) continue;
      const unsigned rb = (unsigned)rhs * per;
      const unsigned i = rb + own;
      // 1. the hop of this thread's entry into the sweep tile (FP64: component
      // q = 3 spin + colour as (re, im); FP32 / 16-bit: q = 2 (3 p + colour) +
      // (0 re, 1 im) as the lanes (spin 2p, spin 2p + 1))
      if (act) {
        if constexpr (P == P64) {
          const Spinor<double> o = hop_entry_64<P, true, DAG, DEPTH>(A, hc, rb);
#pragma unroll
          for (int q = 0; q < 12; q++) mine[q * CST] = make_double2(o.c[q / 3][q % 3].re, o.c[q / 3][q % 3].im);
        } else {
          const SpX2 o = hop_entry_x2<P, true, DAG, DEPTH>(A, hc, rb);
#pragma unroll
          for (int q = 0; q < 6; q++) {
            mine[(2 * q) * CST] = o.re[q / 3][q % 3];
            mine[(2 * q + 1) * CST] = o.im[q / 3][q % 3];
          }
        }
      }
      __syncthreads();
      // 2. the column operations, one thread per (column, component); the
      // upper chirality (spins 0, 1) is q < 6 in both layouts.  Real
      // coefficients act alike on the two members of a pair.
      for (int t = threadIdx.x; t < nx * 12; t += NT) {
        const int cx = t / 12, q = t - cx * 12;
        BT *col = tile_buf + (size_t)(cx * 12 + q) * CST;
        cplx<R> v[LS][1];
#pragma unroll
        for (int s = 0; s < LS; s++) v[s][0] = mk(col[s].x, col[s].y);
        m5_column<LS, DAG ? 1 : 0, 1, R>(v, q < 6, cf);
#pragma unroll
        for (int s = 0; s < LS; s++) {
          col[s].x = v[s][0].re;
          col[s].y = v[s][0].im;
        }
      }
      __syncthreads();
      // 3. epilogue: out = [x +] a v
      if (act) {
        if constexpr (P == P64) {
          Spinor<double> o;
#pragma unroll
          for (int q = 0; q < 12; q++) {
            const double2 v = mine[q * CST];
            o.c[q / 3][q % 3] = mk(A.a * v.x, A.a * v.y);
          }
          if (XPAY) {
            const Spinor<double> xv = unpack64(load_raw<P64>(A.x, i));
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
              for (int r = 0; r < 3; r++) o.c[s2][r] = xv.c[s2][r] + o.c[s2][r];
          }
          store_spinor<P64>(A.out, i, o);
          if (NORM) nrm_sh[rhs * NT + threadIdx.x] += norm2(o);
        } else {
          const float2 a2 = f2b((float)A.a);
          SpX2 o;
#pragma unroll
          for (int q = 0; q < 6; q++) {
            o.re[q / 3][q % 3] = mul2(a2, mine[(2 * q) * CST]);
            o.im[q / 3][q % 3] = mul2(a2, mine[(2 * q + 1) * CST]);
          }
          if (XPAY) {
            float xn;
            const SpX2 xv = unpack(load_raw<P>(A.x, i), &xn);
            const float2 xs = f2b(xn);
#pragma unroll
            for (int p = 0; p < 2; p++)
#pragma unroll
              for (int cc = 0; cc < 3; cc++) {
                o.re[p][cc] = fma2(xv.re[p][cc], xs, o.re[p][cc]);
                o.im[p][cc] = fma2(xv.im[p][cc], xs, o.im[p][cc]);
              }
          }
          const double n2 = store_x2<P>(A.out, i, o);
          if (NORM) nrm_sh[rhs * NT + threadIdx.x] += n2;
        }
      }
      __syncthreads();  // every entry is read back before the next right-hand side's hop
    }
  }
  if (NORM) {
    for (int q = 0; q < g.nrhs; q++) {
      const double bs = block_sum<NT>(nrm_sh[q * NT + threadIdx.x], red);
      if (threadIdx.x == 0) A.red.partial[q * gridDim.x + blockIdx.x] = bs;
    }
    if (last_block(A.red.ticket, gridDim.x)) {
      for (int q = 0; q < g.nrhs; q++) {
        const double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) A.red.result[q] = t;
        __syncthreads();
      }
    }
  }
}

template <int P, int LS, bool DAG, bool XPAY, bool NORM>
static cudaError_t hop_m5_launch_m(const DslashArgs &A, const M5Coef &cf, cudaStream_t st) {
  constexpr int NT = 128;
  constexpr int MINB = P == P64 ? 2 : 4;
  constexpr int DEPTH = P == P64 ? 1 : 2;
  constexpr int TX = NT / LS;
  const size_t shm = hop_m5_shm<P, LS>(TX, NT, A.g.nrhs, NORM);
  if (shm > 200 * 1024) return cudaErrorNotSupported;
  const void *fn = (const void *)hop_m5_kernel<P, NT, MINB, DAG, XPAY, NORM, LS, DEPTH>;
  static bool opted = false;
  if (!opted && shm + 1024 > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  const long ntiles = (A.g.n4cb + TX - 1) / TX;
  const long nb = std::min(ntiles, (long)resident_blocks(fn, NT, shm));
  hop_m5_kernel<P, NT, MINB, DAG, XPAY, NORM, LS, DEPTH><<<(unsigned)nb, NT, shm, st>>>(A, cf);
  return launched();
}

template <int P, int LS>
static cudaError_t hop_m5_launch_ls(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st) {
  if (!A.dag) {
    if (xpay || norm) return cudaErrorNotSupported;
    return hop_m5_launch_m<P, LS, false, false, false>(A, cf, st);
  }
  if (xpay && norm) return hop_m5_launch_m<P, LS, true, true, true>(A, cf, st);
  if (xpay) return hop_m5_launch_m<P, LS, true, true, false>(A, cf, st);
  if (norm) return cudaErrorNotSupported;
  return hop_m5_launch_m<P, LS, true, false, false>(A, cf, st);
}

// The fused hop + M5 for one storage precision; cudaErrorNotSupported for a
// shape without a fused form (5-D checkerboarding, the 5th-direction hop, an
// Ls not listed), for which the caller runs the hop and the M5 kernel.
template <int P>
static cudaError_t hop_m5_launch_p(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st) {
  if (A.five_d || A.hop5 || A.g.ncls != 1 || A.g.cs[0] != A.g.ls || A.cg) return cudaErrorNotSupported;
  switch (A.g.ls) {
    case 4: return hop_m5_launch_ls<P, 4>(A, cf, xpay, norm, st);
    case 8: return hop_m5_launch_ls<P, 8>(A, cf, xpay, norm, st);
    case 12: return hop_m5_launch_ls<P, 12>(A, cf, xpay, norm, st);
    case 16: return hop_m5_launch_ls<P, 16>(A, cf, xpay, norm, st);
    case 20: return hop_m5_launch_ls<P, 20>(A, cf, xpay, norm, st);
    case 24: return hop_m5_launch_ls<P, 24>(A, cf, xpay, norm, st);
    case 32: return hop_m5_launch_ls<P, 32>(A, cf, xpay, norm, st);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace cpsb

// m5.cu -- Mobius fifth-direction kernels: exact M5^-1 fused with the b/c
// mixing of the 4-D hop.
//
// Restates, for real Mobius coefficients, zmobius_m5inv (cps_pp/src/util/
// dirac_op/d_op_zmobius/noarch/zmobius_m5inv.C:247-400 dag 0, :534-686 dag 1):
// a forward and a backward sweep along s per 4-D site and chirality with the
// domain-wall wall correction, and the mixing  b*psi_s + c*(P+ psi_{s-1} +
// P- psi_{s+1})  with -m_f walls of zmobius_kappa_dslash_5_plus_cmplx
// (zmobius_dslash_5_plus.C:125-376); and the zMobius form with complex
// per-slice coefficients from a table.  The sweeps are independent for every
// complex spinor component.
//
//   dag 0:  out = scale * mix(M5^-1 in)                 (precedes D_W in MatPc)
//   dag 1:  out = [x +] scale * M5^-dag(mix^dag(in))    (follows D_W^dag in MatPcDag)
//
// In the column layout (cpsb_device.cuh) the Ls slices of a 4-D site are
// consecutive entries, so a block moves a tile of whole columns between HBM
// and shared memory with coalesced 16-byte accesses (one entry per thread),
// and the sweeps run from shared memory, one thread per (site, storage chunk)
// with the column of Ls values in registers: every value is read from HBM and
// written once.  16-bit storage is decoded on the way in and encoded per site
// (its quantum is the site's maximum) on the way out; the sweep arithmetic is
// FP32.
#include <string.h>

#include "blas.h"
#include "m5_sweep.cuh"

namespace cpsb {

// Per storage precision: the real type of the sweeps, the complex values a
// chunk holds (NC) and the chunks of a site (NCH).  FP64 chunk k is component
// (spin k/3, colour k%3); FP32 / 16-bit chunk k = 3p + c holds colour c of the
// spins 2p and 2p+1.  Chunks k < NCH/2 are the upper chirality (spins 0, 1).
template <int P> struct ChunkT;
template <> struct ChunkT<P64> { static const int NCH = 12, NC = 1; typedef double T; };
template <> struct ChunkT<P32> { static const int NCH = 6, NC = 2; typedef float T; };
template <> struct ChunkT<P16> { static const int NCH = 6, NC = 2; typedef float T; };

template <int NC, typename T>
__device__ __forceinline__ cplx<T> &chunk_elem(Spinor<T> &s, int k, int q) {
  return NC == 1 ? s.c[k / 3][k % 3] : s.c[2 * (k / 3) + q][k % 3];
}

// Per-RHS |out|^2 of the block into red (deterministic: partials summed in
// block order by the last block).
template <int NT>
__device__ __forceinline__ void m5_norm_epilogue(double acc, const Geom &g, Reduce red, const int *skip, double *sh) {
  const int rhs = blockIdx.y;
  double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) red.partial[rhs * gridDim.x + blockIdx.x] = bs;
  if (last_block(red.ticket, gridDim.x * gridDim.y)) {
    for (int q = 0; q < g.nrhs; q++) {
      double t = ordered_sum<NT>(red.partial + q * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0 && !(skip && skip[q])) red.result[q] = t;
      __syncthreads();
    }
  }
}

// ----------------------------------------------------------------- zMobius
template <typename T> __device__ __forceinline__ cplx<T> ldz(const double2 *p) {
  const double2 v = __ldg(p);
  return mk((T)v.x, (T)v.y);
}
#define ZAXPYC(dst, f, src)                                  \
  _Pragma("unroll") for (int q = 0; q < NC; q++) (dst)[q] = (dst)[q] + cmul((f), (src)[q]);
#define ZSCALC(dst, f)                                       \
  _Pragma("unroll") for (int q = 0; q < NC; q++) (dst)[q] = cmul((f), (dst)[q]);

// v[s] <- bb_s v[s] + cc[h]_s v[s -+ 1] in place (cyclic: the wall terms
// are in cc), in the sweep order of mix_inplace.
template <int LS, int NC, typename T>
__device__ __forceinline__ void zmix_inplace(cplx<T> (&v)[LS][NC], bool from_below, int h, const ZM5Tab *tab) {
  cplx<T> wall[NC];
  if (from_below) {
#pragma unroll
    for (int q = 0; q < NC; q++) wall[q] = v[LS - 1][q];
#pragma unroll
    for (int s = LS - 1; s >= 1; s--) {
      const cplx<T> b = ldz<T>(&tab->bb[s]), c = ldz<T>(&tab->cc[h][s]);
#pragma unroll
      for (int q = 0; q < NC; q++) v[s][q] = cmul(b, v[s][q]) + cmul(c, v[s - 1][q]);
    }
    const cplx<T> b = ldz<T>(&tab->bb[0]), c = ldz<T>(&tab->cc[h][0]);
#pragma unroll
    for (int q = 0; q < NC; q++) v[0][q] = cmul(b, v[0][q]) + cmul(c, wall[q]);
  } else {
#pragma unroll
    for (int q = 0; q < NC; q++) wall[q] = v[0][q];
#pragma unroll
    for (int s = 0; s <= LS - 2; s++) {
      const cplx<T> b = ldz<T>(&tab->bb[s]), c = ldz<T>(&tab->cc[h][s]);
#pragma unroll
      for (int q = 0; q < NC; q++) v[s][q] = cmul(b, v[s][q]) + cmul(c, v[s + 1][q]);
    }
    const cplx<T> b = ldz<T>(&tab->bb[LS - 1]), c = ldz<T>(&tab->cc[h][LS - 1]);
#pragma unroll
    for (int q = 0; q < NC; q++) v[LS - 1][q] = cmul(b, v[LS - 1][q]) + cmul(c, wall[q]);
  }
}

// v <- post . mix(M5^-1(pre . v)) (DAG 0) or post . M5^-dag(mix^dag(pre . v))
// (DAG 1) on one column of chirality half h, in place, the stages the table
// enables.
template <int LS, int DAG, int NC, typename T>
__device__ __forceinline__ void m5z_column(cplx<T> (&v)[LS][NC], int h, const ZM5Tab *tab) {
  const int sweep = tab->sweep, mix = tab->mix, pre_on = tab->pre_on, post_on = tab->post_on;
  if (pre_on) {
#pragma unroll
    for (int s = 0; s < LS; s++) { ZSCALC(v[s], ldz<T>(&tab->pre[s])); }
  }
  // upper half at dag 0 and lower half at dag 1 take slice s-1, the others s+1
  const bool from_below = (DAG == 0) == (h == 0);
  if (DAG == 1 && mix) zmix_inplace<LS, NC, T>(v, from_below, h, tab);
  if (sweep) {
    if (tab->walls_first[h]) {
      ZSCALC(v[LS - 1], ldz<T>(&tab->invd[h]));
#pragma unroll
      for (int s = 0; s <= LS - 2; s++) { ZAXPYC(v[LS - 1], ldz<T>(&tab->w[h][s]), v[s]); }
#pragma unroll
      for (int s = LS - 2; s >= 0; s--) { ZAXPYC(v[s], ldz<T>(&tab->a[h][s]), v[s + 1]); }
    } else {
#pragma unroll
      for (int s = 0; s <= LS - 2; s++) { ZAXPYC(v[s + 1], ldz<T>(&tab->a[h][s]), v[s]); }
#pragma unroll
      for (int s = LS - 2; s >= 0; s--) { ZAXPYC(v[s], ldz<T>(&tab->w[h][s]), v[LS - 1]); }
      ZSCALC(v[LS - 1], ldz<T>(&tab->invd[h]));
    }
  }
  if (DAG == 0 && mix) zmix_inplace<LS, NC, T>(v, from_below, h, tab);
  if (post_on) {
#pragma unroll
    for (int s = 0; s < LS; s++) { ZSCALC(v[s], ldz<T>(&tab->post[s])); }
  }
}

// Sites per tile of the tiled kernels: one sweep thread per (site, chunk).
template <int P, int NT> struct M5Tile { static const int TX = NT / ChunkT<P>::NCH; };

// The tiled kernel: Z = false applies m5_column with the real coefficients cf,
// Z = true m5z_column with the table tab.  out = [x +] sc * v (sc = cf.scale
// for Z = false, 1 for Z = true).
template <int P, int LS, int DAG, bool XPAY, bool NORM, int NT, bool Z>
__global__ void __launch_bounds__(NT) m5t_kernel(Geom g, SpinorPtr out, SpinorPtr in, SpinorPtr xv, M5Coef cf,
                                                 const ZM5Tab *tab, Reduce red, const int *skip) {
  typedef typename ChunkT<P>::T T;
  constexpr int NCH = ChunkT<P>::NCH, NC = ChunkT<P>::NC, TX = M5Tile<P, NT>::TX;
  extern __shared__ __align__(16) unsigned char m5sh[];
  Spinor<T> *buf = (Spinor<T> *)m5sh;  // [TX * LS] entries of the tile
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * LS;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const T sc = Z ? T(1) : (T)cf.scale;
  double acc = 0;
  const bool sk = skip && skip[rhs];
  for (int tile = blockIdx.x; !sk && tile < ntiles; tile += gridDim.x) {
    const int nx = min(TX, g.n4cb - tile * TX);
    const long base = rhs * per + (long)tile * TX * LS;  // first entry of the tile
    __syncthreads();  // the previous tile's store phase is done with buf
    for (int t = threadIdx.x; t < nx * LS; t += NT) buf[t] = load_spinor<P>(in, base + t);
    __syncthreads();
    if (threadIdx.x < nx * NCH) {
      const int xl = threadIdx.x / NCH, k = threadIdx.x - xl * NCH;
      cplx<T> v[LS][NC];
#pragma unroll
      for (int s = 0; s < LS; s++)
#pragma unroll
        for (int q = 0; q < NC; q++) v[s][q] = chunk_elem<NC>(buf[xl * LS + s], k, q);
      if (Z) m5z_column<LS, DAG, NC, T>(v, k < NCH / 2 ? 0 : 1, tab);
      else m5_column<LS, DAG, NC, T>(v, k < NCH / 2, cf);
#pragma unroll
      for (int s = 0; s < LS; s++)
#pragma unroll
        for (int q = 0; q < NC; q++) chunk_elem<NC>(buf[xl * LS + s], k, q) = v[s][q];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nx * LS; t += NT) {
      Spinor<T> o = buf[t];
      if (XPAY) {
        const Spinor<T> xo = load_spinor<P>(xv, base + t);
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < 3; c++) o.c[a][c] = xo.c[a][c] + cscale(sc, o.c[a][c]);
      } else if (!Z) {
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < 3; c++) o.c[a][c] = cscale(sc, o.c[a][c]);
      }
      store_spinor<P>(out, base + t, o);
      if (NORM) acc += norm2(rounded<P>(o));
    }
  }
  if (NORM) m5_norm_epilogue<NT>(acc, g, red, skip, sh);
}

template <int P, int LS, bool Z>
static cudaError_t m5t_launch(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                              const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  constexpr int NT = 128;
  typedef typename ChunkT<P>::T T;
  constexpr int TX = M5Tile<P, NT>::TX;
  if (g.ncls != 1 || g.ls != LS) return cudaErrorInvalidValue;
  const size_t shm = sizeof(Spinor<T>) * TX * LS;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  dim3 grid(ntiles < 148 * 8 ? ntiles : 148 * 8, g.nrhs);
#define CPSB_M5T(D, XP, NR)                                                                            \
  if (dag == D && !!xpay == XP && !!norm == NR) {                                                      \
    static bool attr = false;                                                                          \
    if (!attr && shm > 48 * 1024) {                                                                    \
      const cudaError_t e = cudaFuncSetAttribute((const void *)m5t_kernel<P, LS, D, XP, NR, NT, Z>,    \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm); \
      if (e != cudaSuccess) return e;                                                                  \
      attr = true;                                                                                     \
    }                                                                                                  \
    m5t_kernel<P, LS, D, XP, NR, NT, Z><<<grid, NT, shm, st>>>(g, out, in, x, cf, tab, red, skip);     \
    return launched();                                                                                 \
  }
  CPSB_M5T(0, false, false) CPSB_M5T(0, true, false) CPSB_M5T(0, true, true) CPSB_M5T(0, false, true)
  CPSB_M5T(1, false, false) CPSB_M5T(1, true, false) CPSB_M5T(1, true, true) CPSB_M5T(1, false, true)
#undef CPSB_M5T
  return cudaErrorInvalidValue;
}

template <int P, bool Z>
static cudaError_t m5t_launch_p(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                                const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip,
                                cudaStream_t st) {
  switch (g.ls) {
    case 4: return m5t_launch<P, 4, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 8: return m5t_launch<P, 8, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 12: return m5t_launch<P, 12, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 16: return m5t_launch<P, 16, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 20: return m5t_launch<P, 20, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 24: return m5t_launch<P, 24, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    case 32: return m5t_launch<P, 32, Z>(dag, g, out, in, x, cf, tab, xpay, norm, red, skip, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_m5(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                      int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  if (prec == P64) return m5t_launch_p<P64, false>(dag, g, out, in, x, cf, nullptr, xpay, norm, red, skip, st);
  if (prec == P32) return m5t_launch_p<P32, false>(dag, g, out, in, x, cf, nullptr, xpay, norm, red, skip, st);
  if (prec == P16) return m5t_launch_p<P16, false>(dag, g, out, in, x, cf, nullptr, xpay, norm, red, skip, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_m5z(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x,
                       const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  M5Coef none;
  memset(&none, 0, sizeof(none));
  if (prec == P64) return m5t_launch_p<P64, true>(dag, g, out, in, x, none, tab, xpay, norm, red, skip, st);
  if (prec == P32) return m5t_launch_p<P32, true>(dag, g, out, in, x, none, tab, xpay, norm, red, skip, st);
  if (prec == P16) return m5t_launch_p<P16, true>(dag, g, out, in, x, none, tab, xpay, norm, red, skip, st);
  return cudaErrorInvalidValue;
}

}  // namespace cpsb

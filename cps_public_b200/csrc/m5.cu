// m5.cu -- Mobius fifth-direction kernels: exact M5^-1 fused with the b/c
// mixing of the 4-D hop.
//
// Restates, for real Mobius coefficients, zmobius_m5inv (cps_pp/src/util/
// dirac_op/d_op_zmobius/noarch/zmobius_m5inv.C:247-400 dag 0, :534-686 dag 1):
// a forward and a backward sweep along s per 4-D site and chirality with the
// domain-wall wall correction, and the mixing  b*psi_s + c*(P+ psi_{s-1} +
// P- psi_{s+1})  with -m_f walls of zmobius_kappa_dslash_5_plus_cmplx
// (zmobius_dslash_5_plus.C:125-376).  The sweeps are independent for every
// complex spinor component, so one thread owns one (site, storage chunk) column
// of Ls values in registers and the pass reads and writes each value once.
//
//   dag 0:  out = scale * mix(M5^-1 in)                 (precedes D_W in MatPc)
//   dag 1:  out = [x +] scale * M5^-dag(mix^dag(in))    (follows D_W^dag in MatPcDag)
//
// 16-bit storage: a chunk is one (chirality pair, colour) of both spins, half
// of a stored uint4 -- the same values as an FP32 chunk -- so the column
// arithmetic is shared.  The site's quantum is the maximum over its six
// chunks, so a site's chunks sit in one 8-lane group of a warp (two lanes
// idle) and the group agrees on the maximum by shuffles before encoding.
#include "blas.h"

namespace cpsb {

template <int P> struct ChunkT;
template <> struct ChunkT<P64> { static const int NCH = 12, NC = 1; typedef double T; };
template <> struct ChunkT<P32> { static const int NCH = 6, NC = 2; typedef float T; };
template <> struct ChunkT<P16> { static const int NCH = 6, NC = 2; typedef float T; };

template <int P>
__device__ __forceinline__ void ld_chunk(const SpinorPtr &f, long i, int k, cplx<typename ChunkT<P>::T> *v);
template <>
__device__ __forceinline__ void ld_chunk<P64>(const SpinorPtr &f, long i, int k, cplx<double> *v) {
  double2 a = __ldg((const double2 *)f.data + k * f.stride + i);
  v[0] = mk(a.x, a.y);
}
template <>
__device__ __forceinline__ void ld_chunk<P32>(const SpinorPtr &f, long i, int k, cplx<float> *v) {
  float4 a = __ldg((const float4 *)f.data + k * f.stride + i);  // spin-paired chunk
  v[0] = mk(a.x, a.z);
  v[1] = mk(a.y, a.w);
}
// A 16-bit column of Ls slices, chunk j = 3p + c (words 2j (Re) and 2j+1 (Im)
// of each site, both spins in each word): all raw loads issued first, then
// decoded, so the Ls loads are in flight together.
template <int LS>
__device__ __forceinline__ void ld_column16(const SpinorPtr &f, long base, long step, int j, cplx<float> (&v)[LS][2]) {
  uint2 w[LS];
  float q[LS];
#pragma unroll
  for (int s = 0; s < LS; s++) {
    const long i = base + (long)s * step;
    w[s] = __ldg((const uint2 *)((const uint4 *)f.data + (long)(j >> 1) * f.stride + i) + (j & 1));
    q[s] = __ldg(f.norm + i);
  }
#pragma unroll
  for (int s = 0; s < LS; s++) {
    v[s][0] = mk(dec16(w[s].x, 0) * q[s], dec16(w[s].y, 0) * q[s]);
    v[s][1] = mk(dec16(w[s].x, 1) * q[s], dec16(w[s].y, 1) * q[s]);
  }
}
template <int P>
__device__ __forceinline__ void st_chunk(const SpinorPtr &f, long i, int k, const cplx<typename ChunkT<P>::T> *v);
template <>
__device__ __forceinline__ void st_chunk<P64>(const SpinorPtr &f, long i, int k, const cplx<double> *v) {
  ((double2 *)f.data)[k * f.stride + i] = make_double2(v[0].re, v[0].im);
}
template <>
__device__ __forceinline__ void st_chunk<P32>(const SpinorPtr &f, long i, int k, const cplx<float> *v) {
  ((float4 *)f.data)[k * f.stride + i] = make_float4(v[0].re, v[1].re, v[0].im, v[1].im);
}
// Stores the column y[0..LS) of chunk j (16-bit), slice s at base + s*step:
// the site maxima of all slices first, combined across the 8-lane group by
// independent shuffles (pipelined over s rather than one dependent round trip
// per slice), then encode and store.  Every lane of the warp calls it.
// Returns the sum of |stored values|^2 of this lane.
template <int LS>
__device__ __forceinline__ double st_column16(const SpinorPtr &f, long base, long step, int j,
                                              const cplx<float> (&y)[LS][2], bool active) {
  float m[LS];
#pragma unroll
  for (int s = 0; s < LS; s++)
    m[s] = active ? fmaxf(fmaxf(fabsf(y[s][0].re), fabsf(y[s][0].im)), fmaxf(fabsf(y[s][1].re), fabsf(y[s][1].im)))
                  : 0.f;
#pragma unroll
  for (int d = 1; d < 8; d <<= 1)
#pragma unroll
    for (int s = 0; s < LS; s++) m[s] = fmaxf(m[s], __shfl_xor_sync(0xffffffffu, m[s], d));
  double acc = 0;
  if (!active) return acc;
#pragma unroll
  for (int s = 0; s < LS; s++) {
    const float scale = m[s] > 0.f ? 32767.0f / m[s] : 0.f;
    const float nq = m[s] * (1.0f / 32767.0f);
    const long i = base + (long)s * step;
    const unsigned wx = enc16x2(y[s][0].re, y[s][1].re, scale), wy = enc16x2(y[s][0].im, y[s][1].im, scale);
    ((uint2 *)((uint4 *)f.data + (long)(j >> 1) * f.stride + i))[j & 1] = make_uint2(wx, wy);
    if (j == 0) f.norm[i] = nq;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const float a = dec16(wx, h) * nq, b = dec16(wy, h) * nq;
      acc += (double)(a * a + b * b);
    }
  }
  return acc;
}

// v[s] += f * w[s] on one chunk
#define AXPYC(dst, f, src)                                   \
  _Pragma("unroll") for (int q = 0; q < NC; q++) {           \
    (dst)[q].re += (f) * (src)[q].re;                        \
    (dst)[q].im += (f) * (src)[q].im;                        \
  }
#define SCALC(dst, f)                                        \
  _Pragma("unroll") for (int q = 0; q < NC; q++) {           \
    (dst)[q].re *= (f);                                      \
    (dst)[q].im *= (f);                                      \
  }

// v[s] <- b v[s] + c v[s -+ 1] in place (from_below: slice s-1, the wall term
// mwall v[Ls-1] at s = 0; otherwise slice s+1, the wall mwall v[0] at Ls-1):
// sweeping away from the slice each step reads keeps that slice unmodified,
// so no second column of registers is needed.
template <int LS, int NC, typename T>
__device__ __forceinline__ void mix_inplace(cplx<T> (&v)[LS][NC], bool from_below, T b, T c, T mwall) {
  if (from_below) {
    cplx<T> wall[NC];
#pragma unroll
    for (int q = 0; q < NC; q++) wall[q] = v[LS - 1][q];
#pragma unroll
    for (int s = LS - 1; s >= 1; s--)
#pragma unroll
      for (int q = 0; q < NC; q++) v[s][q] = cscale(b, v[s][q]) + cscale(c, v[s - 1][q]);
#pragma unroll
    for (int q = 0; q < NC; q++) v[0][q] = cscale(b, v[0][q]) + cscale(mwall, wall[q]);
  } else {
    cplx<T> wall[NC];
#pragma unroll
    for (int q = 0; q < NC; q++) wall[q] = v[0][q];
#pragma unroll
    for (int s = 0; s <= LS - 2; s++)
#pragma unroll
      for (int q = 0; q < NC; q++) v[s][q] = cscale(b, v[s][q]) + cscale(c, v[s + 1][q]);
#pragma unroll
    for (int q = 0; q < NC; q++) v[LS - 1][q] = cscale(b, v[LS - 1][q]) + cscale(mwall, wall[q]);
  }
}

// v <- mix(M5^-1 v) (DAG 0) or M5^-dag(mix^dag(v)) (DAG 1) on one column, in
// place, real coefficients; the output scale is applied by the caller.
template <int LS, int DAG, int NC, typename T>
__device__ __forceinline__ void m5_column(cplx<T> (&v)[LS][NC], bool upper, const M5Coef &cf) {
  const T K = (T)cf.K, b = (T)cf.b, c = (T)cf.c, mwall = (T)(-cf.mass * cf.c), invd = (T)cf.invd;
  // mix^dag (DAG 1): upper from s+1, lower from s-1
  if (DAG == 1) mix_inplace<LS, NC, T>(v, !upper, b, c, mwall);
  // M5^-1 (DAG 0) or M5^-dag (DAG 1) sweeps.  The structure of the
  // dag-0 lower sweep equals the dag-1 upper sweep and vice versa.
  const bool walls_first = (DAG == 0) ? !upper : upper;
  if (walls_first) {
    SCALC(v[LS - 1], invd);
#pragma unroll
    for (int s = 0; s <= LS - 2; s++) { const T f = (T)cf.f1[s]; AXPYC(v[LS - 1], f, v[s]); }
#pragma unroll
    for (int s = LS - 2; s >= 0; s--) { AXPYC(v[s], -K, v[s + 1]); }
  } else {
#pragma unroll
    for (int s = 0; s <= LS - 2; s++) { AXPYC(v[s + 1], -K, v[s]); }
#pragma unroll
    for (int s = LS - 2; s >= 0; s--) { const T f = (T)cf.f2[s]; AXPYC(v[s], f, v[LS - 1]); }
    SCALC(v[LS - 1], invd);
  }
  // mix (DAG 0): upper from s-1, lower from s+1
  if (DAG == 0) mix_inplace<LS, NC, T>(v, upper, b, c, mwall);
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

template <int P, int LS, int DAG, bool XPAY, bool NORM, int NT>
__global__ void __launch_bounds__(NT) m5_kernel(Geom g, SpinorPtr out, SpinorPtr in, SpinorPtr xv, M5Coef cf,
                                                Reduce red, const int *skip) {
  typedef typename ChunkT<P>::T T;
  const int NCH = ChunkT<P>::NCH, NC = ChunkT<P>::NC;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * LS;
  const long work = (long)g.n4cb * NCH;
  double acc = 0;
  const T sc = (T)cf.scale;
  const bool sk = skip && skip[rhs];
  for (long w = (long)blockIdx.x * NT + threadIdx.x; !sk && w < work; w += (long)gridDim.x * NT) {
    const int x = (int)(w % g.n4cb);
    const int k = (int)(w / g.n4cb);
    const long base = rhs * per + x;
    cplx<T> v[LS][NC];
#pragma unroll
    for (int s = 0; s < LS; s++) ld_chunk<P>(in, base + (long)s * g.n4cb, k, v[s]);
    m5_column<LS, DAG, NC, T>(v, k < NCH / 2, cf);
#pragma unroll
    for (int s = 0; s < LS; s++) {
      cplx<T> o[NC];
      if (XPAY) ld_chunk<P>(xv, base + (long)s * g.n4cb, k, o);
#pragma unroll
      for (int q = 0; q < NC; q++) {
        if (XPAY) o[q] = o[q] + cscale(sc, v[s][q]);
        else o[q] = cscale(sc, v[s][q]);
        if (NORM) acc += (double)o[q].re * o[q].re + (double)o[q].im * o[q].im;
      }
      st_chunk<P>(out, base + (long)s * g.n4cb, k, o);
    }
  }
  if (NORM) m5_norm_epilogue<NT>(acc, g, red, skip, sh);
}

// 16-bit storage: four sites per warp, 8 lanes per site (chunks 0..5, lanes
// 6 and 7 idle); the loop is warp-uniform so every shuffle has the full warp.
template <int LS, int DAG, bool XPAY, bool NORM, int NT>
__global__ void __launch_bounds__(NT) m5h_kernel(Geom g, SpinorPtr out, SpinorPtr in, SpinorPtr xv, M5Coef cf,
                                                 Reduce red, const int *skip) {
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * LS;
  const int lane = threadIdx.x & 31, j = lane & 7;
  const long nw = (long)gridDim.x * (NT / 32);
  double acc = 0;
  const float sc = (float)cf.scale;
  const bool sk = skip && skip[rhs];
  for (long x0 = ((long)blockIdx.x * (NT / 32) + (threadIdx.x >> 5)) * 4; !sk && x0 < g.n4cb; x0 += nw * 4) {
    const long x = x0 + (lane >> 3);
    const bool active = j < 6 && x < g.n4cb;
    const int jj = active ? j : 0;
    const long base = rhs * per + (active ? x : 0);
    cplx<float> v[LS][2];
    // inactive lanes read a valid chunk of site 0 and store nothing
    ld_column16<LS>(in, base, g.n4cb, jj, v);
    m5_column<LS, DAG, 2, float>(v, jj < 3, cf);
    if (XPAY) {
      cplx<float> o[LS][2];
      ld_column16<LS>(xv, base, g.n4cb, jj, o);
#pragma unroll
      for (int s = 0; s < LS; s++)
#pragma unroll
        for (int q = 0; q < 2; q++) v[s][q] = o[s][q] + cscale(sc, v[s][q]);
    } else {
#pragma unroll
      for (int s = 0; s < LS; s++)
#pragma unroll
        for (int q = 0; q < 2; q++) v[s][q] = cscale(sc, v[s][q]);
    }
    const double n = st_column16<LS>(out, base, g.n4cb, jj, v, active);
    if (NORM) acc += n;
  }
  if (NORM) m5_norm_epilogue<NT>(acc, g, red, skip, sh);
}

template <int P, int LS>
static cudaError_t m5_launch_ls(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                                int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  const int NT = 128;
  if constexpr (P == P16) {
    dim3 grid(grid_blocks((long)g.n4cb * 8, NT), g.nrhs);
#define M5H(D, XP, NR)                                                                              \
    if (dag == D && !!xpay == XP && !!norm == NR) {                                                 \
      m5h_kernel<LS, D, XP, NR, NT><<<grid, NT, 0, st>>>(g, out, in, x, cf, red, skip);             \
      return launched();                                                                            \
    }
    M5H(0, false, false) M5H(0, true, false) M5H(0, true, true) M5H(0, false, true)
    M5H(1, false, false) M5H(1, true, false) M5H(1, true, true) M5H(1, false, true)
#undef M5H
    return cudaErrorInvalidValue;
  } else {
  dim3 grid(grid_blocks((long)g.n4cb * ChunkT<P>::NCH, NT), g.nrhs);
#define M5L(D, XP, NR)                                                                              \
  if (dag == D && !!xpay == XP && !!norm == NR) {                                                   \
    m5_kernel<P, LS, D, XP, NR, NT><<<grid, NT, 0, st>>>(g, out, in, x, cf, red, skip);             \
    return launched();                                                                              \
  }
  M5L(0, false, false) M5L(0, true, false) M5L(0, true, true) M5L(0, false, true)
  M5L(1, false, false) M5L(1, true, false) M5L(1, true, true) M5L(1, false, true)
#undef M5L
  return cudaErrorInvalidValue;
  }
}

template <int P>
static cudaError_t m5_launch_p(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                               int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  switch (g.ls) {
    case 4: return m5_launch_ls<P, 4>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 8: return m5_launch_ls<P, 8>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 12: return m5_launch_ls<P, 12>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 16: return m5_launch_ls<P, 16>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 20: return m5_launch_ls<P, 20>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 24: return m5_launch_ls<P, 24>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    case 32: return m5_launch_ls<P, 32>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_m5(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                      int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  if (prec == P64) return m5_launch_p<P64>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
  if (prec == P32) return m5_launch_p<P32>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
  if (prec == P16) return m5_launch_p<P16>(dag, g, out, in, x, cf, xpay, norm, red, skip, st);
  return cudaErrorInvalidValue;
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

template <int P, int LS, int DAG, bool XPAY, bool NORM, int NT>
__global__ void __launch_bounds__(NT) m5z_kernel(Geom g, SpinorPtr out, SpinorPtr in, SpinorPtr xv,
                                                 const ZM5Tab *tab, Reduce red, const int *skip) {
  typedef typename ChunkT<P>::T T;
  const int NCH = ChunkT<P>::NCH, NC = ChunkT<P>::NC;
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * LS;
  const long work = (long)g.n4cb * NCH;
  double acc = 0;
  const bool sk = skip && skip[rhs];
  for (long w = (long)blockIdx.x * NT + threadIdx.x; !sk && w < work; w += (long)gridDim.x * NT) {
    const int x = (int)(w % g.n4cb);
    const int k = (int)(w / g.n4cb);
    const long base = rhs * per + x;
    cplx<T> v[LS][NC];
#pragma unroll
    for (int s = 0; s < LS; s++) ld_chunk<P>(in, base + (long)s * g.n4cb, k, v[s]);
    m5z_column<LS, DAG, NC, T>(v, k < NCH / 2 ? 0 : 1, tab);
#pragma unroll
    for (int s = 0; s < LS; s++) {
      cplx<T> o[NC];
      if (XPAY) ld_chunk<P>(xv, base + (long)s * g.n4cb, k, o);
#pragma unroll
      for (int q = 0; q < NC; q++) {
        o[q] = XPAY ? o[q] + v[s][q] : v[s][q];
        if (NORM) acc += (double)o[q].re * o[q].re + (double)o[q].im * o[q].im;
      }
      st_chunk<P>(out, base + (long)s * g.n4cb, k, o);
    }
  }
  if (NORM) m5_norm_epilogue<NT>(acc, g, red, skip, sh);
}

// 16-bit zMobius: the lane layout of m5h_kernel.
template <int LS, int DAG, bool XPAY, bool NORM, int NT>
__global__ void __launch_bounds__(NT) m5zh_kernel(Geom g, SpinorPtr out, SpinorPtr in, SpinorPtr xv,
                                                  const ZM5Tab *tab, Reduce red, const int *skip) {
  __shared__ double sh[NT / 32];
  const int rhs = blockIdx.y;
  const long per = (long)g.n4cb * LS;
  const int lane = threadIdx.x & 31, j = lane & 7;
  const long nw = (long)gridDim.x * (NT / 32);
  double acc = 0;
  const bool sk = skip && skip[rhs];
  for (long x0 = ((long)blockIdx.x * (NT / 32) + (threadIdx.x >> 5)) * 4; !sk && x0 < g.n4cb; x0 += nw * 4) {
    const long x = x0 + (lane >> 3);
    const bool active = j < 6 && x < g.n4cb;
    const int jj = active ? j : 0;
    const long base = rhs * per + (active ? x : 0);
    cplx<float> v[LS][2];
    // inactive lanes read a valid chunk of site 0 and store nothing
    ld_column16<LS>(in, base, g.n4cb, jj, v);
    m5z_column<LS, DAG, 2, float>(v, jj < 3 ? 0 : 1, tab);
    if (XPAY) {
      cplx<float> o[LS][2];
      ld_column16<LS>(xv, base, g.n4cb, jj, o);
#pragma unroll
      for (int s = 0; s < LS; s++)
#pragma unroll
        for (int q = 0; q < 2; q++) v[s][q] = o[s][q] + v[s][q];
    }
    const double n = st_column16<LS>(out, base, g.n4cb, jj, v, active);
    if (NORM) acc += n;
  }
  if (NORM) m5_norm_epilogue<NT>(acc, g, red, skip, sh);
}

template <int P, int LS>
static cudaError_t m5z_launch_ls(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x,
                                 const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip,
                                 cudaStream_t st) {
  const int NT = 128;
  if constexpr (P == P16) {
    dim3 grid(grid_blocks((long)g.n4cb * 8, NT), g.nrhs);
#define M5ZH(D, XP, NR)                                                                             \
    if (dag == D && !!xpay == XP && !!norm == NR) {                                                 \
      m5zh_kernel<LS, D, XP, NR, NT><<<grid, NT, 0, st>>>(g, out, in, x, tab, red, skip);           \
      return launched();                                                                            \
    }
    M5ZH(0, false, false) M5ZH(0, true, false) M5ZH(0, true, true)
    M5ZH(1, false, false) M5ZH(1, true, false) M5ZH(1, true, true)
#undef M5ZH
    return cudaErrorInvalidValue;
  } else {
  dim3 grid(grid_blocks((long)g.n4cb * ChunkT<P>::NCH, NT), g.nrhs);
#define M5ZL(D, XP, NR)                                                                             \
  if (dag == D && !!xpay == XP && !!norm == NR) {                                                   \
    m5z_kernel<P, LS, D, XP, NR, NT><<<grid, NT, 0, st>>>(g, out, in, x, tab, red, skip);           \
    return launched();                                                                              \
  }
  M5ZL(0, false, false) M5ZL(0, true, false) M5ZL(0, true, true)
  M5ZL(1, false, false) M5ZL(1, true, false) M5ZL(1, true, true)
#undef M5ZL
  return cudaErrorInvalidValue;
  }
}

template <int P>
static cudaError_t m5z_launch_p(int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x,
                                const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip,
                                cudaStream_t st) {
  switch (g.ls) {
    case 4: return m5z_launch_ls<P, 4>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 8: return m5z_launch_ls<P, 8>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 12: return m5z_launch_ls<P, 12>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 16: return m5z_launch_ls<P, 16>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 20: return m5z_launch_ls<P, 20>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 24: return m5z_launch_ls<P, 24>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    case 32: return m5z_launch_ls<P, 32>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_m5z(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x,
                       const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip, cudaStream_t st) {
  if (prec == P64) return m5z_launch_p<P64>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
  if (prec == P32) return m5z_launch_p<P32>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
  if (prec == P16) return m5z_launch_p<P16>(dag, g, out, in, x, tab, xpay, norm, red, skip, st);
  return cudaErrorInvalidValue;
}

}  // namespace cpsb

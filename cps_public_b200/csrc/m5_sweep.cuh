// m5_sweep.cuh -- the real-coefficient Mobius fifth-direction column
// operations: M5^-1 (forward and backward sweeps along s with the domain-wall
// wall correction) fused with the b/c mixing, on one column of Ls values held
// in registers.  Used by the tiled M5 kernel (m5.cu) and by the hop kernel with
// the sweeps fused into its epilogue (hop_m5.cuh).
//
// Restates, for real coefficients, zmobius_m5inv (cps_pp/src/util/dirac_op/
// d_op_zmobius/noarch/zmobius_m5inv.C:247-400 dag 0, :534-686 dag 1) and the
// mixing b*psi_s + c*(P+ psi_{s-1} + P- psi_{s+1}) with -m_f walls of
// zmobius_kappa_dslash_5_plus_cmplx (zmobius_dslash_5_plus.C:125-376).
#pragma once
#include "blas.h"
#include "cpsb_device.cuh"

namespace cpsb {

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

}  // namespace cpsb

// hop.cuh -- the Wilson / domain-wall hopping kernel for sm_100a, all three
// storage precisions (FP64, FP32, 16-bit fixed point).
//
// Operator: CPS's wilson_dslash (cps_pp/src/util/dirac_op/d_op_wilson/noarch/
// wilson_dslash.C:173-516) with spin projection -- each of the 8 neighbours is
// projected to a half spinor, multiplied by its link (or the adjoint) and
// re-expanded -- applied to every slice of a 5-D field: DWF slices use 5-D
// checkerboarding (dwf_dslash_4.C:107-112, slice s holds 4-D parity (s+cb)%2)
// and get the 5th-direction hop of dwf_dslash_5_plus.C:111-340 fused in;
// Mobius slices all share one 4-D parity (DWF_4D_EOPREC_EE).
//
// Work decomposition (the column layout of cpsb_device.cuh).  A field is a
// set of columns, one per (4-D checkerboard site x, slice class k), each
// holding the class's slices of that site as consecutive entries.  A work unit
// is a tile of TX consecutive columns of one class, taken for a group of RG
// right-hand sides at a time (RG = 1 or all of them; A.rg); a block sweeps its
// unit's columns x slices x right-hand sides of the group.  Thread t owns
// slice t % C (C the column height), right-hand side (t / C) % RG and column
// t / (C RG), so:
//  * the 32 lanes of a warp read whole neighbour columns per 16-byte chunk --
//    contiguous 128-byte segments that start on 128-byte boundaries when C is
//    a multiple of 8 (DWF Ls 16: 4 columns x 8 slices per warp);
//  * the unit's 8*TX links are loaded, reconstructed (recon-12 storage) and
//    written to shared memory once, with the antiperiodic time sign folded in,
//    and every slice and right-hand side of the unit reads them from there,
//    C lanes at a time on the same address (a broadcast); for FP32 / 16-bit
//    each element is stored as (re, re, im, im) so that it is one operand pair
//    of the packed FP32x2 instructions (launch shapes without the table, LC
//    false, read recon-12 links from global memory per thread instead);
//  * neighbour column offsets are computed once per unit;
//  * units run in tile order, optionally inside groups of A.rgroup right-hand
//    sides (the group slowest), and the grid holds only the blocks resident at
//    once, so the columns that blocks in flight touch -- their own and their
//    neighbours' up to one time slice away -- are read while they sit in L2.
//
// FP32 and 16-bit storage keep spins (2p, 2p+1) of one colour in the two lanes
// of a float2 and run every step of the hop in Blackwell's packed FP32x2
// arithmetic (FFMA2 / FADD2 / FMUL2).  16-bit spinors are stored as biased
// 15-bit integers (value + 16384, in [1, 32767]) with one float quantum per
// entry; the spin projection of each 16-bit neighbour is done on the packed
// integers themselves (two 16-bit lanes per 32-bit add, exact because the sum
// of two biased values stays below 2^16), decoded once per half spinor, and the
// neighbour's quantum is folded into the FMA that accumulates it.  The output is
// re-encoded with its own quantum.
//
// Epilogues (no extra pass over memory): out = x + a*D in (XPAY) or a*D in,
// optionally |out|^2 per right-hand side (NORM), or the CG residual update
// r -= alpha (D-output + sigma p) with |r|^2 and the recurrence scalars (CGR),
// where the D output is consumed in registers and not stored, together with
// the solution update x += alpha p when A.cg_x is set.  Reductions are
// deterministic (partials in block order, summed by the last block).
#pragma once
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include "cpsb_device.cuh"
#include "cg_state.h"
#include "cpsb_kernels.h"

namespace cpsb {

// ---------------------------------------------------------------- packed FP32x2
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2b(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 swp(float2 a) { return make_float2(a.y, a.x); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// A spinor as two spin pairs: re[p][c] = (Re psi_{2p,c}, Re psi_{2p+1,c}).
struct SpX2 { float2 re[2][3], im[2][3]; };
// A half spinor (spins h0, h1 in the lanes) per colour.
struct HfX2 { float2 re[3], im[3]; };

// Two biased 16-bit values of one word as a float2 of exact integers: the
// integer is placed under the exponent byte 0x4B (the float 2^23 + u) and
// 2^23 + bias is subtracted.  Stored spinor words carry bias 16384 (values in
// [-16383, 16383]); sums and differences of two stored words carry 32768.
template <int BIAS> __device__ __forceinline__ float2 dec16x2b(unsigned w) {
  return add2(f2(__int_as_float((int)__byte_perm(w, 0x4B00u, 0x5410u)),
                 __int_as_float((int)__byte_perm(w, 0x4B00u, 0x5432u))),
              f2b(-(8388608.0f + (float)BIAS)));
}
__device__ __forceinline__ float2 dec16x2(unsigned w) { return dec16x2b<16384>(w); }
// Biased encodings of round(v.x*scale), round(v.y*scale) in one word: adding
// 1.5*2^23 + 2^14 leaves the rounded, biased integer in the low mantissa bits
// (|v|*scale <= 16383 by construction of scale).
__device__ __forceinline__ unsigned enc16x2p(float2 v, float2 scale) {
  const float2 r = fma2(v, scale, f2b(12599296.0f));
  return __byte_perm(__float_as_uint(r.x), __float_as_uint(r.y), 0x5410u);
}

// Lane-wise sums and differences of two packed words of biased 16-bit values
// (each in [1, 32767]); every result lane is v_a +- v_b + 32768 in [2, 65534],
// so no lane carries or borrows into the other.
__device__ __forceinline__ unsigned pk_add(unsigned a, unsigned b) { return a + b; }
__device__ __forceinline__ unsigned pk_sub(unsigned a, unsigned b) { return a + 0x80008000u - b; }
// low lane a - b, high lane a + b (b ^ 0x7FFF = 32767 - b in the low lane)
__device__ __forceinline__ unsigned pk_subadd(unsigned a, unsigned b) { return a + (b ^ 0x00007FFFu) + 1u; }
// low lane a + b, high lane a - b
__device__ __forceinline__ unsigned pk_addsub(unsigned a, unsigned b) { return a + (b ^ 0x7FFF0000u) + 0x10000u; }
__device__ __forceinline__ unsigned pk_swap(unsigned b) { return __byte_perm(b, 0u, 0x1032u); }

// ---------------------------------------------------------------- raw entries
// An entry as loaded, before unpacking, so loads can be issued ahead of the
// arithmetic that consumes them.
template <int P> struct Raw;
template <> struct Raw<P64> { double2 c[12]; };
template <> struct Raw<P32> { float4 c[6]; };
template <> struct Raw<P16> { uint4 c[3]; float nrm; };

template <int P> __device__ __forceinline__ Raw<P> load_raw(const SpinorPtr &f, unsigned i);
template <> __device__ __forceinline__ Raw<P64> load_raw<P64>(const SpinorPtr &f, unsigned i) {
  const double2 *b = entry_ptr<12, double2>(f.data, i);
  Raw<P64> r;
#pragma unroll
  for (int k = 0; k < 12; k++) r.c[k] = __ldg(b + 8 * k);
  return r;
}
// The same through L2 only (ld.global.cg): for kernels that read a field that
// other blocks of the same launch wrote (the read-only path may hold stale lines).
__device__ __forceinline__ Raw<P64> load_raw64_l2(const SpinorPtr &f, unsigned i) {
  const double2 *b = entry_ptr<12, double2>(f.data, i);
  Raw<P64> r;
#pragma unroll
  for (int k = 0; k < 12; k++) r.c[k] = __ldcg(b + 8 * k);
  return r;
}
template <bool L2ONLY> __device__ __forceinline__ Raw<P64> load_raw64(const SpinorPtr &f, unsigned i) {
  if constexpr (L2ONLY) return load_raw64_l2(f, i);
  else return load_raw<P64>(f, i);
}
template <> __device__ __forceinline__ Raw<P32> load_raw<P32>(const SpinorPtr &f, unsigned i) {
  const float4 *b = entry_ptr<6, float4>(f.data, i);
  Raw<P32> r;
#pragma unroll
  for (int k = 0; k < 6; k++) r.c[k] = __ldg(b + 8 * k);
  return r;
}
template <> __device__ __forceinline__ Raw<P16> load_raw<P16>(const SpinorPtr &f, unsigned i) {
  const uint4 *b = entry_ptr<3, uint4>(f.data, i);
  Raw<P16> r;
#pragma unroll
  for (int k = 0; k < 3; k++) r.c[k] = __ldg(b + 8 * k);
  r.nrm = __ldg(f.norm + i);
  return r;
}

__device__ __forceinline__ SpX2 unpack(const Raw<P32> &r, float *nrm) {
  SpX2 s;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    s.re[k / 3][k % 3] = f2(r.c[k].x, r.c[k].y);
    s.im[k / 3][k % 3] = f2(r.c[k].z, r.c[k].w);
  }
  *nrm = 1.0f;
  return s;
}
__device__ __forceinline__ SpX2 unpack(const Raw<P16> &r, float *nrm) {
  SpX2 s;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int pa = 2 * k, pb = 2 * k + 1;  // (3p + c) of the two complex values of the chunk
    s.re[pa / 3][pa % 3] = dec16x2(r.c[k].x);
    s.im[pa / 3][pa % 3] = dec16x2(r.c[k].y);
    s.re[pb / 3][pb % 3] = dec16x2(r.c[k].z);
    s.im[pb / 3][pb % 3] = dec16x2(r.c[k].w);
  }
  *nrm = r.nrm;
  return s;
}
__device__ __forceinline__ Spinor<double> unpack64(const Raw<P64> &r) {
  Spinor<double> s;
#pragma unroll
  for (int k = 0; k < 12; k++) s.c[k / 3][k % 3] = mk(r.c[k].x, r.c[k].y);
  return s;
}

// One chirality pair of an entry (p = 0: spins 0, 1; p = 1: spins 2, 3) for the
// 5th-direction hop.  16-bit pair 0 is chunk 0 and the low half of chunk 1,
// pair 1 the high half of chunk 1 and chunk 2.
template <int P> __device__ __forceinline__ HfX2 load_pair(const SpinorPtr &f, unsigned i, int p, float *nrm);
template <> __device__ __forceinline__ HfX2 load_pair<P32>(const SpinorPtr &f, unsigned i, int p, float *nrm) {
  const float4 *b = entry_ptr<6, float4>(f.data, i) + 24 * p;
  HfX2 h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float4 v = __ldg(b + 8 * c);
    h.re[c] = f2(v.x, v.y);
    h.im[c] = f2(v.z, v.w);
  }
  *nrm = 1.0f;
  return h;
}
template <> __device__ __forceinline__ HfX2 load_pair<P16>(const SpinorPtr &f, unsigned i, int p, float *nrm) {
  const uint4 *b = entry_ptr<3, uint4>(f.data, i);
  const uint4 v = __ldg(b + (p ? 16 : 0));
  const uint2 m = __ldg((const uint2 *)(b + 8) + p);
  HfX2 h;
  if (p == 0) {
    h.re[0] = dec16x2(v.x); h.im[0] = dec16x2(v.y);
    h.re[1] = dec16x2(v.z); h.im[1] = dec16x2(v.w);
    h.re[2] = dec16x2(m.x); h.im[2] = dec16x2(m.y);
  } else {
    h.re[0] = dec16x2(m.x); h.im[0] = dec16x2(m.y);
    h.re[1] = dec16x2(v.x); h.im[1] = dec16x2(v.y);
    h.re[2] = dec16x2(v.z); h.im[2] = dec16x2(v.w);
  }
  *nrm = __ldg(f.norm + i);
  return h;
}

// Stores an entry and returns |stored value|^2 (for 16-bit storage the norm of
// the rounded value that a later load returns; the squares are summed in FP32
// and the quantum's square applied in FP64, since it can lie below FP32 range).
template <int P> __device__ __forceinline__ double store_x2(const SpinorPtr &f, unsigned i, const SpX2 &s);
template <> __device__ __forceinline__ double store_x2<P32>(const SpinorPtr &f, unsigned i, const SpX2 &s) {
  float4 *b = (float4 *)entry_ptr<6, float4>(f.data, i);
  float2 n = f2b(0.f);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float2 re = s.re[k / 3][k % 3], im = s.im[k / 3][k % 3];
    b[8 * k] = make_float4(re.x, re.y, im.x, im.y);
    n = fma2(re, re, n);
    n = fma2(im, im, n);
  }
  return (double)(n.x + n.y);
}
template <> __device__ __forceinline__ double store_x2<P16>(const SpinorPtr &f, unsigned i, const SpX2 &s) {
  float m = 0.f;
#pragma unroll
  for (int p = 0; p < 2; p++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      m = fmaxf(fmaxf(m, fmaxf(fabsf(s.re[p][c].x), fabsf(s.re[p][c].y))),
                fmaxf(fabsf(s.im[p][c].x), fabsf(s.im[p][c].y)));
  const float scale = m > 0.f ? S16_MAX / m : 0.f;
  const float q = m * (1.0f / S16_MAX);
  f.norm[i] = q;
  const float2 sc = f2b(scale);
  uint4 *b = (uint4 *)entry_ptr<3, uint4>(f.data, i);
  float2 n = f2b(0.f);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int pa = 2 * k, pb = 2 * k + 1;
    unsigned w[4];
    w[0] = enc16x2p(s.re[pa / 3][pa % 3], sc);
    w[1] = enc16x2p(s.im[pa / 3][pa % 3], sc);
    w[2] = enc16x2p(s.re[pb / 3][pb % 3], sc);
    w[3] = enc16x2p(s.im[pb / 3][pb % 3], sc);
    b[8 * k] = make_uint4(w[0], w[1], w[2], w[3]);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 d = dec16x2(w[j]);
      n = fma2(d, d, n);
    }
  }
  return (double)(n.x + n.y) * ((double)q * q);
}

// ---------------------------------------------------------------- packed hop pieces
// (1 + sg*gamma_mu) psi -> half spinor (h0, h1) in the lanes; the gamma
// matrices of project() in cpsb_device.cuh written per spin pair: re[1] is
// (psi2, psi3) and swp(re[1]) is (psi3, psi2).
template <int MU> __device__ __forceinline__ HfX2 project_x2(const SpX2 &s, float sg) {
  constexpr bool SW = false;
  HfX2 h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (MU == 0) {         // h0 = psi0 + i sg psi3, h1 = psi1 + i sg psi2
      h.re[c] = fma2(f2b(-sg), SW ? s.im[1][c] : swp(s.im[1][c]), s.re[0][c]);
      h.im[c] = fma2(f2b(sg), SW ? s.re[1][c] : swp(s.re[1][c]), s.im[0][c]);
    } else if (MU == 1) {  // h0 = psi0 - sg psi3, h1 = psi1 + sg psi2
      h.re[c] = fma2(f2(-sg, sg), SW ? s.re[1][c] : swp(s.re[1][c]), s.re[0][c]);
      h.im[c] = fma2(f2(-sg, sg), SW ? s.im[1][c] : swp(s.im[1][c]), s.im[0][c]);
    } else if (MU == 2) {  // h0 = psi0 + i sg psi2, h1 = psi1 - i sg psi3
      h.re[c] = fma2(f2(-sg, sg), s.im[1][c], s.re[0][c]);
      h.im[c] = fma2(f2(sg, -sg), s.re[1][c], s.im[0][c]);
    } else {               // h0 = psi0 + sg psi2, h1 = psi1 + sg psi3
      h.re[c] = fma2(f2b(sg), s.re[1][c], s.re[0][c]);
      h.im[c] = fma2(f2b(sg), s.im[1][c], s.im[0][c]);
    }
  }
  return h;
}

// (1 + sg*gamma_mu) psi of a 16-bit neighbour (POS: sg = +1), projected on
// the stored integers: each word of the half spinor is one (or, with a lane
// swap or a lane-dependent sign, two or three) integer operations on two
// stored words, and only the 6 projected words are decoded (bias 32768) --
// against decoding all 12 words and 6 packed FMAs.  The combinations are those
// of project_x2.
template <int MU, bool POS> __device__ __forceinline__ HfX2 iproject(const Raw<P16> &r) {
  const unsigned w[12] = {r.c[0].x, r.c[0].y, r.c[0].z, r.c[0].w, r.c[1].x, r.c[1].y,
                          r.c[1].z, r.c[1].w, r.c[2].x, r.c[2].y, r.c[2].z, r.c[2].w};
  HfX2 h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    // upper pair (spins 0, 1) and lower pair (spins 2, 3), re and im words
    const unsigned are = w[c * 2], aim = w[c * 2 + 1], bre = w[(3 + c) * 2], bim = w[(3 + c) * 2 + 1];
    unsigned hre, him;
    if (MU == 0) {         // re: (a0 - sg b3.im, a1 - sg b2.im); im: (a0 + sg b3.re, a1 + sg b2.re)
      hre = POS ? pk_sub(are, pk_swap(bim)) : pk_add(are, pk_swap(bim));
      him = POS ? pk_add(aim, pk_swap(bre)) : pk_sub(aim, pk_swap(bre));
    } else if (MU == 1) {  // (a0 - sg b3, a1 + sg b2), re and im alike
      hre = POS ? pk_subadd(are, pk_swap(bre)) : pk_addsub(are, pk_swap(bre));
      him = POS ? pk_subadd(aim, pk_swap(bim)) : pk_addsub(aim, pk_swap(bim));
    } else if (MU == 2) {  // re: (a0 - sg b2.im, a1 + sg b3.im); im: (a0 + sg b2.re, a1 - sg b3.re)
      hre = POS ? pk_subadd(are, bim) : pk_addsub(are, bim);
      him = POS ? pk_addsub(aim, bre) : pk_subadd(aim, bre);
    } else {               // (a0 + sg b2, a1 + sg b3)
      hre = POS ? pk_add(are, bre) : pk_sub(are, bre);
      him = POS ? pk_add(aim, bim) : pk_sub(aim, bim);
    }
    h.re[c] = dec16x2b<32768>(hre);
    h.im[c] = dec16x2b<32768>(him);
  }
  return h;
}

// U h (DAG = false) or U^dag h (DAG = true) for both spins; the link elements
// come from shared memory as (ur, ur, ui, ui), row-major.
template <bool DAG> __device__ __forceinline__ HfX2 umul_x2(const float4 *l, const HfX2 &h) {
  HfX2 o;
  float2 nh[3];
#pragma unroll
  for (int k = 0; k < 3; k++) nh[k] = DAG ? f2(-h.re[k].x, -h.re[k].y) : f2(-h.im[k].x, -h.im[k].y);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 re = f2b(0.f), im = f2b(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float4 e = l[DAG ? 3 * k + r : 3 * r + k];
      const float2 ur = lo2(e), ui = hi2(e);
      re = fma2(ur, h.re[k], re);
      im = fma2(ur, h.im[k], im);
      if (DAG) {  // conj(u) h: re += ui Im h, im -= ui Re h
        re = fma2(ui, h.im[k], re);
        im = fma2(ui, nh[k], im);
      } else {    // u h: re -= ui Im h, im += ui Re h
        re = fma2(ui, nh[k], re);
        im = fma2(ui, h.re[k], im);
      }
    }
    o.re[r] = re;
    o.im[r] = im;
  }
  return o;
}

// The same with the link in registers (launch shapes without the link table).
template <bool DAG> __device__ __forceinline__ HfX2 umul_x2r(const Link<float> &u, const HfX2 &h) {
  HfX2 o;
  float2 nh[3];
#pragma unroll
  for (int k = 0; k < 3; k++) nh[k] = DAG ? f2(-h.re[k].x, -h.re[k].y) : f2(-h.im[k].x, -h.im[k].y);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 re = f2b(0.f), im = f2b(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const cplx<float> e = DAG ? u.u[k][r] : u.u[r][k];
      const float2 ur = f2b(e.re), ui = f2b(e.im);
      re = fma2(ur, h.re[k], re);
      im = fma2(ur, h.im[k], im);
      if (DAG) {
        re = fma2(ui, h.im[k], re);
        im = fma2(ui, nh[k], im);
      } else {
        re = fma2(ui, nh[k], re);
        im = fma2(ui, h.re[k], im);
      }
    }
    o.re[r] = re;
    o.im[r] = im;
  }
  return o;
}

// Accumulator: the upper pair (spins 0,1), and the lower pair split into the
// terms that arrive in natural lane order (ln: spins 2,3) and swapped (ls:
// spins 3,2), merged once at the end.
struct AccX2 { float2 ure[3], uim[3], lnre[3], lnim[3], lsre[3], lsim[3]; };

__device__ __forceinline__ void zero_x2(AccX2 &a) {
#pragma unroll
  for (int c = 0; c < 3; c++) a.ure[c] = a.uim[c] = a.lnre[c] = a.lnim[c] = a.lsre[c] = a.lsim[c] = f2b(0.f);
}

// acc += f * (full spinor rebuilt from the multiplied half spinor h): the
// reconstruction of accum_reconstruct() in cpsb_device.cuh.
template <int MU> __device__ __forceinline__ void accum_x2(AccX2 &a, const HfX2 &h, float sg, float f) {
  const float s = f * sg;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    a.ure[c] = fma2(f2b(f), h.re[c], a.ure[c]);
    a.uim[c] = fma2(f2b(f), h.im[c], a.uim[c]);
    if (MU == 0) {         // psi2 += -i sg h1, psi3 += -i sg h0
      a.lsre[c] = fma2(f2b(s), h.im[c], a.lsre[c]);
      a.lsim[c] = fma2(f2b(-s), h.re[c], a.lsim[c]);
    } else if (MU == 1) {  // psi2 += sg h1, psi3 -= sg h0
      a.lsre[c] = fma2(f2(-s, s), h.re[c], a.lsre[c]);
      a.lsim[c] = fma2(f2(-s, s), h.im[c], a.lsim[c]);
    } else if (MU == 2) {  // psi2 += -i sg h0, psi3 += i sg h1
      a.lnre[c] = fma2(f2(s, -s), h.im[c], a.lnre[c]);
      a.lnim[c] = fma2(f2(-s, s), h.re[c], a.lnim[c]);
    } else {               // psi2 += sg h0, psi3 += sg h1
      a.lnre[c] = fma2(f2b(s), h.re[c], a.lnre[c]);
      a.lnim[c] = fma2(f2b(s), h.im[c], a.lnim[c]);
    }
  }
}

__device__ __forceinline__ SpX2 merge_x2(const AccX2 &a) {
  SpX2 o;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o.re[0][c] = a.ure[c];
    o.im[0][c] = a.uim[c];
    o.re[1][c] = add2(a.lnre[c], swp(a.lsre[c]));
    o.im[1][c] = add2(a.lnim[c], swp(a.lsim[c]));
  }
  return o;
}

// The recurrence scalars and the halting decision of one right-hand side once
// the new |r|^2 = c is known (cg_r_update of blas.cu; inv_cg.C:329-364).
__device__ __forceinline__ void cg_advance(CgState *S, int q, double c) {
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
  if (reason) {
    S->halt[q] = 1;
    S->reason[q] = reason;
  }
}

// ---------------------------------------------------------------- the kernel
// Shared-memory link table of a unit: for tile column xl and link j (0-3 the
// forward links at x, 4-7 the backward links at x - mu) the 9 elements, row
// major, 16 bytes each: (ur, ur, ui, ui) for FP32 / 16-bit, (ur, ui) doubles
// for FP64.  Columns are LSTR elements apart (72 + 1, so that the columns a
// warp reads fall in different banks).
constexpr int LSTR = 73;

// Dynamic shared memory of a launch: links (LC shapes only), neighbour column
// offsets and checkerboard indices, norm slots.
struct HopShm {
  size_t links, nbo, xn, norm, total;
};
__host__ __device__ inline HopShm hop_shm(int TX, int NT, int nrhs, bool red, bool lc) {
  HopShm s;
  s.links = 0;
  s.nbo = lc ? (size_t)TX * LSTR * 16 : 0;
  s.xn = s.nbo + (size_t)TX * 8 * sizeof(int);
  s.norm = s.xn + (size_t)TX * 8 * sizeof(int);
  s.norm = (s.norm + 15) & ~(size_t)15;
  s.total = s.norm + (red ? (size_t)NT * nrhs * sizeof(double) : 0);
  return s;
}

// Fills the unit's neighbour tables -- for column xl and neighbour j the
// offset of the neighbour column's first entry within one right-hand side and
// its checkerboard index -- and, with LC, the link table.
template <int P, bool LC>
__device__ __forceinline__ void load_unit(const DslashArgs &A, int tile, int k, int par_out, int TX, int NT,
                                          unsigned char *sh) {
  const Geom &g = A.g;
  const HopShm L = hop_shm(TX, NT, 0, false, LC);
  const int L4[4] = {g.lx, g.ly, g.lz, g.lt};
  const int C = g.cs[k];
  const unsigned kb = k ? (unsigned)g.kb1 : 0u;
  int *nbo = (int *)(sh + L.nbo);
  int *xns = (int *)(sh + L.xn);
  for (int it = threadIdx.x; it < TX * 8; it += NT) {
    const int xl = it % TX, j = it / TX;
    const int x = tile * TX + xl;
    if (x >= g.n4cb) continue;
    const Coord c = decode(g, x, par_out);
    int p[4] = {c.x, c.y, c.z, c.t};
    const int mu = j & 3;
    if (j < 4) p[mu] = (p[mu] + 1 == L4[mu]) ? 0 : p[mu] + 1;
    else p[mu] = (p[mu] == 0) ? L4[mu] - 1 : p[mu] - 1;
    const int xn = cbindex(g, p[0], p[1], p[2], p[3]);
    nbo[xl * 8 + j] = (int)(kb + (unsigned)xn * (unsigned)C);
    xns[xl * 8 + j] = xn;
    if (!LC) continue;
    // link j: forward U_mu(x) of parity par_out, backward U_mu(x - mu) of the other parity
    if constexpr (P == P64) {
      const Link<double> l = j < 4 ? load_link<P64>(A.U, par_out, mu, x) : load_link<P64>(A.U, 1 - par_out, mu, xn);
      double2 *d = (double2 *)(sh + L.links) + (xl * LSTR + j * 9);
#pragma unroll
      for (int e = 0; e < 9; e++) d[e] = make_double2(l.u[e / 3][e % 3].re, l.u[e / 3][e % 3].im);
    } else {
      const Link<float> l = j < 4 ? load_link<P>(A.U, par_out, mu, x) : load_link<P>(A.U, 1 - par_out, mu, xn);
      // reconstructed links omit the antiperiodic sign: fold it in here
      const bool flip = A.bc_t_sign < 0 && mu == 3 && (j < 4 ? c.t == g.lt - 1 : c.t == 0);
      const float sgn = flip ? -1.f : 1.f;
      float4 *d = (float4 *)(sh + L.links) + (xl * LSTR + j * 9);
#pragma unroll
      for (int e = 0; e < 9; e++) {
        const float ur = sgn * l.u[e / 3][e % 3].re, ui = sgn * l.u[e / 3][e % 3].im;
        d[e] = make_float4(ur, ur, ui, ui);
      }
    }
  }
}

// The tile processed as the u-th unit.  A tile is TX consecutive checkerboard
// sites; when it is a whole number of x-rows of one (z, t) plane, tiles are
// visited with t fastest, then z, then the block of rows, so a tile's t and z
// neighbours are processed by blocks resident at the same time (their shared
// input columns are read while in L2); otherwise in site order.
__device__ __forceinline__ int tile_order(const Geom &g, int u, int TX, int torder) {
  const int plane = g.lxh * g.ly;
  if (!torder || TX % g.lxh != 0 || plane % TX != 0) return u;
  const int nyb = plane / TX;
  const int t = u % g.lt, r = u / g.lt;
  const int z = r % g.lz, yb = r / g.lz;
  return yb + nyb * (z + g.lz * t);
}

// ---------------------------------------------------------------- one entry
// Per-entry context of the hop: the unit's link table column, the neighbour
// column offsets and checkerboard indices, and the 5th-direction neighbours.
struct HopCtx {
  const void *lk;
  int nb[8], xn[8];
  int par_out, x;
  bool flip_f, flip_b;
  unsigned e5m, e5p;
  double f5m, f5p;
};

// The hop of one FP64 entry (right-hand side at entry offset rb): the 8
// neighbours with links from the table (LC) or global memory, and with A.hop5
// the 5th-direction neighbours; no scaling.  L2ONLY: spinor loads bypass the
// read-only cache (the input was written earlier in the same launch).
template <int P, bool LC, bool DAG, int DEPTH, bool L2ONLY = false>
__device__ __forceinline__ Spinor<double> hop_entry_64(const DslashArgs &A, const HopCtx &hc, unsigned rb) {
  constexpr float sdag = DAG ? -1.f : 1.f;
  const void *lk = hc.lk;
  const int par_out = hc.par_out, x = hc.x;
  const double2 *l64 = (const double2 *)lk;
  Spinor<double> acc;
  zero(acc);
  // DEPTH: neighbours whose loads are in flight ahead of the one computed
  Raw<P64> nxt;
  if (DEPTH >= 1) nxt = load_raw64<L2ONLY>(A.in, rb + (unsigned)hc.nb[0]);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    Raw<P64> cur;
    if (DEPTH >= 1) {
      cur = nxt;
      if (j < 7) nxt = load_raw64<L2ONLY>(A.in, rb + (unsigned)hc.nb[j + 1]);
    } else {
      cur = load_raw64<L2ONLY>(A.in, rb + (unsigned)hc.nb[j]);
    }
    const int mu = j & 3;
    const double sg = j < 4 ? -(double)sdag : (double)sdag;
    const Half<double> h = project(unpack64(cur), mu, sg);
    Link<double> l;
    if (LC) {
#pragma unroll
      for (int e = 0; e < 9; e++) {
        const double2 v = l64[j * 9 + e];
        l.u[e / 3][e % 3] = mk(v.x, v.y);
      }
    } else {
      l = j < 4 ? load_link<P64>(A.U, par_out, mu, x) : load_link<P64>(A.U, 1 - par_out, mu, hc.xn[j]);
    }
    accum_reconstruct(acc, j < 4 ? umul(l, h) : umul_dag(l, h), mu, sg);
  }
  if (A.hop5) {
    // dwf_dslash_5_plus: upper (lower) chirality from s-1 (s+1) at dag 0, swapped at dag 1
    const double2 *bm = entry_ptr<12, const double2>(A.in.data, rb + hc.e5m);
    const double2 *bp = entry_ptr<12, const double2>(A.in.data, rb + hc.e5p);
    // chunks 0-5 are spins 0, 1 (the upper chirality), 6-11 spins 2, 3
    const int um = DAG ? 6 : 0, up = DAG ? 0 : 6;  // pair taken from s-1 / s+1
    double2 vm[6], vp[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
      vm[q] = L2ONLY ? __ldcg(bm + 8 * (um + q)) : __ldg(bm + 8 * (um + q));
      vp[q] = L2ONLY ? __ldcg(bp + 8 * (up + q)) : __ldg(bp + 8 * (up + q));
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const cplx<double> lo = cscale(hc.f5m, mk(vm[q].x, vm[q].y)), hi = cscale(hc.f5p, mk(vp[q].x, vp[q].y));
      cplx<double> &u = acc.c[q / 3][q % 3], &l = acc.c[2 + q / 3][q % 3];
      if (!DAG) {
        u = u + lo;
        l = l + hi;
      } else {
        l = l + lo;
        u = u + hi;
      }
    }
  }
  return acc;
}

// The same for FP32 / 16-bit storage in packed FP32x2 arithmetic.
template <int P, bool LC, bool DAG, int DEPTH>
__device__ __forceinline__ SpX2 hop_entry_x2(const DslashArgs &A, const HopCtx &hc, unsigned rb) {
  constexpr float sdag = DAG ? -1.f : 1.f;
  const void *lk = hc.lk;
  const int par_out = hc.par_out, x = hc.x;
  const float4 *l32 = (const float4 *)lk;
  AccX2 acc;
  zero_x2(acc);
  // DEPTH (1 or 2): neighbours whose loads are in flight ahead of the one computed
  Raw<P> nxt, nx2;
  nxt = load_raw<P>(A.in, rb + (unsigned)hc.nb[0]);
  if (DEPTH >= 2) nx2 = load_raw<P>(A.in, rb + (unsigned)hc.nb[1]);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const Raw<P> cur = nxt;
    if (DEPTH >= 2) {
      nxt = nx2;
      if (j < 6) nx2 = load_raw<P>(A.in, rb + (unsigned)hc.nb[j + 2]);
    } else if (j < 7) {
      nxt = load_raw<P>(A.in, rb + (unsigned)hc.nb[j + 1]);
    }
    float nrm;
    const float sg = j < 4 ? -sdag : sdag;
    // FP32: unpack, then project; 16-bit: project on the integers (iproject)
    SpX2 v;
    if constexpr (P == P32) v = unpack(cur, &nrm);
    else nrm = cur.nrm;
    const float4 *lj = l32 + j * 9;
    Link<float> lr;
    if (!LC) {
      lr = j < 4 ? load_link<P>(A.U, par_out, j & 3, x) : load_link<P>(A.U, 1 - par_out, j & 3, hc.xn[j]);
      if ((j == 3 && hc.flip_f) || (j == 7 && hc.flip_b)) nrm = -nrm;
    }
#define CPSB_NB(MU)                                                                            \
  {                                                                                            \
    HfX2 h;                                                                                    \
    if constexpr (P == P16) h = sg > 0.f ? iproject<MU, true>(cur) : iproject<MU, false>(cur); \
    else h = project_x2<MU>(v, sg);                                                            \
    const HfX2 uh = LC ? (j < 4 ? umul_x2<false>(lj, h) : umul_x2<true>(lj, h))                \
                       : (j < 4 ? umul_x2r<false>(lr, h) : umul_x2r<true>(lr, h));             \
    accum_x2<MU>(acc, uh, sg, nrm);                                                            \
  }
    switch (j & 3) {
      case 0: CPSB_NB(0) break;
      case 1: CPSB_NB(1) break;
      case 2: CPSB_NB(2) break;
      default: CPSB_NB(3) break;
    }
#undef CPSB_NB
  }
  if (A.hop5) {
    // upper pair from s-1 and lower from s+1 at dag 0 (swapped at dag 1),
    // scaled by 2 a5_inv or, across the walls, -2 m_f a5_inv
    const int pm = DAG ? 1 : 0;
    float nm, np;
    const HfX2 vm = load_pair<P>(A.in, rb + hc.e5m, pm, &nm);
    const HfX2 vp = load_pair<P>(A.in, rb + hc.e5p, 1 - pm, &np);
    const float2 cm = f2b((float)hc.f5m * nm), cp = f2b((float)hc.f5p * np);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!DAG) {
        acc.ure[c] = fma2(cm, vm.re[c], acc.ure[c]);
        acc.uim[c] = fma2(cm, vm.im[c], acc.uim[c]);
        acc.lnre[c] = fma2(cp, vp.re[c], acc.lnre[c]);
        acc.lnim[c] = fma2(cp, vp.im[c], acc.lnim[c]);
      } else {
        acc.lnre[c] = fma2(cm, vm.re[c], acc.lnre[c]);
        acc.lnim[c] = fma2(cm, vm.im[c], acc.lnim[c]);
        acc.ure[c] = fma2(cp, vp.re[c], acc.ure[c]);
        acc.uim[c] = fma2(cp, vp.im[c], acc.uim[c]);
      }
    }
  }
  return merge_x2(acc);
}

// The context of slice sp of tile column xl (checkerboard site x, class k)
// from the unit's tables.
template <int P, bool LC>
__device__ __forceinline__ void entry_ctx(HopCtx &hc, const DslashArgs &A, const unsigned char *dsh, const HopShm &L,
                                          int xl, int x, int k, int sp, int par_out) {
  const Geom &g = A.g;
  const int *nbo_sh = (const int *)(dsh + L.nbo);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    hc.nb[j] = nbo_sh[xl * 8 + j] + sp;
    hc.xn[j] = LC ? 0 : ((const int *)(dsh + L.xn))[xl * 8 + j];
  }
  hc.par_out = par_out;
  hc.x = x;
  // !LC: the antiperiodic sign of reconstructed links at the t boundary
  const Coord cx = decode(g, x, par_out);
  hc.flip_f = !LC && P != P64 && A.bc_t_sign < 0 && cx.t == g.lt - 1;
  hc.flip_b = !LC && P != P64 && A.bc_t_sign < 0 && cx.t == 0;
  // 5th-direction neighbours (DWF): slices s-1, s+1 of the same 4-D site
  const int s = g.ncls == 2 ? k + 2 * sp : sp;
  const int sm = s == 0 ? g.ls - 1 : s - 1, sq = s == g.ls - 1 ? 0 : s + 1;
  hc.e5m = site_entry(g, sm, x);
  hc.e5p = site_entry(g, sq, x);
  hc.f5m = s == 0 ? A.hop5_wall : A.hop5_fact;
  hc.f5p = s == g.ls - 1 ? A.hop5_wall : A.hop5_fact;
  hc.lk = dsh + L.links + (size_t)xl * LSTR * 16;
}

// LC: links from the unit's shared-memory table (otherwise each entry loads
// and reconstructs its own, which suits columns of one or two entries).
//
// Thread t of a block owns slice sp = t % C0 of column xl = t / (C0*RG) and
// the right-hand sides rl, rl + RG, ... with rl = (t / C0) % RG (A.rg, set by
// the launcher so that C0*RG lanes divide a warp: with DWF Ls 16 and 12
// right-hand sides a warp is one column x 8 slices x 4 right-hand sides, and
// every link read is a broadcast).  The grid holds no more blocks than are
// resident at once, so the units in flight are one contiguous run of tiles and
// their neighbour columns are read while they are in L2.
// CGR: 0 none, 1 the fused residual update r -= alpha A p, 2 the same for the
// shifted operator, r -= alpha (A p + shift p).
template <int P, int NT, int MINB, bool LC, bool XPAY, bool NORM, int CGR, bool DAG, int DEPTH>
__global__ void __launch_bounds__(NT, MINB) hop_kernel(DslashArgs A) {
  const Geom &g = A.g;
  extern __shared__ __align__(16) unsigned char dsh[];
  __shared__ double red[NT / 32];
  // alpha = |r|^2 / (<p, A p> + shift |p|^2) per right-hand side, once per block
  // (the loop over units starts with a barrier)
  __shared__ double cg_alpha[MAX_RHS];
  if (CGR && threadIdx.x < g.nrhs) {
    const CgState *S = A.cg;
    cg_alpha[threadIdx.x] = S->rr[threadIdx.x] / (S->d[threadIdx.x] + S->shift * S->pp[threadIdx.x]);
  }
  const int C0 = g.cs[0];
  const int RG = A.rg;
  const int TX = NT / (C0 * RG);
  const HopShm L = hop_shm(TX, NT, g.nrhs, NORM || CGR, LC);
  double *nrm_sh = (double *)(dsh + L.norm);
  if (NORM || CGR)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const int sp = threadIdx.x % C0;                 // slice index of the thread within its column
  const int rl = (threadIdx.x / C0) % RG;          // right-hand side within the group
  const int xl = threadIdx.x / (C0 * RG);          // column of the tile
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int ncls = g.ncls;
  // units: (group of A.rgroup right-hand sides, tile, class), the group slowest
  const int G = A.rgroup;
  const int per_group = ntiles * ncls;
  const int nunits = per_group * ((g.nrhs + G - 1) / G);
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    const int grp = unit / per_group, rem = unit - grp * per_group;
    const int k = rem % ncls, tile = tile_order(g, rem / ncls, TX, A.torder);
    const int par_out = A.five_d ? ((1 - A.cb + k) & 1) : 1 - A.cb;
    __syncthreads();  // the previous unit is done with the tables
    load_unit<P, LC>(A, tile, k, par_out, TX, NT, dsh);
    __syncthreads();
    const int x = tile * TX + xl;
    const int C = g.cs[k];
    if (xl >= TX || x >= g.n4cb || sp >= C) continue;
    HopCtx hc;
    entry_ctx<P, LC>(hc, A, dsh, L, xl, x, k, sp, par_out);
    const unsigned own = (k ? (unsigned)g.kb1 : 0u) + (unsigned)x * (unsigned)C + (unsigned)sp;
    const int rhs_end = min(g.nrhs, (grp + 1) * G);
    for (int rhs = grp * G + rl; rhs < rhs_end; rhs += RG) {
      if (A.skip && A.skip[rhs]) continue;
      const unsigned rb = (unsigned)rhs * per;
      const unsigned i = rb + own;
      if constexpr (P == P64) {
        // ------------------------------------------------ FP64
        Spinor<double> acc = hop_entry_64<P, LC, DAG, DEPTH>(A, hc, rb);
        const double a = A.a;
        if (XPAY) {
          const Spinor<double> xv = unpack64(load_raw<P64>(A.x, i));
#pragma unroll
          for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
            for (int r = 0; r < 3; r++) acc.c[s2][r] = xv.c[s2][r] + cscale(a, acc.c[s2][r]);
        } else if (a != 1.0) {
#pragma unroll
          for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
            for (int r = 0; r < 3; r++) acc.c[s2][r] = cscale(a, acc.c[s2][r]);
        }
        if (CGR) {
          const double alpha = cg_alpha[rhs];
          Spinor<double> rv = unpack64(load_raw<P64>(A.cg_r, i));
          if (CGR == 2 || A.cg_x.data) {
            const Spinor<double> pv = unpack64(load_raw<P64>(A.cg_p, i));
            if (CGR == 2) {
              const double sigma = A.cg->shift;
#pragma unroll
              for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
                for (int r = 0; r < 3; r++) acc.c[s2][r] = acc.c[s2][r] + cscale(sigma, pv.c[s2][r]);
            }
            if (A.cg_x.data) {
              // x += alpha p (the solution half of cg_xp_update, blas.cu)
              Spinor<double> xv = unpack64(load_raw<P64>(A.cg_x, i));
#pragma unroll
              for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
                for (int r = 0; r < 3; r++) xv.c[s2][r] = cscale(alpha, pv.c[s2][r]) + xv.c[s2][r];
              store_spinor<P64>(A.cg_x, i, xv);
            }
          }
#pragma unroll
          for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
            for (int r = 0; r < 3; r++) rv.c[s2][r] = rv.c[s2][r] - cscale(alpha, acc.c[s2][r]);
          store_spinor<P64>(A.cg_r, i, rv);
          nrm_sh[rhs * NT + threadIdx.x] += norm2(rv);
        } else {
          store_spinor<P64>(A.out, i, acc);
          if (NORM) nrm_sh[rhs * NT + threadIdx.x] += norm2(acc);
        }
      } else {
        // ------------------------------------------------ FP32 / 16-bit, packed
        SpX2 o = hop_entry_x2<P, LC, DAG, DEPTH>(A, hc, rb);
        const float2 a2 = f2b((float)A.a);
        if (XPAY) {
          float xn;
          const SpX2 xv = unpack(load_raw<P>(A.x, i), &xn);
#pragma unroll
          for (int p = 0; p < 2; p++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
              if (P == P16) {
                o.re[p][cc] = fma2(xv.re[p][cc], f2b(xn), mul2(a2, o.re[p][cc]));
                o.im[p][cc] = fma2(xv.im[p][cc], f2b(xn), mul2(a2, o.im[p][cc]));
              } else {
                o.re[p][cc] = fma2(a2, o.re[p][cc], xv.re[p][cc]);
                o.im[p][cc] = fma2(a2, o.im[p][cc], xv.im[p][cc]);
              }
            }
        } else if (A.a != 1.0) {
#pragma unroll
          for (int p = 0; p < 2; p++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
              o.re[p][cc] = mul2(a2, o.re[p][cc]);
              o.im[p][cc] = mul2(a2, o.im[p][cc]);
            }
        }
        if (CGR) {
          // r -= alpha (A p + shift p), A p = o in registers (cg_r_update of blas.cu)
          const float alpha = (float)cg_alpha[rhs];
          float rn;
          SpX2 rv = unpack(load_raw<P>(A.cg_r, i), &rn);
          float pn = 0.f;
          SpX2 pv;
          double sigma = 0.0;
          if (CGR == 2 || A.cg_x.data) pv = unpack(load_raw<P>(A.cg_p, i), &pn);
          if (CGR == 2) sigma = A.cg->shift;
          if (A.cg_x.data) {
            // x += alpha p in FP32 (the solution half of cg_xp_update, blas.cu)
            float xn;
            SpX2 xv = unpack(load_raw<P32>(A.cg_x, i), &xn);
            const float2 ap = f2b(alpha * pn);
#pragma unroll
            for (int p = 0; p < 2; p++)
#pragma unroll
              for (int cc = 0; cc < 3; cc++) {
                xv.re[p][cc] = fma2(ap, pv.re[p][cc], xv.re[p][cc]);
                xv.im[p][cc] = fma2(ap, pv.im[p][cc], xv.im[p][cc]);
              }
            store_x2<P32>(A.cg_x, i, xv);
          }
          const float2 ma = f2b(-alpha), rs = f2b(rn), ps = f2b((float)sigma * pn);
#pragma unroll
          for (int p = 0; p < 2; p++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
              float2 are = o.re[p][cc], aim = o.im[p][cc];
              if (CGR == 2) {
                are = fma2(ps, pv.re[p][cc], are);
                aim = fma2(ps, pv.im[p][cc], aim);
              }
              rv.re[p][cc] = fma2(ma, are, P == P16 ? mul2(rv.re[p][cc], rs) : rv.re[p][cc]);
              rv.im[p][cc] = fma2(ma, aim, P == P16 ? mul2(rv.im[p][cc], rs) : rv.im[p][cc]);
            }
          nrm_sh[rhs * NT + threadIdx.x] += store_x2<P>(A.cg_r, i, rv);
        } else {
          const double n2 = store_x2<P>(A.out, i, o);
          if (NORM) nrm_sh[rhs * NT + threadIdx.x] += n2;
        }
      }
    }
  }
  if (NORM || CGR) {
    for (int q = 0; q < g.nrhs; q++) {
      const double bs = block_sum<NT>(nrm_sh[q * NT + threadIdx.x], red);
      if (threadIdx.x == 0) A.red.partial[q * gridDim.x + blockIdx.x] = bs;
    }
    if (last_block(A.red.ticket, gridDim.x)) {
      for (int q = 0; q < g.nrhs; q++) {
        const double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) {
          if (!CGR) {
            A.red.result[q] = t;
          } else {
            cg_advance(A.cg, q, t);
            if (A.red.result) A.red.result[q] = t;
          }
        }
        __syncthreads();
      }
    }
  }
}

// ---------------------------------------------------------------- direction-parallel FP64 hop
// For lattices too small to fill the GPU with one thread per entry (Wilson 8^4:
// 2048 entries per checkerboard), eight consecutive lanes share an entry: lane
// d takes neighbour d (0-3 forward, 4-7 backward) -- one spinor and one link
// load each, all eight in flight at once instead of one after another -- and
// lanes 0 and 1 load the two 5th-direction terms.  Lane 0 then gathers the
// eight partial spinors through shared memory and sums them in direction order,
// adds the 5th-direction terms last and runs the epilogue of hop_kernel: the
// same operations in the same order as hop_entry_64, so every launch shape
// gives the same bits.  Every warp runs the same number of rounds, so the
// shuffles always have all 32 lanes.
template <int NT, bool XPAY, bool NORM, int CGR, bool DAG>
__global__ void __launch_bounds__(NT) hop8_kernel(DslashArgs A) {
  const Geom &g = A.g;
  extern __shared__ __align__(16) unsigned char dsh[];
  __shared__ double red[NT / 32];
  __shared__ double cg_alpha[MAX_RHS];
  double2 *gsh = (double2 *)dsh;                        // 12 x NT partial-spinor slots
  double *nrm_sh = (double *)(dsh + (size_t)12 * NT * sizeof(double2));
  if (CGR && threadIdx.x < g.nrhs) {
    const CgState *S = A.cg;
    cg_alpha[threadIdx.x] = S->rr[threadIdx.x] / (S->d[threadIdx.x] + S->shift * S->pp[threadIdx.x]);
  }
  if (NORM || CGR)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  __syncthreads();
  constexpr double sdag = DAG ? -1.0 : 1.0;
  const int d = threadIdx.x & 7;
  const int lane = threadIdx.x & 31;
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  const long wstride = (long)gridDim.x * (NT / 32) * 4;
  // right-hand sides one after another, each spread over the grid the same way
  // whatever their number (so a right-hand side's reductions do not depend on it)
  for (int q = 0; q < g.nrhs; q++)
  for (long e0 = ((long)blockIdx.x * (NT / 32) + threadIdx.x / 32) * 4; e0 < (long)per; e0 += wstride) {
    const long e = e0 + (lane >> 3);
    const bool valid = e < (long)per && !(A.skip && A.skip[q]);
    Spinor<double> acc;
    zero(acc);
    double2 v5[6];  // lane 0: the pair from slice s-1, lane 1: from s+1
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
      const Raw<P64> nr = load_raw<P64>(A.in, ni);
      if (A.hop5 && d < 2) {
        // dwf_dslash_5_plus: upper (lower) chirality from s-1 (s+1) at dag 0, swapped at dag 1
        const int sn = d == 0 ? (s == 0 ? g.ls - 1 : s - 1) : (s == g.ls - 1 ? 0 : s + 1);
        const int chunk0 = (d == 0) != DAG ? 0 : 6;
        const double2 *b = entry_ptr<12, const double2>(A.in.data, rb + site_entry(g, sn, x));
#pragma unroll
        for (int qq = 0; qq < 6; qq++) v5[qq] = __ldg(b + 8 * (chunk0 + qq));
        f5m = s == 0 ? A.hop5_wall : A.hop5_fact;
        f5p = s == g.ls - 1 ? A.hop5_wall : A.hop5_fact;
      }
      const Link<double> l = d < 4 ? load_link<P64>(A.U, par_out, mu, x) : load_link<P64>(A.U, 1 - par_out, mu, xn);
      const Half<double> h = project(unpack64(nr), mu, sg);
      switch (mu) {  // accum_reconstruct with a compile-time direction
        case 0: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 0, sg); break;
        case 1: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 1, sg); break;
        case 2: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 2, sg); break;
        default: accum_reconstruct(acc, d < 4 ? umul(l, h) : umul_dag(l, h), 3, sg); break;
      }
    }
    // lane 0 sums the eight partial spinors in direction order, as hop_entry_64,
    // reading them from shared memory (component-major slots: conflict-free)
    const int base = lane & ~7;
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
    __syncwarp();  // the slots are written again in the next round
    double2 vp[6];  // lane 1's pair, for lane 0
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
    const double a = A.a;
    if (XPAY) {
      const Spinor<double> xv = unpack64(load_raw<P64>(A.x, i));
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = xv.c[s2][r] + cscale(a, acc.c[s2][r]);
    } else if (a != 1.0) {
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) acc.c[s2][r] = cscale(a, acc.c[s2][r]);
    }
    if (CGR) {
      const double alpha = cg_alpha[q];
      Spinor<double> rv = unpack64(load_raw<P64>(A.cg_r, i));
      if (CGR == 2 || A.cg_x.data) {
        const Spinor<double> pv = unpack64(load_raw<P64>(A.cg_p, i));
        if (CGR == 2) {
          const double sigma = A.cg->shift;
#pragma unroll
          for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
            for (int r = 0; r < 3; r++) acc.c[s2][r] = acc.c[s2][r] + cscale(sigma, pv.c[s2][r]);
        }
        if (A.cg_x.data) {
          Spinor<double> xv = unpack64(load_raw<P64>(A.cg_x, i));
#pragma unroll
          for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
            for (int r = 0; r < 3; r++) xv.c[s2][r] = cscale(alpha, pv.c[s2][r]) + xv.c[s2][r];
          store_spinor<P64>(A.cg_x, i, xv);
        }
      }
#pragma unroll
      for (int s2 = 0; s2 < 4; s2++)
#pragma unroll
        for (int r = 0; r < 3; r++) rv.c[s2][r] = rv.c[s2][r] - cscale(alpha, acc.c[s2][r]);
      store_spinor<P64>(A.cg_r, i, rv);
      nrm_sh[q * NT + threadIdx.x] += norm2(rv);
    } else {
      store_spinor<P64>(A.out, i, acc);
      if (NORM) nrm_sh[q * NT + threadIdx.x] += norm2(acc);
    }
  }
  if (NORM || CGR) {
    for (int q = 0; q < g.nrhs; q++) {
      const double bs = block_sum<NT>(nrm_sh[q * NT + threadIdx.x], red);
      if (threadIdx.x == 0) A.red.partial[q * gridDim.x + blockIdx.x] = bs;
    }
    if (last_block(A.red.ticket, gridDim.x)) {
      for (int q = 0; q < g.nrhs; q++) {
        const double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) {
          if (!CGR) {
            A.red.result[q] = t;
          } else {
            cg_advance(A.cg, q, t);
            if (A.red.result) A.red.result[q] = t;
          }
        }
        __syncthreads();
      }
    }
  }
}

// Blocks of a kernel that fit on the device at once with this dynamic shared
// memory (at least 1, at most the 148*16 partial slots of a reduction).
static int resident_blocks(const void *fn, int nt, size_t shm) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, int, size_t, int>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 148;
  }
  const auto key = std::make_tuple(fn, nt, shm, dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int nsm = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, shm) != cudaSuccess) {
    cudaGetLastError();
    return 148;
  }
  int n = nsm * (per_sm > 0 ? per_sm : 1);
  n = n < 148 * 16 ? n : 148 * 16;
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = n;
  return n;
}

// One launch shape: NT threads, at least MINB resident blocks per SM, link
// table (LC), right-hand-side grouping (GRP: as many right-hand sides per warp
// as divide it, else one).  The fused residual update (A.cg) needs the xpay
// form.
template <int P, int NT, int MINB, bool LC, bool GRP, int DEPTH>
static cudaError_t hop_launch_v(DslashArgs A, int xpay, int norm, cudaStream_t st, int rgroup, int torder) {
  const int C0 = A.g.cs[0];
  if (C0 < 1 || C0 > NT) return cudaErrorNotSupported;
  int rg = 1;
  if (GRP)
    while (rg * 2 <= A.g.nrhs && C0 * rg * 2 <= 32 && 32 % (C0 * rg * 2) == 0) rg *= 2;
  if (GRP && rg == 1) return cudaErrorNotSupported;  // the same as the ungrouped shape
  A.rg = rg;
  A.torder = torder;
  // right-hand sides per unit: all, or groups of rgroup (a multiple of rg), so
  // that the blocks resident at one time touch only a few right-hand sides
  A.rgroup = rgroup > 0 ? std::max(rg, rgroup / rg * rg) : A.g.nrhs;
  if (rgroup > 0 && A.rgroup >= A.g.nrhs) return cudaErrorNotSupported;  // the same as all
  const int TX = NT / (C0 * rg);
  if (TX < 1 || (LC && TX > 32)) return cudaErrorNotSupported;  // link tables of more than 32 columns: use !LC
  const bool cgr = A.cg != nullptr;
  if (cgr && !xpay) return cudaErrorInvalidValue;
  const HopShm L = hop_shm(TX, NT, A.g.nrhs, norm || cgr, LC);
  if (L.total > 200 * 1024) return cudaErrorNotSupported;
  const long units = (long)((A.g.n4cb + TX - 1) / TX) * A.g.ncls * ((A.g.nrhs + A.rgroup - 1) / A.rgroup);
  // the opt-in above the 48 KB default is set once per instantiation
  auto opt_in = [&](const void *f, bool &done) -> cudaError_t {
    if (done || L.total + 1024 <= 48 * 1024) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) done = true;
    return e;
  };
  cudaError_t e = cudaSuccess;
#define CPSB_HOP(XP, NR, CG, D)                                                            \
  {                                                                                        \
    const void *fn = (const void *)hop_kernel<P, NT, MINB, LC, XP, NR, CG, D, DEPTH>;             \
    static bool done = false;                                                              \
    e = opt_in(fn, done);                                                                  \
    if (e != cudaSuccess) return e;                                                        \
    const long nb = std::min(units, (long)resident_blocks(fn, NT, L.total));                \
    hop_kernel<P, NT, MINB, LC, XP, NR, CG, D, DEPTH><<<(unsigned)nb, NT, L.total, st>>>(A);      \
  }
#define CPSB_HOP_D(XP, NR, CG)          \
  if (A.dag) CPSB_HOP(XP, NR, CG, true) \
  else CPSB_HOP(XP, NR, CG, false)
  if (cgr && A.cg_shift) CPSB_HOP_D(true, false, 2)
  else if (cgr) CPSB_HOP_D(true, false, 1)
  else if (xpay && norm) CPSB_HOP_D(true, true, 0)
  else if (xpay) CPSB_HOP_D(true, false, 0)
  else if (norm) CPSB_HOP_D(false, true, 0)
  else CPSB_HOP_D(false, false, 0)
#undef CPSB_HOP_D
#undef CPSB_HOP
  return launched();
}

// The direction-parallel FP64 hop: eight lanes per entry, the grid no larger
// than the blocks resident at once.
template <int NT>
static cudaError_t hop8_launch(const DslashArgs &A, int xpay, int norm, cudaStream_t st) {
  const bool cgr = A.cg != nullptr;
  if (cgr && !xpay) return cudaErrorInvalidValue;
  const size_t shm = (size_t)12 * NT * sizeof(double2) + ((norm || cgr) ? (size_t)NT * A.g.nrhs * sizeof(double) : 0);
  const long entries = (long)A.g.n4cb * A.g.ls;  // of one right-hand side
  const long want = (entries + NT / 8 - 1) / (NT / 8);
#define CPSB_HOP8(XP, NR, CG, D)                                                   \
  {                                                                                \
    const void *fn = (const void *)hop8_kernel<NT, XP, NR, CG, D>;                 \
    const long nb = std::min(want, (long)resident_blocks(fn, NT, shm));            \
    hop8_kernel<NT, XP, NR, CG, D><<<(unsigned)nb, NT, shm, st>>>(A);              \
  }
#define CPSB_HOP8_D(XP, NR, CG)          \
  if (A.dag) CPSB_HOP8(XP, NR, CG, true) \
  else CPSB_HOP8(XP, NR, CG, false)
  if (cgr && A.cg_shift) CPSB_HOP8_D(true, false, 2)
  else if (cgr) CPSB_HOP8_D(true, false, 1)
  else if (xpay && norm) CPSB_HOP8_D(true, true, 0)
  else if (xpay) CPSB_HOP8_D(true, false, 0)
  else if (norm) CPSB_HOP8_D(false, true, 0)
  else CPSB_HOP8_D(false, false, 0)
#undef CPSB_HOP8_D
#undef CPSB_HOP8
  return launched();
}

// Launch shapes the autotuner chooses from: (threads, min blocks per SM, link
// table, right-hand-side grouping).  Shapes with link tables need columns of at
// least NT/32 entries (DWF, Mobius); shape 4 serves short columns (Wilson).
template <int P>
static cudaError_t hop_launch_p(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  switch (variant) {
    // (threads, blocks per SM, link table, RHS per warp lane group, prefetch
    // depth; RHS per unit, t-fastest tile order).  FP64 keeps fewer blocks
    // (more registers) and one neighbour less in flight.
    case 0: return hop_launch_v<P, 128, P == P64 ? 2 : 4, true, false, P == P64 ? 1 : 2>(A, xpay, norm, st, 0, 0);
    case 1: return hop_launch_v<P, 128, P == P64 ? 3 : 5, true, false, P == P64 ? 1 : 2>(A, xpay, norm, st, 0, 0);
    case 2: return hop_launch_v<P, 256, P == P64 ? 1 : 2, true, false, P == P64 ? 1 : 2>(A, xpay, norm, st, 0, 0);
    case 3: return hop_launch_v<P, 256, P == P64 ? 1 : 2, true, false, P == P64 ? 1 : 2>(A, xpay, norm, st, 0, 1);
    case 4: return hop_launch_v<P, 128, P == P64 ? 2 : 4, false, false, P == P64 ? 1 : 2>(A, xpay, norm, st, 0, 0);
    case 5: return hop_launch_v<P, 128, P == P64 ? 3 : 5, true, false, P == P64 ? 0 : 1>(A, xpay, norm, st, 0, 0);
    case 6: return hop_launch_v<P, 128, P == P64 ? 4 : 6, true, false, P == P64 ? 0 : 1>(A, xpay, norm, st, 0, 0);
    case 7: return hop_launch_v<P, 256, P == P64 ? 1 : 2, true, true, P == P64 ? 1 : 2>(A, xpay, norm, st, 4, 0);
    // FP64: eight lanes per entry, one neighbour each (small lattices)
    case 8:
      if constexpr (P == P64) return hop8_launch<128>(A, xpay, norm, st);
      else return cudaErrorNotSupported;
    default: return cudaErrorNotSupported;
  }
}

}  // namespace cpsb

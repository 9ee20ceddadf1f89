// dslash_x2.cuh -- FP32 / 16-bit Wilson and domain-wall hopping kernels written
// in Blackwell's packed FP32x2 arithmetic (FFMA2 / FADD2 / FMUL2).
//
// The operator is the one of dslash_impl.cuh (CPS wilson_dslash,
// cps_pp/src/util/dirac_op/d_op_wilson/noarch/wilson_dslash.C:173-516, with the
// DWF 5-D checkerboard of dwf_dslash_4.C:107-112 and the 5th-direction hop of
// dwf_dslash_5_plus.C:111-340), evaluated two spin components at a time: the
// spin-paired storage (cpsb_device.cuh) puts spins (2p, 2p+1) of one colour in
// the two lanes of a float2, and every step of the hop -- projection, link
// multiplication, re-expansion -- applies the same arithmetic to both spins of
// a pair, so each packed instruction does two scalar FMAs.
//
// 16-bit storage: the site's quantum is not applied when the fixed-point
// words are decoded; the hop is linear, so the quantum of each neighbour is
// folded into the factor with which its multiplied half spinor is accumulated
// (an FMA that is needed anyway).  Encoding uses the 1.5*2^23 rounding
// constant: v*scale + (1.5*2^23 + 2^15) rounds v*scale to the nearest integer
// in the low mantissa bits, whose low 16 bits are then the biased value.
#pragma once
#include "cpsb_device.cuh"
#include "cg_state.h"
#include "cpsb_kernels.h"

namespace cpsb {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2b(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 swp(float2 a) { return make_float2(a.y, a.x); }

// A spinor as two spin pairs: re[p][c] = (Re psi_{2p,c}, Re psi_{2p+1,c}).
struct SpX2 { float2 re[2][3], im[2][3]; };
// A half spinor (spins h0, h1 in the lanes) per colour.
struct HfX2 { float2 re[3], im[3]; };
// A link with every element broadcast to both lanes: e[r][c] = (ur, ur, ui, ui).
struct LkB { float4 e[3][3]; };

// Two biased 16-bit values of one word as a float2 of exact integers in [-32767, 32767].
__device__ __forceinline__ float2 dec16x2(unsigned w) {
  return add2(f2(__int_as_float((int)__byte_perm(w, 0x4B00u, 0x5410u)),
                 __int_as_float((int)__byte_perm(w, 0x4B00u, 0x5432u))),
              f2b(-8421376.0f));
}
// Biased 16-bit encodings of round(v.x*scale), round(v.y*scale) packed in one word
// (|v|*scale <= 32767 by construction of scale, so no clamp is needed).
__device__ __forceinline__ unsigned enc16x2p(float2 v, float2 scale) {
  const float2 r = fma2(v, scale, f2b(12615680.0f));  // 1.5*2^23 + 2^15
  return __byte_perm(__float_as_uint(r.x), __float_as_uint(r.y), 0x5410u);
}

// Loads a site; for 16-bit storage the values are the raw integers and *nrm the
// quantum, for FP32 *nrm = 1.
template <int P> __device__ __forceinline__ SpX2 load_x2(const SpinorPtr &f, long i, float *nrm);

template <> __device__ __forceinline__ SpX2 load_x2<P32>(const SpinorPtr &f, long i, float *nrm) {
  const float4 *b = (const float4 *)f.data;
  SpX2 s;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float4 v = __ldg(b + k * f.stride + i);
    s.re[k / 3][k % 3] = f2(v.x, v.y);
    s.im[k / 3][k % 3] = f2(v.z, v.w);
  }
  *nrm = 1.0f;
  return s;
}

template <> __device__ __forceinline__ SpX2 load_x2<P16>(const SpinorPtr &f, long i, float *nrm) {
  const uint4 *b = (const uint4 *)f.data;
  SpX2 s;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint4 v = __ldg(b + k * f.stride + i);
    const int pa = 2 * k, pb = 2 * k + 1;  // (3p + c) of the two complex values
    s.re[pa / 3][pa % 3] = dec16x2(v.x);
    s.im[pa / 3][pa % 3] = dec16x2(v.y);
    s.re[pb / 3][pb % 3] = dec16x2(v.z);
    s.im[pb / 3][pb % 3] = dec16x2(v.w);
  }
  *nrm = __ldg(f.norm + i);
  return s;
}

// Loads one spin pair (p = 0: spins 0,1, the upper chirality; p = 1: spins 2,3).
template <int P> __device__ __forceinline__ HfX2 load_pair_x2(const SpinorPtr &f, long i, int p, float *nrm);

template <> __device__ __forceinline__ HfX2 load_pair_x2<P32>(const SpinorPtr &f, long i, int p, float *nrm) {
  const float4 *b = (const float4 *)f.data;
  HfX2 h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float4 v = __ldg(b + (3 * p + c) * f.stride + i);
    h.re[c] = f2(v.x, v.y);
    h.im[c] = f2(v.z, v.w);
  }
  *nrm = 1.0f;
  return h;
}

// Pair 0 occupies words 0..5 (chunk 0 and the low half of chunk 1), pair 1
// words 6..11 (the high half of chunk 1 and chunk 2).
template <> __device__ __forceinline__ HfX2 load_pair_x2<P16>(const SpinorPtr &f, long i, int p, float *nrm) {
  const uint4 *b = (const uint4 *)f.data;
  const uint2 *mid = (const uint2 *)(b + f.stride + i) + p;
  const uint4 v = __ldg(b + (p ? 2 : 0) * f.stride + i);
  const uint2 m = __ldg(mid);
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

// Stores a site and returns |stored value|^2 (for 16-bit storage the norm of
// the rounded value that a later load returns).  The squares are summed in
// FP32 (components of magnitude 1e-19 .. 1e19); the quantum's square is
// applied in FP64 since it can lie below the FP32 range.
template <int P> __device__ __forceinline__ double store_x2(const SpinorPtr &f, long i, const SpX2 &s);

template <> __device__ __forceinline__ double store_x2<P32>(const SpinorPtr &f, long i, const SpX2 &s) {
  float4 *b = (float4 *)f.data;
  float2 n = f2b(0.f);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const float2 re = s.re[k / 3][k % 3], im = s.im[k / 3][k % 3];
    b[k * f.stride + i] = make_float4(re.x, re.y, im.x, im.y);
    n = fma2(re, re, n);
    n = fma2(im, im, n);
  }
  return (double)(n.x + n.y);
}

template <> __device__ __forceinline__ double store_x2<P16>(const SpinorPtr &f, long i, const SpX2 &s) {
  float m = 0.f;
#pragma unroll
  for (int p = 0; p < 2; p++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      m = fmaxf(fmaxf(m, fmaxf(fabsf(s.re[p][c].x), fabsf(s.re[p][c].y))),
                fmaxf(fabsf(s.im[p][c].x), fabsf(s.im[p][c].y)));
  const float scale = m > 0.f ? 32767.0f / m : 0.f;
  const float q = m * (1.0f / 32767.0f);
  f.norm[i] = q;
  const float2 sc = f2b(scale);
  uint4 *b = (uint4 *)f.data;
  float2 n = f2b(0.f);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int pa = 2 * k, pb = 2 * k + 1;
    unsigned w[4];
    w[0] = enc16x2p(s.re[pa / 3][pa % 3], sc);
    w[1] = enc16x2p(s.im[pa / 3][pa % 3], sc);
    w[2] = enc16x2p(s.re[pb / 3][pb % 3], sc);
    w[3] = enc16x2p(s.im[pb / 3][pb % 3], sc);
    b[k * f.stride + i] = make_uint4(w[0], w[1], w[2], w[3]);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 d = dec16x2(w[j]);
      n = fma2(d, d, n);
    }
  }
  return (double)(n.x + n.y) * ((double)q * q);
}

// (1 + sg*gamma_mu) psi -> half spinor (h0, h1) in the lanes; the gamma
// matrices are those of project() in cpsb_device.cuh written per spin pair:
// X[1] is (psi2, psi3) and swp(X[1]) is (psi3, psi2).
template <int MU> __device__ __forceinline__ HfX2 project_x2(const SpX2 &s, float sg) {
  HfX2 h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (MU == 0) {         // h0 = psi0 + i sg psi3, h1 = psi1 + i sg psi2
      h.re[c] = fma2(f2b(-sg), swp(s.im[1][c]), s.re[0][c]);
      h.im[c] = fma2(f2b(sg), swp(s.re[1][c]), s.im[0][c]);
    } else if (MU == 1) {  // h0 = psi0 - sg psi3, h1 = psi1 + sg psi2
      h.re[c] = fma2(f2(-sg, sg), swp(s.re[1][c]), s.re[0][c]);
      h.im[c] = fma2(f2(-sg, sg), swp(s.im[1][c]), s.im[0][c]);
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

// U h (DAG = false) or U^dag h (DAG = true) for both spins of the half spinor.
template <bool DAG> __device__ __forceinline__ HfX2 umul_x2(const LkB &u, const HfX2 &h) {
  HfX2 o;
  float2 nh[3];
#pragma unroll
  for (int k = 0; k < 3; k++) nh[k] = DAG ? f2(-h.re[k].x, -h.re[k].y) : f2(-h.im[k].x, -h.im[k].y);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 re = f2b(0.f), im = f2b(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float4 e = DAG ? u.e[k][r] : u.e[r][k];
      const float2 ur = f2(e.x, e.y), ui = f2(e.z, e.w);
      re = fma2(ur, h.re[k], re);
      im = fma2(ur, h.im[k], im);
      if (DAG) {  // conj(u) h: re += ui*Im h, im -= ui*Re h
        re = fma2(ui, h.im[k], re);
        im = fma2(ui, nh[k], im);
      } else {    // u h: re -= ui*Im h, im += ui*Re h
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
// terms that arrive in natural lane order (ln: spins 2,3) and those that
// arrive swapped (ls: spins 3,2), merged once at the end.
struct AccX2 { float2 ure[3], uim[3], lnre[3], lnim[3], lsre[3], lsim[3]; };

__device__ __forceinline__ void zero_x2(AccX2 &a) {
#pragma unroll
  for (int c = 0; c < 3; c++)
    a.ure[c] = a.uim[c] = a.lnre[c] = a.lnim[c] = a.lsre[c] = a.lsim[c] = f2b(0.f);
}

// acc += f * (full spinor rebuilt from the multiplied half spinor h), the
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

__device__ __forceinline__ LkB broadcast_link(const Link<float> &l) {
  LkB b;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) b.e[r][c] = make_float4(l.u[r][c].re, l.u[r][c].re, l.u[r][c].im, l.u[r][c].im);
  return b;
}

// Shared-memory link cache of a tile (see dslash_impl.cuh), holding broadcast links.
struct LinkCacheX2 {
  float4 *sh;  // [(pidx*8 + j)*9 + k][TX]
  int TX;
  __device__ __forceinline__ void put(int pidx, int j, int xi, const LkB &l) {
#pragma unroll
    for (int k = 0; k < 9; k++) sh[((pidx * 8 + j) * 9 + k) * TX + xi] = l.e[k / 3][k % 3];
  }
  __device__ __forceinline__ LkB get(int pidx, int j, int xi) const {
    LkB l;
#pragma unroll
    for (int k = 0; k < 9; k++) l.e[k / 3][k % 3] = sh[((pidx * 8 + j) * 9 + k) * TX + xi];
    return l;
  }
};

template <int P, bool LC>
__device__ __forceinline__ void hop_site_x2(const DslashArgs &A, int x, int xi, int par_out, int pidx, long sbase,
                                            const LinkCacheX2 &lc, AccX2 &acc) {
  const Geom &g = A.g;
  const int par_in = 1 - par_out;
  const float sdag = A.dag ? -1.f : 1.f;
  const Coord c = decode(g, x, par_out);
  const int L[4] = {g.lx, g.ly, g.lz, g.lt};
  const bool flip_f = A.bc_t_sign < 0 && c.t == g.lt - 1;
  const bool flip_b = A.bc_t_sign < 0 && c.t == 0;
  zero_x2(acc);
#define CPSB_FWD(MU)                                                                        \
  {                                                                                         \
    int p[4] = {c.x, c.y, c.z, c.t};                                                        \
    p[MU] = (p[MU] + 1 == L[MU]) ? 0 : p[MU] + 1;                                           \
    float nrm;                                                                              \
    const SpX2 v = load_x2<P>(A.in, sbase + cbindex(g, p[0], p[1], p[2], p[3]), &nrm);      \
    const HfX2 h = project_x2<MU>(v, -sdag);                                                \
    const LkB l = LC ? lc.get(pidx, MU, xi) : broadcast_link(load_link<P>(A.U, par_out, MU, x)); \
    const HfX2 uh = umul_x2<false>(l, h);                                                   \
    accum_x2<MU>(acc, uh, -sdag, (MU == 3 && flip_f) ? -nrm : nrm);                         \
  }
#define CPSB_BWD(MU)                                                                        \
  {                                                                                         \
    int p[4] = {c.x, c.y, c.z, c.t};                                                        \
    p[MU] = (p[MU] == 0) ? L[MU] - 1 : p[MU] - 1;                                           \
    const int xb = cbindex(g, p[0], p[1], p[2], p[3]);                                      \
    float nrm;                                                                              \
    const SpX2 v = load_x2<P>(A.in, sbase + xb, &nrm);                                      \
    const HfX2 h = project_x2<MU>(v, sdag);                                                 \
    const LkB l = LC ? lc.get(pidx, 4 + MU, xi) : broadcast_link(load_link<P>(A.U, par_in, MU, xb)); \
    const HfX2 uh = umul_x2<true>(l, h);                                                    \
    accum_x2<MU>(acc, uh, sdag, (MU == 3 && flip_b) ? -nrm : nrm);                          \
  }
  CPSB_FWD(0) CPSB_FWD(1) CPSB_FWD(2) CPSB_FWD(3)
  CPSB_BWD(0) CPSB_BWD(1) CPSB_BWD(2) CPSB_BWD(3)
#undef CPSB_FWD
#undef CPSB_BWD
}

// 5th-direction hop of dwf_dslash_5_plus: for dag = 0 the upper pair comes
// from s-1 and the lower from s+1 (swapped for dag = 1), scaled by 2*a5_inv
// or, across the walls, by -2*m_f*a5_inv.  Only the pair that is used is loaded.
template <int P>
__device__ __forceinline__ void hop5_x2(const DslashArgs &A, int x, int s, long rbase, AccX2 &acc) {
  const Geom &g = A.g;
  const int ls = g.ls;
  const int sm = (s == 0) ? ls - 1 : s - 1;
  const int sp = (s == ls - 1) ? 0 : s + 1;
  const float fm = (float)((s == 0) ? A.hop5_wall : A.hop5_fact);
  const float fp = (float)((s == ls - 1) ? A.hop5_wall : A.hop5_fact);
  const int pm = A.dag ? 1 : 0;  // pair taken from s-1
  float nm, np;
  const HfX2 vm = load_pair_x2<P>(A.in, rbase + (long)sm * g.n4cb + x, pm, &nm);
  const HfX2 vp = load_pair_x2<P>(A.in, rbase + (long)sp * g.n4cb + x, 1 - pm, &np);
  const float2 cm = f2b(fm * nm), cp = f2b(fp * np);
  float2 *up_re = acc.ure, *up_im = acc.uim, *lo_re = acc.lnre, *lo_im = acc.lnim;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (!A.dag) {
      up_re[c] = fma2(cm, vm.re[c], up_re[c]);
      up_im[c] = fma2(cm, vm.im[c], up_im[c]);
      lo_re[c] = fma2(cp, vp.re[c], lo_re[c]);
      lo_im[c] = fma2(cp, vp.im[c], lo_im[c]);
    } else {
      lo_re[c] = fma2(cm, vm.re[c], lo_re[c]);
      lo_im[c] = fma2(cm, vm.im[c], lo_im[c]);
      up_re[c] = fma2(cp, vp.re[c], up_re[c]);
      up_im[c] = fma2(cp, vp.im[c], up_im[c]);
    }
  }
}

// Same tiling, link cache and epilogues as dslash_kernel in dslash_impl.cuh.
template <int P, int NT, int MINB, bool LC, bool XPAY, bool NORM>
__global__ void __launch_bounds__(NT, MINB) dslash_x2_kernel(DslashArgs A) {
  const Geom &g = A.g;
  __shared__ double red[NT / 32];
  extern __shared__ double dyn_sh[];
  const int SL = A.sl;
  const int TX = NT / SL;
  const int tx = threadIdx.x % TX, sl = threadIdx.x / TX;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int per = g.n4cb * g.ls;
  const int npar = A.five_d ? 2 : 1;
  LinkCacheX2 lc;
  lc.sh = (float4 *)dyn_sh;
  lc.TX = TX;
  double *nrm_sh = dyn_sh + (LC ? (size_t)npar * 8 * 9 * TX * sizeof(float4) / sizeof(double) : 0);
  if (NORM)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const float2 a2 = f2b((float)A.a);
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
        Link<float> l;
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
        lc.put(pidx, j, xi, broadcast_link(l));
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
        AccX2 acc;
        hop_site_x2<P, LC>(A, x, tx, par_out, pidx, sbase, lc, acc);
        const long i = sbase + x;
        if (A.hop5) hop5_x2<P>(A, x, s, rbase, acc);
        SpX2 o = merge_x2(acc);
        if (XPAY) {
          float xn;
          const SpX2 xv = load_x2<P>(A.x, i, &xn);
#pragma unroll
          for (int p = 0; p < 2; p++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
              if (P == P16) {
                o.re[p][c] = fma2(xv.re[p][c], f2b(xn), mul2(a2, o.re[p][c]));
                o.im[p][c] = fma2(xv.im[p][c], f2b(xn), mul2(a2, o.im[p][c]));
              } else {
                o.re[p][c] = fma2(a2, o.re[p][c], xv.re[p][c]);
                o.im[p][c] = fma2(a2, o.im[p][c], xv.im[p][c]);
              }
            }
        } else if (A.a != 1.0) {
#pragma unroll
          for (int p = 0; p < 2; p++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
              o.re[p][c] = mul2(a2, o.re[p][c]);
              o.im[p][c] = mul2(a2, o.im[p][c]);
            }
        }
        const double n2 = store_x2<P>(A.out, i, o);
        if (NORM) nrm_sh[rhs * NT + threadIdx.x] += n2;
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
static inline int slice_lanes_x2(int nt, int ls) {
  int sl = 1;
  for (int c = 2; c <= nt / 32; c *= 2)
    if (ls % c == 0) sl = c;
  return sl;
}

template <int P, int NT, int MINB, bool LC>
static cudaError_t dslash_x2_launch_v(DslashArgs A, int xpay, int norm, cudaStream_t st) {
  A.sl = slice_lanes_x2(NT, A.g.ls);
  if (LC && A.g.ls * A.g.nrhs < 4) return cudaErrorNotSupported;
  const int tx = NT / A.sl;
  const long ntiles = (A.g.n4cb + tx - 1) / tx;
  long nb = ntiles < 148L * 16 ? ntiles : 148L * 16;
  const int npar = A.five_d ? 2 : 1;
  size_t shm = LC ? (size_t)npar * 8 * 9 * tx * sizeof(float4) : 0;
  if (norm) shm += sizeof(double) * NT * A.g.nrhs;
  if (shm > 200 * 1024) return cudaErrorNotSupported;  // above the opt-in set below
  static bool attr_set[2][2] = {{false, false}, {false, false}};
  if (shm + 1024 > 48 * 1024) {  // the 48 KB default counts static shared memory too
    auto set = [&](const void *f) { return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); };
    cudaError_t e = cudaSuccess;
    if (!attr_set[xpay][norm]) {
      if (xpay && norm) e = set((const void *)dslash_x2_kernel<P, NT, MINB, LC, true, true>);
      else if (xpay) e = set((const void *)dslash_x2_kernel<P, NT, MINB, LC, true, false>);
      else if (norm) e = set((const void *)dslash_x2_kernel<P, NT, MINB, LC, false, true>);
      else e = set((const void *)dslash_x2_kernel<P, NT, MINB, LC, false, false>);
      if (e != cudaSuccess) return e;
      attr_set[xpay][norm] = true;
    }
  }
  dim3 grid((unsigned)nb, 1);
  if (xpay && norm) dslash_x2_kernel<P, NT, MINB, LC, true, true><<<grid, NT, shm, st>>>(A);
  else if (xpay) dslash_x2_kernel<P, NT, MINB, LC, true, false><<<grid, NT, shm, st>>>(A);
  else if (norm) dslash_x2_kernel<P, NT, MINB, LC, false, true><<<grid, NT, shm, st>>>(A);
  else dslash_x2_kernel<P, NT, MINB, LC, false, false><<<grid, NT, shm, st>>>(A);
  return launched();
}

// Launch shapes the autotuner chooses from: (threads, min blocks/SM, link cache).
template <int P>
static cudaError_t dslash_x2_launch_p(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  switch (variant) {
    case 1: return dslash_x2_launch_v<P, 128, 4, false>(A, xpay, norm, st);
    case 2: return dslash_x2_launch_v<P, 256, 2, false>(A, xpay, norm, st);
    case 3: return dslash_x2_launch_v<P, 128, 1, true>(A, xpay, norm, st);
    case 4: return dslash_x2_launch_v<P, 256, 1, true>(A, xpay, norm, st);
    case 5: return dslash_x2_launch_v<P, 256, 2, true>(A, xpay, norm, st);
    case 6: return dslash_x2_launch_v<P, 128, 4, true>(A, xpay, norm, st);
    case 0: return dslash_x2_launch_v<P, 128, 1, false>(A, xpay, norm, st);
    default: return cudaErrorNotSupported;
  }
}


// ---------------------------------------------------------------------------
// Parity-class kernel: links of a tile held once in shared memory for every
// slice and right-hand side of one output parity, neighbour indices computed
// once per tile.
//
// A work unit is (tile of TX checkerboard sites, output-parity class).  For the
// 5-D checkerboard (DWF) the slices of one class are s0, s0+2, ... and all use
// the links of that 4-D parity, so the unit's 8*TX links are decoded and
// reconstructed once into shared memory as (Re, Im) pairs and every slice and
// right-hand side of the unit reads them from there; each thread computes its
// site's 8 neighbour indices and boundary flags once and then sweeps its
// (rhs, slice) pairs -- SL lanes of the block share them.
// ---------------------------------------------------------------------------
namespace x3 {

template <int P> __device__ __forceinline__ SpX2 load(const SpinorPtr &f, unsigned i, float *nrm) {
  return load_x2<P>(f, (long)i, nrm);
}

// A site as loaded from memory, before unpacking (so loads can be issued
// ahead of the arithmetic that consumes them).
template <int P> struct Raw;
template <> struct Raw<P32> { float4 c[6]; };
template <> struct Raw<P16> { uint4 c[3]; float nrm; };

template <int P> __device__ __forceinline__ Raw<P> load_raw(const SpinorPtr &f, unsigned i);
template <> __device__ __forceinline__ Raw<P32> load_raw<P32>(const SpinorPtr &f, unsigned i) {
  Raw<P32> r;
#pragma unroll
  for (int k = 0; k < 6; k++) r.c[k] = __ldg((const float4 *)f.data + k * f.stride + i);
  return r;
}
template <> __device__ __forceinline__ Raw<P16> load_raw<P16>(const SpinorPtr &f, unsigned i) {
  Raw<P16> r;
#pragma unroll
  for (int k = 0; k < 3; k++) r.c[k] = __ldg((const uint4 *)f.data + k * f.stride + i);
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
    const int pa = 2 * k, pb = 2 * k + 1;
    s.re[pa / 3][pa % 3] = dec16x2(r.c[k].x);
    s.im[pa / 3][pa % 3] = dec16x2(r.c[k].y);
    s.re[pb / 3][pb % 3] = dec16x2(r.c[k].z);
    s.im[pb / 3][pb % 3] = dec16x2(r.c[k].w);
  }
  *nrm = r.nrm;
  return s;
}

// U h / U^dag h with the link elements (ur, ui) read from shared memory.
template <bool DAG> __device__ __forceinline__ HfX2 umul(const float2 *sh, int TX, const HfX2 &h) {
  float2 e[3][3];
#pragma unroll
  for (int k = 0; k < 9; k++) e[k / 3][k % 3] = sh[k * TX];
  HfX2 o;
  float2 nh[3];
#pragma unroll
  for (int k = 0; k < 3; k++) nh[k] = DAG ? f2(-h.re[k].x, -h.re[k].y) : f2(-h.im[k].x, -h.im[k].y);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 re = f2b(0.f), im = f2b(0.f);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float2 u = DAG ? e[k][r] : e[r][k];
      const float2 ur = f2b(u.x), ui = f2b(u.y);
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

// DEPTH: neighbours whose loads are issued ahead of the one being computed
// (0: each is loaded where it is used; 8: all eight at the start of the site).
// WG: slice lanes inside one warp.  WG = 1: a warp is 32 consecutive sites of
// one slice.  WG = SL: a warp is 32/WG consecutive sites x WG slices, so the
// WG lanes that share a site read the same link words from shared memory
// (one wavefront serves them) while each slice's sites stay one 16-byte-per-
// site contiguous segment per chunk.
template <int P, int NT, int MINB, int SL, int DEPTH, int WG, bool XPAY, bool NORM, bool CGR = false>
__global__ void __launch_bounds__(NT, MINB) kernel(DslashArgs A) {
  constexpr int TX = NT / SL;
  static_assert(WG == 1 || WG == SL, "slice lanes are either all inside a warp or all across warps");
  const Geom &g = A.g;
  __shared__ double red[NT / 32];
  extern __shared__ double dyn_sh[];
  float2 *lsh = (float2 *)dyn_sh;                       // [8*9][TX]
  double *nrm_sh = dyn_sh + (size_t)72 * TX * sizeof(float2) / sizeof(double);
  constexpr int GX = 32 / WG;  // consecutive sites per warp and slice lane
  const int lane = threadIdx.x & 31;
  const int tx = WG == 1 ? (int)(threadIdx.x % TX) : (int)(threadIdx.x >> 5) * GX + lane % GX;
  const int sl = WG == 1 ? (int)(threadIdx.x / TX) : lane / GX;
  const int ntiles = (g.n4cb + TX - 1) / TX;
  const int nclass = A.five_d ? 2 : 1;
  const unsigned per = (unsigned)g.n4cb * (unsigned)g.ls;
  if (NORM || CGR)
    for (int q = 0; q < g.nrhs; q++) nrm_sh[q * NT + threadIdx.x] = 0;
  const float2 a2 = f2b((float)A.a);
  const float sdag = A.dag ? -1.f : 1.f;
  const int L[4] = {g.lx, g.ly, g.lz, g.lt};
  for (int unit = blockIdx.x; unit < ntiles * nclass; unit += gridDim.x) {
    const int tile = unit / nclass, cls = unit - tile * nclass;
    // output parity of the class and its first slice
    const int par_out = A.five_d ? cls : 1 - A.cb;
    const int s0 = A.five_d ? ((par_out + A.cb + 1) & 1) : 0;
    const int sstep = A.five_d ? 2 : 1;
    const int nsl = (g.ls - s0 + sstep - 1) / sstep;
    __syncthreads();  // the previous unit is done with the links
    for (int it = threadIdx.x; it < TX * 8; it += NT) {
      const int xi = it % TX, j = it / TX;
      const int xx = tile * TX + xi;
      if (xx >= g.n4cb) continue;
      Link<float> l;
      if (j < 4) {
        l = load_link<P>(A.U, par_out, j, xx);
      } else {
        const int mu = j - 4;
        const Coord c = decode(g, xx, par_out);
        int p[4] = {c.x, c.y, c.z, c.t};
        p[mu] = (p[mu] == 0) ? L[mu] - 1 : p[mu] - 1;
        l = load_link<P>(A.U, 1 - par_out, mu, cbindex(g, p[0], p[1], p[2], p[3]));
      }
#pragma unroll
      for (int k = 0; k < 9; k++) lsh[(j * 9 + k) * TX + xi] = make_float2(l.u[k / 3][k % 3].re, l.u[k / 3][k % 3].im);
    }
    __syncthreads();
    const int x = tile * TX + tx;
    if (x >= g.n4cb) continue;
    const Coord c = decode(g, x, par_out);
    int nb[8];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      int p[4] = {c.x, c.y, c.z, c.t};
      p[mu] = (p[mu] + 1 == L[mu]) ? 0 : p[mu] + 1;
      nb[mu] = cbindex(g, p[0], p[1], p[2], p[3]);
      int q[4] = {c.x, c.y, c.z, c.t};
      q[mu] = (q[mu] == 0) ? L[mu] - 1 : q[mu] - 1;
      nb[4 + mu] = cbindex(g, q[0], q[1], q[2], q[3]);
    }
    const bool flip_f = A.bc_t_sign < 0 && c.t == g.lt - 1;
    const bool flip_b = A.bc_t_sign < 0 && c.t == 0;
    const float2 *lx = lsh + tx;
    for (int w = sl; w < g.nrhs * nsl; w += SL) {
      const int rhs = w / nsl;
      const int s = s0 + sstep * (w - rhs * nsl);
      if (A.skip && A.skip[rhs]) continue;
      const unsigned rbase = (unsigned)rhs * per;
      const unsigned sbase = rbase + (unsigned)s * (unsigned)g.n4cb;
      AccX2 acc;
      zero_x2(acc);
      Raw<P> rw[8];
#pragma unroll
      for (int j = 0; j < DEPTH && j < 8; j++) rw[j] = load_raw<P>(A.in, sbase + (unsigned)nb[j]);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (DEPTH > 0 && j + DEPTH < 8) rw[j + DEPTH] = load_raw<P>(A.in, sbase + (unsigned)nb[j + DEPTH]);
        float nrm;
        const SpX2 v = unpack(DEPTH > 0 ? rw[j] : load_raw<P>(A.in, sbase + (unsigned)nb[j]), &nrm);
        const float sg = j < 4 ? -sdag : sdag;
        const float f = (j == 3 && flip_f) || (j == 7 && flip_b) ? -nrm : nrm;
        const float2 *lj = lx + j * 9 * TX;
        switch (j & 3) {
          case 0: {
            const HfX2 h = project_x2<0>(v, sg);
            accum_x2<0>(acc, j < 4 ? umul<false>(lj, TX, h) : umul<true>(lj, TX, h), sg, f);
          } break;
          case 1: {
            const HfX2 h = project_x2<1>(v, sg);
            accum_x2<1>(acc, j < 4 ? umul<false>(lj, TX, h) : umul<true>(lj, TX, h), sg, f);
          } break;
          case 2: {
            const HfX2 h = project_x2<2>(v, sg);
            accum_x2<2>(acc, j < 4 ? umul<false>(lj, TX, h) : umul<true>(lj, TX, h), sg, f);
          } break;
          default: {
            const HfX2 h = project_x2<3>(v, sg);
            accum_x2<3>(acc, j < 4 ? umul<false>(lj, TX, h) : umul<true>(lj, TX, h), sg, f);
          } break;
        }
      }
      if (A.hop5) hop5_x2<P>(A, x, s, (long)rbase, acc);
      SpX2 o = merge_x2(acc);
      const unsigned i = sbase + (unsigned)x;
      if (XPAY) {
        float xn;
        const SpX2 xv = load<P>(A.x, i, &xn);
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
        // r -= alpha (Ap + shift p), Ap = o held in registers (cg_r_update of blas.cu)
        const CgState *S = A.cg;
        const double sigma = S->shift;
        const float alpha = (float)(S->rr[rhs] / (S->d[rhs] + sigma * S->pp[rhs]));
        float rn;
        SpX2 rv = load<P>(A.cg_r, i, &rn);
        float pn = 0.f;
        SpX2 pv;
        if (sigma != 0.0) pv = load<P>(A.cg_p, i, &pn);
        const float2 ma = f2b(-alpha), rs = f2b(rn), ps = f2b((float)sigma * pn);
#pragma unroll
        for (int p = 0; p < 2; p++)
#pragma unroll
          for (int cc = 0; cc < 3; cc++) {
            float2 are = o.re[p][cc], aim = o.im[p][cc];
            if (sigma != 0.0) {
              are = fma2(ps, pv.re[p][cc], are);
              aim = fma2(ps, pv.im[p][cc], aim);
            }
            rv.re[p][cc] = fma2(ma, are, P == P16 ? mul2(rv.re[p][cc], rs) : rv.re[p][cc]);
            rv.im[p][cc] = fma2(ma, aim, P == P16 ? mul2(rv.im[p][cc], rs) : rv.im[p][cc]);
          }
        nrm_sh[rhs * NT + threadIdx.x] += store_x2<P>(A.cg_r, (long)i, rv);
      } else {
        const double n2 = store_x2<P>(A.out, (long)i, o);
        if (NORM) nrm_sh[rhs * NT + threadIdx.x] += n2;
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
        double t = ordered_sum<NT>(A.red.partial + q * gridDim.x, gridDim.x, red);
        if (threadIdx.x == 0 && !(A.skip && A.skip[q])) {
          if (!CGR) {
            A.red.result[q] = t;
          } else {
            // the recurrence scalars and the halting decision of cg_r_update (blas.cu)
            CgState *S = A.cg;
            const double c = t;
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
            if (A.red.result) A.red.result[q] = c;
          }
        }
        __syncthreads();
      }
    }
  }
}

template <int P, int NT, int MINB, int SL, int DEPTH, int WG>
static cudaError_t launch_v(DslashArgs A, int xpay, int norm, cudaStream_t st) {
  if (A.cg) {  // fused residual update: xpay hop whose output feeds r -= alpha Ap
    if (!xpay) return cudaErrorInvalidValue;
    // The update epilogue needs more registers than the plain hop: above 4
    // blocks/SM (<= 128 registers) it spills, so those shapes run it at 4.
    constexpr int MB = MINB > 4 ? 4 : MINB;
    constexpr int TX = NT / SL;
    const long units = (long)((A.g.n4cb + TX - 1) / TX) * (A.five_d ? 2 : 1);
    const long nb = units < 148L * 16 ? units : 148L * 16;
    const size_t shm = (size_t)72 * TX * sizeof(float2) + sizeof(double) * NT * A.g.nrhs;
    if (shm > 200 * 1024) return cudaErrorNotSupported;
    static bool attr = false;
    if (shm + 1024 > 48 * 1024 && !attr) {
      const cudaError_t e = cudaFuncSetAttribute((const void *)kernel<P, NT, MB, SL, DEPTH, WG, true, false, true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return e;
      attr = true;
    }
    kernel<P, NT, MB, SL, DEPTH, WG, true, false, true><<<(unsigned)nb, NT, shm, st>>>(A);
    return launched();
  }
  constexpr int TX = NT / SL;
  const int nclass = A.five_d ? 2 : 1;
  const int nsl = A.five_d ? (A.g.ls + 1) / 2 : A.g.ls;
  // every lane of the block must have work for this shape to make sense
  if (SL > 1 && nsl * A.g.nrhs < SL) return cudaErrorNotSupported;
  const long units = (long)((A.g.n4cb + TX - 1) / TX) * nclass;
  const long nb = units < 148L * 16 ? units : 148L * 16;
  size_t shm = (size_t)72 * TX * sizeof(float2);
  if (norm) shm += sizeof(double) * NT * A.g.nrhs;
  if (shm > 200 * 1024) return cudaErrorNotSupported;  // above the opt-in set below
  static bool attr_set[2][2] = {{false, false}, {false, false}};
  if (shm + 1024 > 48 * 1024 && !attr_set[xpay][norm]) {  // the 48 KB default counts static shared memory too
    const void *f = xpay && norm ? (const void *)kernel<P, NT, MINB, SL, DEPTH, WG, true, true>
                  : xpay         ? (const void *)kernel<P, NT, MINB, SL, DEPTH, WG, true, false>
                  : norm         ? (const void *)kernel<P, NT, MINB, SL, DEPTH, WG, false, true>
                                 : (const void *)kernel<P, NT, MINB, SL, DEPTH, WG, false, false>;
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    attr_set[xpay][norm] = true;
  }
  if (xpay && norm) kernel<P, NT, MINB, SL, DEPTH, WG, true, true><<<(unsigned)nb, NT, shm, st>>>(A);
  else if (xpay) kernel<P, NT, MINB, SL, DEPTH, WG, true, false><<<(unsigned)nb, NT, shm, st>>>(A);
  else if (norm) kernel<P, NT, MINB, SL, DEPTH, WG, false, true><<<(unsigned)nb, NT, shm, st>>>(A);
  else kernel<P, NT, MINB, SL, DEPTH, WG, false, false><<<(unsigned)nb, NT, shm, st>>>(A);
  return launched();
}

}  // namespace x3

// Launch shapes the autotuner chooses from: 0-6 the kernel above, 7-11 the
// parity-class kernel with (threads, min blocks/SM, slice lanes, load depth,
// slice lanes per warp).
template <int P>
static cudaError_t dslash_fp32x2_launch(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  if (A.cg && variant < 7) variant = 7;  // the fused residual update exists in the parity-class kernel only
  switch (variant) {
    case 7: return x3::launch_v<P, 128, 4, 4, 8, 4>(A, xpay, norm, st);
    case 8: return x3::launch_v<P, 128, 4, 4, 8, 1>(A, xpay, norm, st);
    case 9: return x3::launch_v<P, 128, 4, 2, 8, 2>(A, xpay, norm, st);
    case 10: return x3::launch_v<P, 128, 5, 4, 2, 4>(A, xpay, norm, st);
    case 11: return x3::launch_v<P, 128, 6, 4, 2, 4>(A, xpay, norm, st);
    default: return dslash_x2_launch_p<P>(A, xpay, norm, variant, st);
  }
}

}  // namespace cpsb

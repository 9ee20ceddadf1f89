// cpsb_device.cuh -- device-side building blocks shared by the sm_100a kernels.
//
// Field layouts in HBM:
//
//  * spinor field (a 4-D checkerboard, or Ls such slices, or Nrhs x Ls
//    slices): entries ordered by right-hand side, then column (4-D site and
//    slice class, site_entry below), then slice; stored in blocks of 8
//    entries, chunk k of the block's 8 entries as one 128-byte segment
//    (entry_ptr below), so a warp's 32 consecutive entries read four aligned
//    128-byte segments per chunk.  A chunk is 16 bytes:
//      FP64: 12 chunks of double2 = one complex component (spin k/3, colour k%3)
//      FP32:  6 chunks of float4, spin-paired: chunk 3p+c holds colour c of the
//             spins (2p, 2p+1) as (re_2p, re_2p+1, im_2p, im_2p+1), so the two
//             spins of a pair sit in the two lanes of a float2 (packed FP32x2 math)
//      16-bit: 3 chunks of 8 fixed-point values (uint4), the same spin-paired
//             order (32-bit word w = (3p+c)*2 + re/im holds spins 2p, 2p+1),
//             plus one float per site (max-abs / 16383, the quantum) in a
//             separate norm array.  A value v is stored as the biased integer
//             rint(v/quantum) + 16384, in [1, 32767] (14 bits of mantissa and a
//             sign, against IEEE fp16's 11): two stored values add or subtract
//             inside their 16-bit lane without overflow, so the hop kernel can
//             spin-project on the packed integers before decoding.
//  * gauge field, one 4-D checkerboard index x per parity p and direction mu:
//      FP64 (18 reals): 9 double2 chunks, chunk k = U[k/3][k%3], at
//                       data[((p*4+mu)*9 + k)*n4cb + x]
//      FP32 (recon-12): 3 float4 chunks holding rows 0 and 1
//      16-bit (recon-12): 3 uint2 chunks (4 fixed-point values, quantum 1/32767)
//                         holding rows 0 and 1
//    Reconstructed links omit the antiperiodic-time sign, which the kernel
//    applies to the hop (bc_t_sign) at the t boundary.
//
// Conventions follow CPS (cps_pp/src/util/dirac_op/d_op_wilson/noarch/
// wilson_dslash.C:64-167): chiral gamma basis, forward hop (1 - sdag*gamma_mu)
// U_mu(x) psi(x+mu), backward hop (1 + sdag*gamma_mu) U_mu(x-mu)^dag psi(x-mu),
// sdag = +1 (dag=0) / -1 (dag=1), checkerboard index x/2 + lx/2*(y+ly*(z+lz*t)).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cpsb {

enum Prec { P64 = 0, P32 = 1, P16 = 2 };

template <typename T> struct cplx { T re, im; };

template <typename T> __device__ __forceinline__ cplx<T> mk(T r, T i) { cplx<T> c; c.re = r; c.im = i; return c; }
template <typename T> __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename T> __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// conj(a) * b
template <typename T> __device__ __forceinline__ cplx<T> cmulc(cplx<T> a, cplx<T> b) {
  return mk(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
}
template <typename T> __device__ __forceinline__ cplx<T> cscale(T s, cplx<T> a) { return mk(s * a.re, s * a.im); }
// i*s*a for s = +-1 expressed as a real factor
template <typename T> __device__ __forceinline__ cplx<T> times_i(T s, cplx<T> a) { return mk(-s * a.im, s * a.re); }

template <typename T> struct Spinor { cplx<T> c[4][3]; };
template <typename T> struct Half { cplx<T> c[2][3]; };
template <typename T> struct Link { cplx<T> u[3][3]; };

// ---------------------------------------------------------------------------
// Lattice geometry on one checkerboard
// ---------------------------------------------------------------------------
struct Geom {
  int lx, ly, lz, lt;
  int lxh;          // lx/2
  int n4cb;         // half 4-D volume
  int ls;           // slices per right-hand side (1 for Wilson)
  int nrhs;         // right-hand sides stacked along the slowest index
  long nsites;      // n4cb * ls * nrhs = sites of one checkerboard field
  // Column layout (see below): ncls slice classes (2 for the DWF 5-D
  // checkerboard, where class k holds the slices s = k, k+2, ...; 1 otherwise),
  // cs[k] slices per column of class k, kb1 = first entry of class 1.
  int ncls;
  int cs[2];
  int kb1;
};

// Entry of slice s of 4-D checkerboard site x within one right-hand side.
// A field is stored as columns: the entries of one (site x, slice class k)
// pair are consecutive, ordered by slice, and the columns of class 0 precede
// those of class 1:  entry = k*kb1 + x*cs[k] + s/ncls.  Right-hand side q
// adds q * n4cb * ls.  Every slice of a class shares the 4-D parity of its
// sites, so the 4-D neighbours of a column are whole columns of the input.
__host__ __device__ __forceinline__ unsigned site_entry(const Geom &g, int s, int x) {
  const int k = g.ncls == 2 ? (s & 1) : 0;
  const int sp = g.ncls == 2 ? (s >> 1) : s;
  return (k ? (unsigned)g.kb1 : 0u) + (unsigned)x * (unsigned)g.cs[k] + (unsigned)sp;
}

// Entries are stored in blocks of 8: block b holds chunk 0 of its 8 entries,
// then chunk 1, ... (chunks are 16 bytes), so chunk k of entry i sits at
// entry_ptr(i)[8*k] and 8 consecutive entries read one 128-byte segment per
// chunk.  NCH chunks per entry: 12 (FP64), 6 (FP32), 3 (16-bit).
template <int NCH, typename V>
__device__ __forceinline__ V *entry_ptr(const void *base, unsigned i) {
  return (V *)((const char *)base + (size_t)((i >> 3) * (unsigned)NCH) * 128u + (size_t)(i & 7u) * 16u);
}

struct Coord { int x, y, z, t; };

// 4-D coordinates of checkerboard index idx of parity par.
__device__ __forceinline__ Coord decode(const Geom &g, int idx, int par) {
  Coord c;
  const unsigned u = (unsigned)idx;
  const unsigned r0 = u / (unsigned)g.lxh;
  const unsigned xh = u - r0 * (unsigned)g.lxh;
  const unsigned r1 = r0 / (unsigned)g.ly;
  c.y = (int)(r0 - r1 * (unsigned)g.ly);
  const unsigned r2 = r1 / (unsigned)g.lz;
  c.z = (int)(r1 - r2 * (unsigned)g.lz);
  c.t = (int)r2;
  c.x = 2 * (int)xh + ((c.y + c.z + c.t + par) & 1);
  return c;
}
__device__ __forceinline__ int cbindex(const Geom &g, int x, int y, int z, int t) {
  return (x >> 1) + g.lxh * (y + g.ly * (z + g.lz * t));
}

// ---------------------------------------------------------------------------
// Spinor and gauge access per precision
// ---------------------------------------------------------------------------
struct SpinorPtr {
  void *data;
  float *norm;   // FP16 only
  long stride;   // entries in the field
};

template <int P> struct PrecTraits;
template <> struct PrecTraits<P64> { typedef double real; };
template <> struct PrecTraits<P32> { typedef float real; };
template <> struct PrecTraits<P16> { typedef float real; };

// 16-bit fixed point.  The biased integer u in one half of a 32-bit word is
// turned into the float 2^23 + u by placing its bits under the exponent byte
// 0x4B, then 2^23 + 32768 is subtracted: two exact instructions per value.
__device__ __forceinline__ float dec16(unsigned w, int hi) {
  const unsigned bits = __byte_perm(w, 0x4B00u, hi ? 0x5432u : 0x5410u);
  return __int_as_float((int)bits) - 8421376.0f;
}
__device__ __forceinline__ unsigned q16(float v, float scale) {
  int q = __float2int_rn(v * scale);
  q = max(-32767, min(32767, q));
  return (unsigned)(q + 32768);
}
__device__ __forceinline__ unsigned enc16x2(float a, float b, float scale) {
  return q16(a, scale) | (q16(b, scale) << 16);
}
// Spinor storage: values in [-16383, 16383] with bias 16384.
constexpr float S16_MAX = 16383.0f;
__device__ __forceinline__ float dec16s(unsigned w, int hi) {
  const unsigned bits = __byte_perm(w, 0x4B00u, hi ? 0x5432u : 0x5410u);
  return __int_as_float((int)bits) - 8404992.0f;  // 2^23 + 16384
}
__device__ __forceinline__ unsigned q16s(float v, float scale) {
  int q = __float2int_rn(v * scale);
  q = max(-16383, min(16383, q));
  return (unsigned)(q + 16384);
}
__device__ __forceinline__ unsigned enc16x2s(float a, float b, float scale) {
  return q16s(a, scale) | (q16s(b, scale) << 16);
}

template <int P>
__device__ __forceinline__ Spinor<typename PrecTraits<P>::real> load_spinor(const SpinorPtr &f, long i);

template <>
__device__ __forceinline__ Spinor<double> load_spinor<P64>(const SpinorPtr &f, long i) {
  const double2 *b = entry_ptr<12, const double2>(f.data, (unsigned)i);
  Spinor<double> s;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    double2 v = __ldg(b + 8 * k);
    s.c[k / 3][k % 3] = mk(v.x, v.y);
  }
  return s;
}

template <>
__device__ __forceinline__ Spinor<float> load_spinor<P32>(const SpinorPtr &f, long i) {
  const float4 *b = entry_ptr<6, const float4>(f.data, (unsigned)i);
  Spinor<float> s;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    float4 v = __ldg(b + 8 * k);
    const int p = k / 3, c = k % 3;
    s.c[2 * p][c] = mk(v.x, v.z);
    s.c[2 * p + 1][c] = mk(v.y, v.w);
  }
  return s;
}

template <>
__device__ __forceinline__ Spinor<float> load_spinor<P16>(const SpinorPtr &f, long i) {
  const uint4 *b = entry_ptr<3, const uint4>(f.data, (unsigned)i);
  const float nrm = __ldg(f.norm + i);
  Spinor<float> s;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    uint4 v = __ldg(b + 8 * k);
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 4; j += 2) {
      const int pc = (4 * k + j) / 2;  // = 3p + c
      const int p = pc / 3, c = pc % 3;
      s.c[2 * p][c] = mk(dec16s(w[j], 0) * nrm, dec16s(w[j + 1], 0) * nrm);
      s.c[2 * p + 1][c] = mk(dec16s(w[j], 1) * nrm, dec16s(w[j + 1], 1) * nrm);
    }
  }
  return s;
}

template <int P>
__device__ __forceinline__ void store_spinor(const SpinorPtr &f, long i, const Spinor<typename PrecTraits<P>::real> &s);

template <>
__device__ __forceinline__ void store_spinor<P64>(const SpinorPtr &f, long i, const Spinor<double> &s) {
  double2 *b = entry_ptr<12, double2>(f.data, (unsigned)i);
#pragma unroll
  for (int k = 0; k < 12; k++) b[8 * k] = make_double2(s.c[k / 3][k % 3].re, s.c[k / 3][k % 3].im);
}

template <>
__device__ __forceinline__ void store_spinor<P32>(const SpinorPtr &f, long i, const Spinor<float> &s) {
  float4 *b = entry_ptr<6, float4>(f.data, (unsigned)i);
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int p = k / 3, c = k % 3;
    b[8 * k] = make_float4(s.c[2 * p][c].re, s.c[2 * p + 1][c].re, s.c[2 * p][c].im, s.c[2 * p + 1][c].im);
  }
}

template <>
__device__ __forceinline__ void store_spinor<P16>(const SpinorPtr &f, long i, const Spinor<float> &s) {
  float m = 0.f;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) m = fmaxf(m, fmaxf(fabsf(s.c[a][c].re), fabsf(s.c[a][c].im)));
  const float scale = m > 0.f ? S16_MAX / m : 0.f;
  f.norm[i] = m * (1.0f / S16_MAX);
  uint4 *b = entry_ptr<3, uint4>(f.data, (unsigned)i);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    unsigned w[4];
#pragma unroll
    for (int j = 0; j < 4; j += 2) {
      const int pc = (4 * k + j) / 2;
      const int p = pc / 3, c = pc % 3;
      w[j] = enc16x2s(s.c[2 * p][c].re, s.c[2 * p + 1][c].re, scale);
      w[j + 1] = enc16x2s(s.c[2 * p][c].im, s.c[2 * p + 1][c].im, scale);
    }
    b[8 * k] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Storage rounding of a spinor: what load_spinor<P> would return after
// store_spinor<P> (identity except for 16-bit storage).
template <int P, typename T> __device__ __forceinline__ Spinor<T> rounded(const Spinor<T> &s) {
  if (P != P16) return s;
  float m = 0.f;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) m = fmaxf(m, fmaxf(fabsf((float)s.c[a][c].re), fabsf((float)s.c[a][c].im)));
  const float scale = m > 0.f ? S16_MAX / m : 0.f;
  const float nq = m * (1.0f / S16_MAX);
  Spinor<T> o;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const unsigned w = enc16x2s((float)s.c[a][c].re, (float)s.c[a][c].im, scale);
      o.c[a][c] = mk((T)(dec16s(w, 0) * nq), (T)(dec16s(w, 1) * nq));
    }
  return o;
}

struct GaugePtr {
  const void *data;
  long n4cb;
};

template <int P>
__device__ __forceinline__ Link<typename PrecTraits<P>::real> load_link(const GaugePtr &g, int par, int mu, int x);

template <>
__device__ __forceinline__ Link<double> load_link<P64>(const GaugePtr &g, int par, int mu, int x) {
  const double2 *b = (const double2 *)g.data + (long)((par * 4 + mu) * 9) * g.n4cb + x;
  Link<double> l;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    double2 v = __ldg(b + k * g.n4cb);
    l.u[k / 3][k % 3] = mk(v.x, v.y);
  }
  return l;
}

template <typename T> __device__ __forceinline__ void reconstruct_row2(Link<T> &l) {
  // row2 = conj(row0 x row1)
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int k = (j + 1) % 3, m = (j + 2) % 3;
    cplx<T> v = cmul(l.u[0][k], l.u[1][m]) - cmul(l.u[0][m], l.u[1][k]);
    l.u[2][j] = mk(v.re, -v.im);
  }
}

template <>
__device__ __forceinline__ Link<float> load_link<P32>(const GaugePtr &g, int par, int mu, int x) {
  const float4 *b = (const float4 *)g.data + (long)((par * 4 + mu) * 3) * g.n4cb + x;
  Link<float> l;
  float4 a0 = __ldg(b), a1 = __ldg(b + g.n4cb), a2 = __ldg(b + 2 * g.n4cb);
  l.u[0][0] = mk(a0.x, a0.y); l.u[0][1] = mk(a0.z, a0.w);
  l.u[0][2] = mk(a1.x, a1.y); l.u[1][0] = mk(a1.z, a1.w);
  l.u[1][1] = mk(a2.x, a2.y); l.u[1][2] = mk(a2.z, a2.w);
  reconstruct_row2(l);
  return l;
}

template <>
__device__ __forceinline__ Link<float> load_link<P16>(const GaugePtr &g, int par, int mu, int x) {
  const uint2 *b = (const uint2 *)g.data + (long)((par * 4 + mu) * 3) * g.n4cb + x;
  const float q = 1.0f / 32767.0f;
  Link<float> l;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    uint2 v = __ldg(b + k * g.n4cb);
    int e0 = 2 * k, e1 = 2 * k + 1;
    l.u[e0 / 3][e0 % 3] = mk(dec16(v.x, 0) * q, dec16(v.x, 1) * q);
    l.u[e1 / 3][e1 % 3] = mk(dec16(v.y, 0) * q, dec16(v.y, 1) * q);
  }
  reconstruct_row2(l);
  return l;
}

// ---------------------------------------------------------------------------
// Spin projection.  (1 + sg*gamma_mu) psi = (h0, h1, r2(h), r3(h)) with
// h0, h1 the upper two spin components; the lower two are the fixed
// multiples of h below (derived from the gamma matrices of wilson_dslash.C:64-128).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ Half<T> project(const Spinor<T> &p, int mu, T sg) {
  Half<T> h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (mu == 0) {         // gamma_x: (i psi3, i psi2, -i psi1, -i psi0)
      h.c[0][c] = p.c[0][c] + times_i(sg, p.c[3][c]);
      h.c[1][c] = p.c[1][c] + times_i(sg, p.c[2][c]);
    } else if (mu == 1) {  // gamma_y: (-psi3, psi2, psi1, -psi0)
      h.c[0][c] = p.c[0][c] - cscale(sg, p.c[3][c]);
      h.c[1][c] = p.c[1][c] + cscale(sg, p.c[2][c]);
    } else if (mu == 2) {  // gamma_z: (i psi2, -i psi3, -i psi0, i psi1)
      h.c[0][c] = p.c[0][c] + times_i(sg, p.c[2][c]);
      h.c[1][c] = p.c[1][c] - times_i(sg, p.c[3][c]);
    } else {               // gamma_t: (psi2, psi3, psi0, psi1)
      h.c[0][c] = p.c[0][c] + cscale(sg, p.c[2][c]);
      h.c[1][c] = p.c[1][c] + cscale(sg, p.c[3][c]);
    }
  }
  return h;
}

// acc += full spinor rebuilt from the (multiplied) half spinor h.
template <typename T>
__device__ __forceinline__ void accum_reconstruct(Spinor<T> &acc, const Half<T> &h, int mu, T sg) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc.c[0][c] = acc.c[0][c] + h.c[0][c];
    acc.c[1][c] = acc.c[1][c] + h.c[1][c];
    if (mu == 0) {
      acc.c[2][c] = acc.c[2][c] + times_i(-sg, h.c[1][c]);
      acc.c[3][c] = acc.c[3][c] + times_i(-sg, h.c[0][c]);
    } else if (mu == 1) {
      acc.c[2][c] = acc.c[2][c] + cscale(sg, h.c[1][c]);
      acc.c[3][c] = acc.c[3][c] - cscale(sg, h.c[0][c]);
    } else if (mu == 2) {
      acc.c[2][c] = acc.c[2][c] + times_i(-sg, h.c[0][c]);
      acc.c[3][c] = acc.c[3][c] + times_i(sg, h.c[1][c]);
    } else {
      acc.c[2][c] = acc.c[2][c] + cscale(sg, h.c[0][c]);
      acc.c[3][c] = acc.c[3][c] + cscale(sg, h.c[1][c]);
    }
  }
}

template <typename T>
__device__ __forceinline__ Half<T> umul(const Link<T> &l, const Half<T> &h) {
  Half<T> o;
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int r = 0; r < 3; r++)
      o.c[a][r] = cmul(l.u[r][0], h.c[a][0]) + cmul(l.u[r][1], h.c[a][1]) + cmul(l.u[r][2], h.c[a][2]);
  return o;
}

template <typename T>
__device__ __forceinline__ Half<T> umul_dag(const Link<T> &l, const Half<T> &h) {
  Half<T> o;
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int r = 0; r < 3; r++)
      o.c[a][r] = cmulc(l.u[0][r], h.c[a][0]) + cmulc(l.u[1][r], h.c[a][1]) + cmulc(l.u[2][r], h.c[a][2]);
  return o;
}

template <typename T> __device__ __forceinline__ void zero(Spinor<T> &s) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) s.c[a][c] = mk(T(0), T(0));
}

template <typename T> __device__ __forceinline__ double norm2(const Spinor<T> &s) {
  double n = 0;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) n += (double)s.c[a][c].re * s.c[a][c].re + (double)s.c[a][c].im * s.c[a][c].im;
  return n;
}

template <typename T> __device__ __forceinline__ double redot(const Spinor<T> &a, const Spinor<T> &b) {
  double n = 0;
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) n += (double)a.c[s][c].re * b.c[s][c].re + (double)a.c[s][c].im * b.c[s][c].im;
  return n;
}

template <typename TO, typename TI> __device__ __forceinline__ Spinor<TO> convert(const Spinor<TI> &s) {
  Spinor<TO> o;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) o.c[a][c] = mk((TO)s.c[a][c].re, (TO)s.c[a][c].im);
  return o;
}

// ---------------------------------------------------------------------------
// Deterministic block reductions.  Every reduction writes one partial per
// block; the last block to finish (atomic ticket) sums the partials in block
// order, so results do not depend on scheduling or on concurrent work.
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NT / 32; i++) r += sh[i];
  }
  return r;  // valid in thread 0
}

// Returns true (in every thread) of the last block to arrive; the partials of
// all blocks are then visible and the ticket has been reset for the next use.
__device__ __forceinline__ bool last_block(unsigned *ticket, unsigned nblocks) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    is_last = (t == nblocks - 1);
    if (is_last) *ticket = 0;
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Sum of partial[0..n) in a fixed order (strided per thread, then the block
// tree), called by every thread of one block; the result is valid in thread 0.
template <int NT>
__device__ __forceinline__ double ordered_sum(const volatile double *partial, int n, double *sh) {
  double v = 0;
  for (int k = threadIdx.x; k < n; k += NT) v += partial[k];
  return block_sum<NT>(v, sh);
}

}  // namespace cpsb

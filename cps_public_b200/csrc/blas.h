// blas.h -- launchers of the streaming kernels in blas.cu and m5.cu.
#pragma once
#include "cg_state.h"
#include "cpsb_kernels.h"

namespace cpsb {

struct Scal2 {
  double a[MAX_RHS];
  double b[MAX_RHS];
};

cudaError_t launch_unitarity(const double *u, long nlinks, const int dims[4], int bc_t, unsigned long long *out,
                             cudaStream_t st);
cudaError_t launch_cg_r_update(int prec, const Geom &g, SpinorPtr r, SpinorPtr Ap, SpinorPtr p, CgState *S, Reduce red,
                               cudaStream_t st);
cudaError_t launch_cg_xp_update(int px, int prec, const Geom &g, SpinorPtr x, SpinorPtr p, SpinorPtr r, CgState *S,
                                Reduce red, cudaStream_t st);
cudaError_t launch_axpby(int po, SpinorPtr out, int px, SpinorPtr X, int py, SpinorPtr Y, const Geom &g, Scal2 sc,
                         const int *skip, Reduce red, int norm, cudaStream_t st);
cudaError_t launch_redot(int prec, const Geom &g, SpinorPtr X, SpinorPtr Y, Reduce red, cudaStream_t st);
// FP64 whole fields of nsites sites: conj(X).Y into red.result[0..1]; out = (cr + i ci) X + Y.
cudaError_t launch_cdot(SpinorPtr X, SpinorPtr Y, long nsites, Reduce red, cudaStream_t st);
cudaError_t launch_caxpy(SpinorPtr out, double cr, double ci, SpinorPtr X, SpinorPtr Y, long nsites, cudaStream_t st);

// Mobius 5th-direction kernels (m5.cu).
struct M5Coef {
  double K;            // kappa_b/kappa_c (the M5 hopping coefficient ratio)
  double invd;         // 1/(1 + m_f prod(-K)) (dag 0) or its dag-1 form
  double f1[64];       // per-step wall factors of the forward sweep
  double f2[64];       // per-step wall factors of the backward sweep
  double b, c, mass;   // mixing b + c*H5, walls -m_f
  double scale;        // output scale
};
cudaError_t launch_m5(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x, const M5Coef &cf,
                      int xpay, int norm, Reduce red, const int *skip, cudaStream_t st);
// The Mobius hop with the M5 sweeps of its output fused in (hop_m5.cuh), A as
// for launch_dslash with A.a the output scale:
//   A.dag 0: out = a mix(M5^-1 (D in))   (cf the dag-0 coefficients; no xpay, no norm)
//   A.dag 1: out = [x +] a M5^-dag(mix^dag(D^dag in))  [, |out|^2 into A.red]
// cudaErrorNotSupported where no fused form exists; the caller then runs
// launch_dslash and launch_m5.
cudaError_t launch_hop_m5(int prec, const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st);

// zMobius form (complex per-slice coefficients, zmobius_m5inv.C:247-400 and
// :403-686, zmobius_dslash_5_plus.C:125-376): one table per launch shape, in
// device memory.  The kernel applies, per 4-D site and chirality half h
// (0: spins 0,1; 1: spins 2,3) to the column v[0..Ls) of one component:
//   pre:   v_s *= pre_s
//   dag 1: v_s <- bb_s v_s + cc[h]_s v_nb          (mixing before the sweeps)
//   sweep: walls first:  v_last *= invd[h]; v_last += w[h]_s v_s (s ascending);
//                        v_s += a[h]_s v_{s+1} (s descending)
//          chain first:  v_{s+1} += a[h]_s v_s (s ascending);
//                        v_s += w[h]_s v_last (s descending); v_last *= invd[h]
//   dag 0: v_s <- bb_s v_s + cc[h]_s v_nb          (mixing after the sweeps)
//   post:  v_s *= post_s, then out = [x +] v
// with nb = s-1 / s+1 (cyclic) for the upper / lower half at dag 0 and the
// reverse at dag 1 (the wall terms carry -m_f in cc).
struct ZM5Tab {
  double2 a[2][64], w[2][64];
  double2 invd[2];
  int walls_first[2];
  double2 bb[64], cc[2][64];
  double2 pre[64], post[64];
  int sweep, mix, pre_on, post_on;
};
cudaError_t launch_m5z(int prec, int dag, const Geom &g, SpinorPtr out, SpinorPtr in, SpinorPtr x,
                       const ZM5Tab *tab, int xpay, int norm, Reduce red, const int *skip, cudaStream_t st);

}  // namespace cpsb

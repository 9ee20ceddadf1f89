// cpsb_kernels.h -- host-visible launch interface of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include "cpsb_device.cuh"

namespace cpsb {

// Reduction target: one partial per block (rhs-major), a ticket, and nrhs results.
struct Reduce {
  double *partial;
  unsigned *ticket;
  double *result;
};

struct CgState;  // cg_state.h

struct DslashArgs {
  Geom g;
  GaugePtr U;
  SpinorPtr in, out, x;   // x: the vector added by the xpay epilogue
  int cb;                 // checkerboard of the input (output is 1-cb)
  int dag;
  int five_d;             // 1: DWF 5-D checkerboarding, 0: all slices share a 4-D parity
  int hop5;               // 1: add the Shamir 5th-direction hop
  double hop5_fact;       // 2*a5_inv
  double hop5_wall;       // -2*m_f*a5_inv
  double a;               // epilogue coefficient
  double bc_t_sign;       // -1: reconstructed links need the antiperiodic sign at the t boundary
  Reduce red;             // |out|^2 per RHS when requested
  const int *skip;        // per-RHS: nonzero skips that RHS (device memory), may be null
  int rg;                 // right-hand sides per warp lane group (set by the launcher)
  int rgroup;             // right-hand sides per work unit (set by the launcher)
  int torder;             // 1: tiles visited t-fastest where they are whole rows (set by the launcher)
  // Fused CG residual update: when cg is set, out = x + a D in is not stored; instead r -= alpha (out +
  // shift p) with alpha from cg, |r|^2 per RHS is reduced, and the last block
  // advances the recurrence scalars as the r-update kernel of blas.cu does.
  CgState *cg;
  SpinorPtr cg_r, cg_p;
  SpinorPtr cg_x;         // when set: also x += alpha p (x FP64 for FP64 storage, else FP32)
  int cg_shift;           // nonzero: the solve's shift is nonzero (the update reads p)
};

// Kernel-launch accounting (cpsb_kernel_launches): every launcher calls
// count_launch(); launches recorded into a CUDA graph are counted when the
// graph is replayed instead.
void count_launch(unsigned long long n = 1);
void set_capturing(bool on);
unsigned long long launch_count();
// Every launcher returns through this: counts the launch, reports launch errors.
inline cudaError_t launched() {
  count_launch();
  return cudaGetLastError();
}

// Grid: blockIdx.y = right-hand side, blockIdx.x strides over the sites of one RHS.
int grid_blocks(long sites_per_rhs, int nt);

// variant: launch shape 0..NUM_DSLASH_VARIANTS-1 of hop.cuh, chosen by the
// autotuner; a launcher returns cudaErrorNotSupported for shapes that do not
// fit the operator.
constexpr int NUM_DSLASH_VARIANTS = 9;
cudaError_t launch_dslash(int prec, const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);

// ---------------------------------------------------------------- BLAS
// All vectors share one Geom (nsites sites, nrhs right-hand sides).  Scalars
// marked "dev" are read from device memory so the kernels can be captured in
// CUDA graphs and need no host round trip.
struct CgState;   // defined in cg_state.h

// CPS-order vectors <-> device fields of geometry g (g.nsites entries).
cudaError_t launch_pack(int prec, SpinorPtr dst, const double *src, const Geom &g, cudaStream_t st);
cudaError_t launch_unpack(int prec, double *dst, SpinorPtr src, const Geom &g, cudaStream_t st);
cudaError_t launch_convert(int pdst, SpinorPtr dst, int psrc, SpinorPtr src, long nsites, cudaStream_t st);
cudaError_t launch_fconvert(double *out, const double *in, const int dims[4], int ls, int order, int direction,
                            cudaStream_t st);
cudaError_t launch_gauge_pack(int prec, void *dst, const double *u_canonical, const int dims[4],
                              int bc_t, cudaStream_t st);

}  // namespace cpsb

// ms_state.h -- device-resident scalar state of the multishift CG.
//
// Mirrors the scalars of DiracOp::MInvCG (cps_pp/src/util/dirac_op/d_op_base/
// noarch/minvcg.C:97-125): a, b, c, cp, d, the shifted z/bs recurrences and the
// per-shift convergence flags, one set per source vector of a batched solve.
// The last block of the residual reduction advances all of them, so an
// iteration is a fixed launch sequence.
#pragma once
#include "cg_state.h"

namespace cpsb {

constexpr int MAX_SHIFT = 32;

struct MsState {
  double a, b, bp, c, cp, pp;         // d = d_mm + shift[0]*pp
  double z[2][MAX_SHIFT];
  double bs[MAX_SHIFT];
  double as[MAX_SHIFT];
  double mass[MAX_SHIFT];
  double rsd_sq[MAX_SHIFT];
  double alpha[MAX_SHIFT];
  double css[MAX_SHIFT];              // c*z^2 when the shift converged
  int conv[MAX_SHIFT];                // convsP after the latest check
  int conv_prev[MAX_SHIFT];           // convsP at the start of the iteration
  int conv_iter[MAX_SHIFT];
  int iz;
  int nshift;
  int type;                           // 0 MULTI, 1 SINGLE
  int k;                              // iterations performed (the init step is k = 0)
  int max_iter;
  int done;                           // set when every shift converged or k reached max_iter
  int breakdown;
};

// The states of the source vectors solved together, with the per-vector
// values that kernels read or write as arrays: |M p_0|^2 (the fused norm of
// MatPcDagMatPc writes result[q]) and the flag set after the solution update
// of a vector's final iteration (the operator's per-right-hand-side skip mask).
struct MsBatch {
  MsState s[MAX_RHS];
  double d_mm[MAX_RHS];
  int done_applied[MAX_RHS];
  int nvec;
};

}  // namespace cpsb

// cg_state.h -- device-resident scalar state of the Krylov solvers.
//
// Every scalar of the CG recurrence (inv_cg.C:293-364 of CPS) lives in device
// memory and is produced by the last block of the reduction that computes it,
// so an iteration is a fixed sequence of kernel launches with no host round
// trip; the host polls this struct between batches of iterations.
#pragma once

namespace cpsb {

constexpr int MAX_RHS = 16;

enum HaltReason { HALT_NONE = 0, HALT_CONVERGED = 1, HALT_RELIABLE = 2, HALT_MAXITER = 3, HALT_BREAKDOWN = 4 };

struct CgState {
  double rr[MAX_RHS];        // |r|^2 of the current residual
  double rr_prev[MAX_RHS];   // |r|^2 at the start of the iteration
  double d[MAX_RHS];         // <p, A p>
  double alpha[MAX_RHS];
  double beta[MAX_RHS];
  double stp[MAX_RHS];       // stop when rr <= stp  (stop_rsd^2 |b|^2)
  double maxr[MAX_RHS];      // largest |r| since the last reliable update
  double pp[MAX_RHS];        // |p|^2 (needed for the shifted operator A + sigma)
  double delta;              // reliable-update threshold (0: pure CG)
  double shift;              // constant shift sigma of (A + sigma): <p,(A+sigma)p> = d + sigma pp
  int halt[MAX_RHS];         // set by the r-update: this RHS pauses for the host
  int halt_done[MAX_RHS];    // set after the x/p update of the halting iteration
  int reason[MAX_RHS];
  int iters[MAX_RHS];        // iterations performed
  int max_iter;              // CPS max_num_iter: at most max_num_iter-1 iterations
  int nrhs;
};

}  // namespace cpsb

namespace cpsb {

// Control block of a device-side loop over batches of iterations (the body of a
// CUDA-graph WHILE node, graph_loop.cu).  Before each launch the host sets
// count = 0, cap and done[]; the condition kernel that ends every batch counts
// it and ends the loop once every right-hand side has halted, or (when the
// host has per-RHS work, `any`) one that is not in done[] has halted, or cap
// batches have run.
struct LoopCtl {
  unsigned count;
  unsigned cap;
  int done[MAX_RHS];
};

}  // namespace cpsb

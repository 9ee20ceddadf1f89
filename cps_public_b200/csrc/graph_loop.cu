// graph_loop.cu -- device-side iteration loops for the Krylov solvers.
//
// A solve's iterations are recorded once as a batch and replayed.  Replaying
// the batch from the host costs a device-to-host read of the solver state and
// a stream synchronisation per batch; for small lattices (an L2-resident 8^4
// Wilson solve runs a batch in tens of microseconds) that round trip is most of
// the time.  Here the batch is the body of a CUDA-graph WHILE node whose
// condition is set on the device by a one-thread kernel at the end of every
// batch (cudaGraphSetConditional), so one graph launch runs batches until the
// solver needs the host -- convergence, a reliable update, the iteration limit
// -- and the host reads the state once.  The condition kernel also counts the
// batches and stops at LoopCtl::cap, so a launch always ends.
#include <stdlib.h>
#include <string.h>

#include "host.h"
#include "ms_state.h"

namespace cpsb {

__global__ void cg_loop_cond_kernel(cudaGraphConditionalHandle h, const CgState *S, LoopCtl *L, int nrhs, int any) {
  const unsigned c = ++L->count;
  bool all = true, one = false;
  for (int q = 0; q < nrhs; q++) {
    const bool hd = S->halt_done[q] != 0;
    all = all && hd;
    one = one || (hd && !L->done[q]);
  }
  cudaGraphSetConditional(h, (all || (any && one) || c >= L->cap) ? 0u : 1u);
}

__global__ void ms_loop_cond_kernel(cudaGraphConditionalHandle h, const MsBatch *B, LoopCtl *L, int nvec) {
  const unsigned c = ++L->count;
  bool all = true;
  for (int q = 0; q < nvec; q++) all = all && B->done_applied[q] != 0;
  cudaGraphSetConditional(h, (all || c >= L->cap) ? 0u : 1u);
}

cudaError_t launch_cg_loop_cond(cudaGraphConditionalHandle h, const CgState *S, LoopCtl *L, int nrhs, int any,
                                cudaStream_t st) {
  cg_loop_cond_kernel<<<1, 1, 0, st>>>(h, S, L, nrhs, any);
  return launched();
}

cudaError_t launch_ms_loop_cond(cudaGraphConditionalHandle h, const MsBatch *B, LoopCtl *L, int nvec,
                                cudaStream_t st) {
  ms_loop_cond_kernel<<<1, 1, 0, st>>>(h, B, L, nvec);
  return launched();
}

bool graph_loops_enabled() {
  const char *e = getenv("CPSB_GRAPH_LOOP");
  return !(e && atoi(e) == 0);
}

bool build_loop_graph(cudaStream_t st, const std::function<void(cudaGraphConditionalHandle)> &record,
                      cudaGraphExec_t *exec, size_t *body_nodes) {
  cudaGraph_t outer = nullptr;
  CK(cudaGraphCreate(&outer, 0));
  struct GraphGuard {
    cudaGraph_t g;
    ~GraphGuard() { if (g) cudaGraphDestroy(g); }
  } guard{outer};
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, outer, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGetLastError();
    return false;  // no conditional nodes on this driver: the caller replays plain batches
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, outer, nullptr, 0, &cp) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  set_capturing(true);
  try {
    record(h);
  } catch (...) {
    set_capturing(false);
    cudaGraph_t tmp;
    cudaStreamEndCapture(st, &tmp);
    throw;
  }
  set_capturing(false);
  cudaGraph_t captured;
  CK(cudaStreamEndCapture(st, &captured));
  size_t nn = 0;
  CK(cudaGraphGetNodes(body, nullptr, &nn));
  *body_nodes = nn;
  CK(cudaGraphInstantiate(exec, outer, 0));
  return true;
}

}  // namespace cpsb

// tune.cu -- launch-shape autotuner for the hopping kernels.
//
// The first time a hopping-kernel configuration (precision, epilogue, lattice,
// Ls, right-hand sides, checkerboarding) is launched outside a CUDA-graph
// capture, every launch variant is timed on the live arguments with CUDA
// events and the fastest is kept for the rest of the process.  Launches met
// during a capture before tuning use variant 0.  CPSB_TUNE=0 disables tuning;
// CPSB_TUNE_VERBOSE=1 prints each decision; CPSB_TUNE_FORCE=v pins variant v
// (for profiling) wherever it fits.  Every launch shape computes the same
// operator output bit for bit; the fused norms and dot products are summed over
// each shape's blocks in its own way, so they agree to rounding.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>

#include "host.h"

namespace cpsb {

namespace {
struct Key {
  int prec, xpay, norm, five_d, hop5, lx, ly, lz, lt, ls, nrhs, dev;
  bool operator<(const Key &o) const { return memcmp(this, &o, sizeof(Key)) < 0; }
};
std::map<Key, int> &table() {
  static std::map<Key, int> t;
  return t;
}
std::mutex mu;

bool tuning_enabled() {
  const char *e = getenv("CPSB_TUNE");
  return !(e && e[0] == '0');
}
}  // namespace

int tuned_variant(const DslashArgs &A, int prec, int xpay, int norm, cudaStream_t st) {
  Key k;
  memset(&k, 0, sizeof(k));
  k.prec = prec;
  k.xpay = xpay;
  k.norm = norm;
  k.five_d = A.five_d;
  k.hop5 = A.hop5;
  k.lx = A.g.lx;
  k.ly = A.g.ly;
  k.lz = A.g.lz;
  k.lt = A.g.lt;
  k.ls = A.g.ls;
  k.nrhs = A.g.nrhs;
  k.dev = ctx().device;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = table().find(k);
    if (it != table().end()) return it->second;
  }
  if (!tuning_enabled()) return 0;
  if (const char *f = getenv("CPSB_TUNE_FORCE")) {
    // Forced launch shape (profiling): used when it fits this configuration.
    const int v = atoi(f);
    if (v >= 0 && v < NUM_DSLASH_VARIANTS) {
      cudaStreamCaptureStatus cs0 = cudaStreamCaptureStatusNone;
      CK(cudaStreamIsCapturing(st, &cs0));
      if (cs0 == cudaStreamCaptureStatusNone) {
        const cudaError_t e = launch_dslash(prec, A, xpay, norm, v, st);
        if (e == cudaSuccess) {
          std::lock_guard<std::mutex> lk(mu);
          table()[k] = v;
          return v;
        }
        if (e != cudaErrorNotSupported) CK(e);
      }
    }
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int best = 0;
  float best_ms = 1e30f;
  const int reps = 3;
  for (int v = 0; v < NUM_DSLASH_VARIANTS; v++) {
    const cudaError_t e = launch_dslash(prec, A, xpay, norm, v, st);  // warm
    if (e == cudaErrorNotSupported) continue;
    CK(e);
    CK(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; r++) CK(launch_dslash(prec, A, xpay, norm, v, st));
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (getenv("CPSB_TUNE_VERBOSE"))
      fprintf(stderr, "cpsb tune:   variant %d %.4f ms\n", v, ms / reps);
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (getenv("CPSB_TUNE_VERBOSE"))
    fprintf(stderr, "cpsb tune: prec %d xpay %d norm %d ls %d nrhs %d -> variant %d (%.3f ms)\n", prec, xpay, norm,
            A.g.ls, A.g.nrhs, best, best_ms / reps);
  std::lock_guard<std::mutex> lk(mu);
  table()[k] = best;
  return best;
}

}  // namespace cpsb

// dslash_f32.cu -- instantiates the hopping kernel of hop.cuh for FP32
// storage (one translation unit per precision, so they compile in parallel).
#include "hop.cuh"

namespace cpsb {
cudaError_t launch_dslash_f32(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  return hop_launch_p<P32>(A, xpay, norm, variant, st);
}
}  // namespace cpsb

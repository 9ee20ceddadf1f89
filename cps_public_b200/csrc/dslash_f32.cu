// dslash_f32.cu -- instantiates the packed FP32x2 hopping kernels of dslash_x2.cuh for P32
// storage (one translation unit per precision so they compile in parallel).
#include "dslash_x2.cuh"

namespace cpsb {
cudaError_t launch_dslash_f32(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  return dslash_fp32x2_launch<P32>(A, xpay, norm, variant, st);
}
}  // namespace cpsb

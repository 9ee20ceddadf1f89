// dslash_f16.cu -- instantiates the packed FP32x2 hopping kernels of dslash_x2.cuh for P16
// storage (one translation unit per precision so they compile in parallel).
#include "dslash_x2.cuh"

namespace cpsb {
cudaError_t launch_dslash_f16(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  return dslash_fp32x2_launch<P16>(A, xpay, norm, variant, st);
}
}  // namespace cpsb

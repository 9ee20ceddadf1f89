// dslash_f16.cu -- instantiates the hopping kernels of dslash_impl.cuh for P16
// storage (one translation unit per precision so they compile in parallel).
#include "dslash_impl.cuh"

namespace cpsb {
cudaError_t launch_dslash_f16(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  return dslash_launch_p<P16>(A, xpay, norm, variant, st);
}
}  // namespace cpsb

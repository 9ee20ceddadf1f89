// dslash.cu -- precision dispatch of the hopping kernel (hop.cuh).
#include "cpsb_kernels.h"

namespace cpsb {

cudaError_t launch_dslash_f64(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);
cudaError_t launch_dslash_f32(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);
cudaError_t launch_dslash_f16(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);

cudaError_t launch_dslash(int prec, const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  if (prec == P64) return launch_dslash_f64(A, xpay, norm, variant, st);
  if (prec == P32) return launch_dslash_f32(A, xpay, norm, variant, st);
  return launch_dslash_f16(A, xpay, norm, variant, st);
}

}  // namespace cpsb

// dslash.cu -- precision dispatch of the hopping kernel (hop.cuh) and of the
// Mobius hop with fused M5 sweeps (hop_m5.cuh).
#include "blas.h"

namespace cpsb {

cudaError_t launch_dslash_f64(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);
cudaError_t launch_dslash_f32(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);
cudaError_t launch_dslash_f16(const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st);

cudaError_t launch_dslash(int prec, const DslashArgs &A, int xpay, int norm, int variant, cudaStream_t st) {
  if (prec == P64) return launch_dslash_f64(A, xpay, norm, variant, st);
  if (prec == P32) return launch_dslash_f32(A, xpay, norm, variant, st);
  return launch_dslash_f16(A, xpay, norm, variant, st);
}

cudaError_t launch_hop_m5_f64(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st);
cudaError_t launch_hop_m5_f32(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st);
cudaError_t launch_hop_m5_f16(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st);

cudaError_t launch_hop_m5(int prec, const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st) {
  if (prec == P64) return launch_hop_m5_f64(A, cf, xpay, norm, st);
  if (prec == P32) return launch_hop_m5_f32(A, cf, xpay, norm, st);
  return launch_hop_m5_f16(A, cf, xpay, norm, st);
}

}  // namespace cpsb

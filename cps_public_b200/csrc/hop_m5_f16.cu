// hop_m5_f16.cu -- instantiates the Mobius hop with fused M5 sweeps of
// hop_m5.cuh for 16-bit storage (one translation unit per precision).
#include "hop_m5.cuh"

namespace cpsb {
cudaError_t launch_hop_m5_f16(const DslashArgs &A, const M5Coef &cf, int xpay, int norm, cudaStream_t st) {
  return hop_m5_launch_p<P16>(A, cf, xpay, norm, st);
}
}  // namespace cpsb

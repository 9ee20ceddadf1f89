// noalloc.cu -- global dot products that allocate no memory.
//
// cpsb_redot_noalloc is the deterministic reduction of redot_kernel (blas.cu)
// for callers that must not allocate device memory: HMC and serving loops that
// reserve their whole HBM budget up front and run every solve out of that
// arena, and codes that keep the device free of implicit synchronisation
// (cudaFree synchronises the device).  Its
// reduction scratch -- one partial sum per block and vector, plus the
// last-block ticket -- lives in a file-scope __device__ array of
// NOALLOC_SCRATCH_BYTES (80 KiB) that every GPU loading the library holds
// until the process exits.  Host code cannot pass that array's name to a
// kernel (it is a host-side stand-in, not a device address), so the device
// address is looked up once per device with cudaGetSymbolAddress.
#include <mutex>

#include "../../include/cpsb200.h"
#include "cpsb_device.cuh"
#include "cpsb_kernels.h"

namespace cpsb {

constexpr int NOALLOC_MAX_VEC = 16;
constexpr int NOALLOC_BLOCKS = 148 * 4;
constexpr int NOALLOC_NT = 256;
constexpr size_t NOALLOC_SCRATCH_BYTES = 80 * 1024;
static_assert(NOALLOC_BLOCKS * NOALLOC_MAX_VEC * sizeof(double) + 256 <= NOALLOC_SCRATCH_BYTES,
              "scratch too small for the partial sums");

// Partials at [0, NOALLOC_BLOCKS*NOALLOC_MAX_VEC) doubles, ticket after them.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

__global__ void __launch_bounds__(NOALLOC_NT) redot_noalloc_kernel(const double *x, const double *y, long n,
                                                                    unsigned char *scratch, double *result) {
  __shared__ double sh[NOALLOC_NT / 32];
  double *partial = (double *)scratch;
  unsigned *ticket = (unsigned *)(scratch + NOALLOC_BLOCKS * NOALLOC_MAX_VEC * sizeof(double));
  const int v = blockIdx.y;
  const double *xv = x + (long)v * n, *yv = y + (long)v * n;
  double acc = 0;
  for (long i = (long)blockIdx.x * NOALLOC_NT + threadIdx.x; i < n; i += (long)gridDim.x * NOALLOC_NT)
    acc += xv[i] * yv[i];
  const double bs = block_sum<NOALLOC_NT>(acc, sh);
  if (threadIdx.x == 0) partial[v * gridDim.x + blockIdx.x] = bs;
  if (last_block(ticket, gridDim.x * gridDim.y)) {
    for (int q = 0; q < (int)gridDim.y; q++) {
      const double t = ordered_sum<NOALLOC_NT>(partial + q * gridDim.x, gridDim.x, sh);
      if (threadIdx.x == 0) result[q] = t;
      __syncthreads();
    }
  }
}

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[MAX_DEVICES];
}  // namespace

}  // namespace cpsb

using namespace cpsb;

extern "C" int cpsb_redot_noalloc(const double *x, const double *y, long n, int nvec, double *result,
                                  void *stream) {
  if (!x || !y || !result || n < 1) return CPSB_ERR_ARG;
  if (nvec < 1 || nvec > NOALLOC_MAX_VEC) return CPSB_ERR_ARG;  // beyond the scratch's partial slots
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return CPSB_ERR_NO_DEVICE;
  unsigned char *scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
      // First call on this device: look up the device address of the array
      // with this device current.  Make this first call before any capture.
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return CPSB_ERR_CUDA;
      }
      g_scratch_addr[dev] = (unsigned char *)p;
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  // The array keeps the previous call's contents: the ticket must start at zero.
  unsigned *ticket = (unsigned *)(scratch + NOALLOC_BLOCKS * NOALLOC_MAX_VEC * sizeof(double));
  if (cudaMemsetAsync(ticket, 0, sizeof(unsigned), st) != cudaSuccess) {
    cudaGetLastError();
    return CPSB_ERR_CUDA;
  }
  long nb = (n + NOALLOC_NT - 1) / NOALLOC_NT;
  if (nb > NOALLOC_BLOCKS) nb = NOALLOC_BLOCKS;
  redot_noalloc_kernel<<<dim3((unsigned)nb, (unsigned)nvec), NOALLOC_NT, 0, st>>>(x, y, n, scratch, result);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? CPSB_OK : CPSB_ERR_CUDA;
}

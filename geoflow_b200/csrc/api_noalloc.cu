// api_noalloc.cu -- gf_integrate_noalloc: the integral reduction of
// gf_integrate with no device allocation anywhere on its path.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// integrate.  Typical cases are host frameworks that reserve device memory
// up front for their own pool allocator (a foreign cudaMalloc then fails or
// fragments that pool), time-stepping loops that must not stall (cudaFree
// synchronises the whole device, and a first allocation can too), and
// deployments that forbid allocation after start-up.  Such a caller owns
// the inputs and the output; this entry point brings its own scratch.
//
// The scratch is a fixed array in the library's device image, 256 KB plus a
// 256-byte header per GPU that loads the library, held until the process
// exits.  It limits n to GF_NOALLOC_MAX_BLOCKS * GF_NOALLOC_CHUNK elements.
// Every call shares it, and it keeps the last call's contents: the ticket
// counter that must start at zero is cleared by each call (and left at zero
// by the last block), and the block partials are always written before they
// are read.  Two calls that overlap on the GPU (for example on two streams)
// race on the array; order them on one stream.
//
// In host code the array's name is only a host-side stand-in, so every
// call looks up its device address on the current device with
// cudaGetSymbolAddress and passes the address to the kernel (cheap once the
// library's module is loaded there; nothing is cached, so a call after
// cudaDeviceReset finds the reloaded array).  The first call on a device
// may load the module: make it before any stream capture.

#include "gf_common.cuh"
#include "k_vec.cuh"

namespace {

constexpr int kChunk = GF_NOALLOC_CHUNK;        // elements per block
constexpr int kMaxBlocks = GF_NOALLOC_MAX_BLOCKS;
constexpr int kHeader = 32;                     // doubles: ticket counter + padding
constexpr int kThreads = 256;

// [0, kHeader): the ticket counter (an unsigned int at offset 0);
// [kHeader, kHeader + kMaxBlocks): one partial sum per block.
static __device__ __align__(256) double g_noalloc_scratch[kHeader + kMaxBlocks];

__global__ void __launch_bounds__(kThreads)
    k_integrate_noalloc(int64_t n, const double *__restrict__ mass, const double *__restrict__ u,
                        double *scratch, double *result) {
  __shared__ double sh[32];
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
  double *partials = scratch + kHeader;
  const int64_t begin = (int64_t)blockIdx.x * kChunk;
  const int64_t end = begin + kChunk < n ? begin + kChunk : n;
  double s = 0.0;
  for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) s += mass[i] * u[i];
  s = gfk::block_reduce<false>(s, sh);
  double pv[1] = {s};
  if (gfk::publish_partials<1>(pv, partials, counter, gridDim.x)) {
    const double tot = gfk::fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      *result = tot;
      *counter = 0;
    }
  }
}

}  // namespace

extern "C" int gf_integrate_noalloc(int64_t n, const double *mass, const double *u,
                                    double *result, void *stream) {
  const int64_t limit = (int64_t)kMaxBlocks * kChunk;
  if (n < 0 || n > limit)
    return gf_fail(nullptr, GF_ERR_ARG,
                   "gf_integrate_noalloc: n = %lld is outside [0, %lld], the size its fixed "
                   "scratch array supports",
                   (long long)n, (long long)limit);
  if (!result || (n > 0 && (!mass || !u)))
    return gf_fail(nullptr, GF_ERR_ARG, "gf_integrate_noalloc: null pointer");
  void *addr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
  if (e != cudaSuccess || !addr)
    return gf_fail(nullptr, GF_ERR_CUDA, "gf_integrate_noalloc: cudaGetSymbolAddress: %s",
                   cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(addr, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess)
    return gf_fail(nullptr, GF_ERR_CUDA, "gf_integrate_noalloc: %s", cudaGetErrorString(e));
  const unsigned blocks = n > 0 ? (unsigned)((n + kChunk - 1) / kChunk) : 1u;
  k_integrate_noalloc<<<blocks, kThreads, 0, st>>>(n, mass, u, (double *)addr, result);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return gf_fail(nullptr, GF_ERR_CUDA, "gf_integrate_noalloc: %s", cudaGetErrorString(e));
  return GF_OK;
}

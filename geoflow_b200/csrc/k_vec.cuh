// k_vec.cuh -- reductions and elementwise helpers.
//
// Reductions are deterministic: a fixed grid, each thread folds its
// grid-stride elements in order, blocks reduce in a fixed tree, and the
// last block to finish (ticket counter) folds the block partials in block
// order.  Re-running with the same inputs gives the same bits.
#pragma once
#include "gf_common.cuh"

__device__ __forceinline__ double __fadd_rn_t(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float __fadd_rn_t(float a, float b) { return __fadd_rn(a, b); }

namespace gfk {

constexpr int RED_THREADS = 256;

// Sum (or max) over the block; result valid in thread 0.
template <bool MAX>
__device__ __forceinline__ double block_reduce(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_down_sync(0xffffffffu, v, o);
    v = MAX ? fmax(v, w) : v + w;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (warp == 0) {
    v = lane < nw ? sh[lane] : (MAX ? 0.0 : 0.0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_down_sync(0xffffffffu, v, o);
      v = MAX ? fmax(v, w) : v + w;
    }
  }
  __syncthreads();
  return v;
}

// Publishes NV block partials and returns true in the last block to
// arrive; that block then sees every partial.
template <int NV>
__device__ __forceinline__ bool publish_partials(const double (&v)[NV], double *partials,
                                                 unsigned int *counter, int stride) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) partials[k * stride + blockIdx.x] = v[k];
    __threadfence();
    unsigned int ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// In the last block: fold partials[k*stride + 0..nblk) in block order.
template <bool MAX>
__device__ __forceinline__ double fold_partials(const double *partials, int nblk, double *sh) {
  double v = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    double w = ((volatile const double *)partials)[b];
    v = MAX ? fmax(v, w) : v + w;
  }
  return block_reduce<MAX>(v, sh);
}

// y = a*x + b*y (saxpby of GMTK, gmtk.ipp:1159-1205 with roles as named)
template <typename T>
__global__ void k_axpby(int64_t n, T a, const T *__restrict__ x, T b, T *__restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

template <typename T>
__global__ void k_pointprod(int64_t n, const T *__restrict__ a, const T *__restrict__ x,
                            T *__restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a[i] * x[i];
}

template <typename TO, typename TI>
__global__ void k_convert(int64_t n, const TI *__restrict__ x, TO *__restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (TO)x[i];
}

// integral sum_i mass_i u_i (GGrid::integrate): partial sums; last block
// writes out[0].
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
    k_integrate(int64_t n, const double *__restrict__ mass, const T *__restrict__ u,
                double *partials, unsigned int *counter, double *out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += mass[i] * (double)u[i];
  s = block_reduce<false>(s, sh);
  double v[1] = {s};
  if (publish_partials<1>(v, partials, counter, gridDim.x)) {
    double tot = fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      out[0] = tot;
      *counter = 0;
    }
  }
}

// ---- GMTK::constrain2sphere (2) (blas/gmtk.ipp:2957-2976) ----
// In place, in the reference's order: v0 first, then v1 from the updated
// v0, then v2 from both; r^2 of node 0.  Explicit round-to-nearest
// operations keep the compiler from contracting them into FMAs, so the
// result is the reference's bit for bit.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

template <typename T>
__global__ void k_constrain2sphere(int64_t n, T *__restrict__ v0, T *__restrict__ v1,
                                   T *__restrict__ v2, const T *__restrict__ x,
                                   const T *__restrict__ y, const T *__restrict__ z) {
  const T r2 = add_rn(add_rn(mul_rn(x[0], x[0]), mul_rn(y[0], y[0])), mul_rn(z[0], z[0]));
  const T ri = div_rn(T(1), r2);
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const T xj = x[j], yj = y[j], zj = z[j];
    T a = v0[j], b = v1[j], c = v2[j];
    a = mul_rn(sub_rn(sub_rn(mul_rn(a, sub_rn(r2, mul_rn(xj, xj))), mul_rn(mul_rn(b, xj), yj)),
                      mul_rn(mul_rn(c, xj), zj)),
               ri);
    b = mul_rn(sub_rn(add_rn(mul_rn(mul_rn(-a, yj), xj), mul_rn(b, sub_rn(r2, mul_rn(yj, yj)))),
                      mul_rn(mul_rn(c, yj), zj)),
               ri);
    c = mul_rn(add_rn(sub_rn(mul_rn(mul_rn(-a, zj), xj), mul_rn(mul_rn(b, zj), yj)),
                      mul_rn(c, sub_rn(r2, mul_rn(zj, zj)))),
               ri);
    v0[j] = a;
    v1[j] = b;
    v2[j] = c;
  }
}

}  // namespace gfk

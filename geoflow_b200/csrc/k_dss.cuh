// k_dss.cuh -- direct-stiffness gather-scatter (GGFX::doOp) kernels.
//
// One thread per equivalence class: it gathers the class members in
// ascending local id, folds them exactly as the reference's reduction
// functors do (comm/ggfx.hpp:36-76: std::accumulate from 0 for Sum and
// Smooth, std::max/std::min folds from lowest()/max()), and scatters the
// result to every member.  The fold order is fixed, so FP64 results are
// bit-identical to the reference's and independent of the launch shape.
#pragma once
#include <cfloat>

#include "gf_common.cuh"
#include "k_vec.cuh"

namespace gfk {

template <typename T> struct Lim;
template <> struct Lim<double> {
  static __device__ __forceinline__ double lowest() { return -DBL_MAX; }
  static __device__ __forceinline__ double highest() { return DBL_MAX; }
};
template <> struct Lim<float> {
  static __device__ __forceinline__ float lowest() { return -FLT_MAX; }
  static __device__ __forceinline__ float highest() { return FLT_MAX; }
};

template <typename T, int OP>
__device__ __forceinline__ T class_fold(const T *__restrict__ u, const int32_t *__restrict__ mem,
                                        int32_t b, int32_t e) {
  T acc;
  if (OP == GF_DSS_SUM || OP == GF_DSS_SMOOTH) {
    acc = T(0);
    for (int32_t k = b; k < e; k++) acc = __fadd_rn_t(acc, u[mem[k]]);
    if (OP == GF_DSS_SMOOTH) acc = acc / (T)(e - b);
  } else if (OP == GF_DSS_MAX) {
    acc = Lim<T>::lowest();
    for (int32_t k = b; k < e; k++) {
      T v = u[mem[k]];
      acc = (acc < v) ? v : acc;
    }
  } else {
    acc = Lim<T>::highest();
    for (int32_t k = b; k < e; k++) {
      T v = u[mem[k]];
      acc = (v < acc) ? v : acc;
    }
  }
  return acc;
}

template <typename T, int OP>
__global__ void __launch_bounds__(256)
    k_dss_csr(T *__restrict__ u, const int32_t *__restrict__ ptr,
              const int32_t *__restrict__ mem, int64_t nclass) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nclass;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = ptr[c], e = ptr[c + 1];
    const T acc = class_fold<T, OP>(u, mem, b, e);
    for (int32_t k = b; k < e; k++) u[mem[k]] = acc;
  }
}

}  // namespace gfk

// k_maps.cuh -- element-local (E) <-> unique-node (L) index maps.
//
// The gather-scatter classes of GGFX (comm/ggfx.hpp) define the unique
// nodes.  Two device representations:
//   BoxLattice: a regular box grid (GGridBox).  The unique nodes are the
//     points of the global GLL lattice, M_d = ne_d p (+1 if the direction is
//     not periodic) per direction; the class of node (e; i,j,k) is computed
//     from the element coordinates, so no index array is read.
//   CSR: any grid; node_class[] gives E -> L and (class_ptr, members) the
//     members of each class in ascending local id.
// Both enumerate a class's members in ascending local id, the order in
// which GGFX::doOp folds them.
#pragma once
#include "gf_common.cuh"

namespace gfk {

// ---- loaders used by the element kernels: a z-line (3-d) or a point
// (2-d) of element e ----
template <typename T>
struct LoadE {  // element-local vector
  using value_type = T;
  const T *u;
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
    const T *b = u + e * (N * N * N) + j * N + i;
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = b[k * N * N];
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    return u[e * (N * N) + j * N + i];
  }
};

template <typename T>
struct LoadBox {  // unique-node vector on a box lattice
  using value_type = T;
  const T *w;
  BoxLattice L;
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
    int c[3];
    L.elem_coords(e, c);
    const int64_t base = L.g1(0, c[0], i) + L.M[0] * L.g1(1, c[1], j);
    const int64_t plane = L.M[0] * L.M[1];
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = w[base + plane * L.g1(2, c[2], k)];
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    int c[3];
    L.elem_coords(e, c);
    return w[L.g1(0, c[0], i) + L.M[0] * L.g1(1, c[1], j)];
  }
};

template <typename T>
struct LoadCsr {  // unique-node vector through node_class
  using value_type = T;
  const T *w;
  const int32_t *ncls;
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
    const int32_t *b = ncls + e * (N * N * N) + j * N + i;
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = w[b[k * N * N]];
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    return w[ncls[e * (N * N) + j * N + i]];
  }
};

}  // namespace gfk

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
  // 32-bit index arithmetic: element and lattice counts are below 2^31
  // (checked when the problem is created)
  __device__ __forceinline__ void coords32(int64_t e, int &c0, int &c1, int &c2) const {
    const unsigned ue = (unsigned)e, n0 = (unsigned)L.ne[0], n1 = (unsigned)L.ne[1];
    const unsigned r = ue / n0, q = r / n1;
    c0 = (int)(ue - r * n0);
    c1 = (int)(r - q * n1);
    c2 = (int)q;
  }
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
    int c0, c1, c2;
    coords32(e, c0, c1, c2);
    const int P = L.p, M0 = (int)L.M[0], M1 = (int)L.M[1], M2 = (int)L.M[2];
    int gx = c0 * P + i, gy = c1 * P + j;
    if (L.per[0] && gx == M0) gx = 0;
    if (L.per[1] && gy == M1) gy = 0;
    const int base = gx + M0 * gy, plane = M0 * M1;
#pragma unroll
    for (int k = 0; k < N; k++) {
      int gz = c2 * P + k;
      if (L.per[2] && gz == M2) gz = 0;
      out[k] = w[base + plane * gz];
    }
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    int c0, c1, c2;
    coords32(e, c0, c1, c2);
    const int P = L.p, M0 = (int)L.M[0], M1 = (int)L.M[1];
    int gx = c0 * P + i, gy = c1 * P + j;
    if (L.per[0] && gx == M0) gx = 0;
    if (L.per[1] && gy == M1) gy = 0;
    return w[gx + M0 * gy];
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

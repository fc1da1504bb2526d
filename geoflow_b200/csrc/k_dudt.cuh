// k_dudt.cuh -- fused right-hand side of GBurgers::dudt_impl
// (pdes/gburgers.ipp:203-257) and GAdvect::apply (sem/gadvect.ipp:58-100).
//
// Per element and per evolved component u_k, one pass computes
//   adv_k  = M sum_j c_j (dXidX_j D_j u_k)            (GAdvect::apply)
//   L u_k  = nu sum_j D_j^T (M G_jj D_j u_k)           (GHelmholtz, p = nu)
//   dudt_k = Minv (-L u_k - adv_k)                     (saxpby + GMass inverse)
// with c = prescribed velocity (pure advection), c = u (Burgers) or no
// advection (heat).  The reference gradient D_j u_k is computed once and
// shared by the advection and the diffusion terms.  Fields are staged in
// shared memory and contracted line by line as in k_tensor.cuh.
#pragma once
#include "k_dss.cuh"
#include "k_tensor.cuh"

namespace gfk {

enum { MODE_DUDT = 0, MODE_ADVECT = 1, MODE_EULER = 2 };

// MODE_EULER: the right-hand side K = dudt of each evolved component is
// not stored; the kernel stores the SSP substep's update before its Smooth
// instead, with the stage arithmetic of k_dss_rk_box_n (FUSE_EULER):
//   x = dt K + 1 uin;  x = a x + b y (if y);  x = a2 x + b2 y2 (if y2)
// (gexrk_stepper.ipp:533-780, 809-819), K rounded to T first, so the
// following Smooth gives the same bits as the fused update-and-Smooth pass.
template <typename T>
struct RKEpi {
  const T *uin[3];
  const T *y[3];
  const T *y2[3];
  T dt, a, b, a2, b2;
  int uin_is_u;  // uin[c] is the RHS input u[c]: read it from the staged copy
};

template <int N, int NF> constexpr int epb_dudt3() {
  return (160 / (N * N)) < 1 ? 1 : (160 / (N * N));
}

// Words per element slot of k_dudt3d's shared memory: NF + 2 padded
// volumes, plus (FP32, N <= 7) a pad that puts the next slot at the bank
// offset (slot words mod 32) minimising the shared-memory wavefronts of the
// x-, y- and z-line accesses of the warps that straddle two slots
// (36-thread elements at N = 6 and so on).  The residues come from
// counting the wavefronts of every warp of the block for each residue
// 0..31: N = 6: 168 -> 138 per component pass, N = 5: 140 -> 120.
template <typename T, int N, int NF> constexpr int dudt_slot() {
  constexpr int P = (N % 2) ? N : N + 1, W = (NF + 2) * N * N * P;
  constexpr int want = N == 3 ? 27 : N == 4 ? 16 : N == 5 ? 25 : N == 6 ? 28 : N == 7 ? 17 : -1;
  if (sizeof(T) != 4 || want < 0) return W;
  return W + ((want - W % 32) + 32) % 32;
}

// fields[0..NF): ADVECT: {p, c0, c1, c2}; BURGERS: {u0, u1, u2}; HEAT: {u}.
// Evolved components: ADVECT/HEAT: field 0; BURGERS: fields 0..2.
// AFF: affine elements (g.egeom), known at compile time, so the per-node
// geometry path (node indices and loads) is not compiled in.
template <typename T, int N, int EPB, int EQN, int MODE, bool AFF>
__global__ void __launch_bounds__(N *N *EPB, (sizeof(T) == 4 && MODE != MODE_EULER) ? 6 : 0)
    k_dudt3d(const __grid_constant__ Basis<T, N> B, const Geom<T> g, int64_t ne, T nu,
             const T *__restrict__ f0, const T *__restrict__ f1, const T *__restrict__ f2,
             const T *__restrict__ f3, const T *__restrict__ imass, T *__restrict__ o0,
             T *__restrict__ o1, T *__restrict__ o2, const RKEpi<T> epi) {
  constexpr int NF = EQN == GF_EQN_ADVECT ? 4 : (EQN == GF_EQN_BURGERS ? 3 : 1);
  constexpr int NC = EQN == GF_EQN_BURGERS ? 3 : 1;  // evolved components
  constexpr int P = Pad<N>::P, PLANE = N * P, VOL = N * PLANE, NN = N * N, NNN = N * N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw) + threadIdx.y * dudt_slot<T, N, NF>();
  T *sdx = s + NF * VOL, *sdy = s + (NF + 1) * VOL;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int a0 = t % N, a1 = t / N;
  const int64_t base = e * NNN;
  const T *fin[4] = {f0, f1, f2, f3};

  NodeGeom<T, 3> eg;
  eg.X[0] = eg.X[1] = eg.X[2] = eg.J = T(0);
  if (active) elem_geom<T, 3>(g, e, eg);

  // FP32 without the update epilogue: each thread keeps the fields of its
  // own z-column (i = a0, j = a1) in registers, read by the z-line and the
  // advection term instead of from shared memory (the kernel is bound by its
  // shared-memory pipe; 64 registers, 6 blocks per SM: the right-hand side
  // at 64^3 p = 5 0.748 -> 0.633 ms).  With the epilogue the extra registers
  // cost more occupancy than they save (stage 1.72 -> 1.89 ms).
  constexpr bool CREG = sizeof(T) == 4 && MODE != MODE_EULER;
  T fr[CREG ? NF : 1][N];
#pragma unroll
  for (int f = 0; f < NF; f++) {
#pragma unroll
    for (int k = 0; k < N; k++) {
      const T v = active ? fin[f][base + k * NN + t] : T(0);
      if (CREG) fr[CREG ? f : 0][k] = v;
      s[f * VOL + k * PLANE + a1 * P + a0] = v;
    }
  }
  __syncthreads();
  // field f of this thread's column at level k (registers in FP32)
  auto col = [&](int f, int k, int sidx) -> T {
    if constexpr (CREG) {
      return f == 0 ? fr[0][k] : (f == 1 ? fr[NF > 1 ? 1 : 0][k]
                                         : (f == 2 ? fr[NF > 2 ? 2 : 0][k] : fr[NF > 3 ? 3 : 0][k]));
    } else {
      return s[f * VOL + sidx];
    }
  };

#pragma unroll 1
  for (int c = 0; c < NC; c++) {
    const T *su = s + c * VOL;
    // output of component c: by selection in FP32 (48 registers, 8 blocks
    // per SM at N = 6, against 56 with the array); from a small local array
    // in FP64, where selection costs registers
    T *fout[3] = {o0, o1, o2};
    T *const oc = sizeof(T) == 8 ? fout[c] : (c == 0 ? o0 : (c == 1 ? o1 : o2));
    // x-lines (j=a0,k=a1) and y-lines (i=a0,k=a1): reference gradients
    {
      T a[N], d[N];
#pragma unroll
      for (int m = 0; m < N; m++) a[m] = su[a1 * PLANE + a0 * P + m];
      line_D<T, N>(B.D, a, d);
#pragma unroll
      for (int i = 0; i < N; i++) sdx[a1 * PLANE + a0 * P + i] = d[i];
#pragma unroll
      for (int m = 0; m < N; m++) a[m] = su[a1 * PLANE + m * P + a0];
      line_D<T, N>(B.D, a, d);
#pragma unroll
      for (int j = 0; j < N; j++) sdy[a1 * PLANE + j * P + a0] = d[j];
    }
    // z-line (i=a0, j=a1)
    T rz[N], radv[N];
    {
      T a[N];
#pragma unroll
      for (int m = 0; m < N; m++) a[m] = col(c, m, m * PLANE + a1 * P + a0);
      line_D<T, N>(B.D, a, rz);
    }
    __syncthreads();
    {
      const int i = a0, j = a1;
#pragma unroll
      for (int k = 0; k < N; k++) {
        const int sidx = k * PLANE + j * P + i;
        NodeGeom<T, 3> ng = eg;
        if (!AFF && active) node_geom<T, 3>(g, base + k * NN + j * N + i, ng);
        const T mass = B.W[k] * B.W[j] * B.W[i] * ng.J;
        if (EQN != GF_EQN_HEAT) {
          const int cb = EQN == GF_EQN_ADVECT ? 1 : 0;
          T po = (sdx[sidx] * ng.X[0]) * col(cb + 0, k, sidx);
          po += (sdy[sidx] * ng.X[1]) * col(cb + 1, k, sidx);
          po += (rz[k] * ng.X[2]) * col(cb + 2, k, sidx);
          radv[k] = po * mass;
        } else {
          radv[k] = T(0);
        }
        rz[k] = mass * (rz[k] * (ng.X[2] * ng.X[2]));
      }
    }
    if (MODE == MODE_ADVECT) {
      if (active) {
#pragma unroll
        for (int k = 0; k < N; k++) oc[base + k * NN + a1 * N + a0] = radv[k];
      }
      __syncthreads();
      continue;
    }
    __syncthreads();
    // x-lines of Dx^T (M G0 dx), in place
    {
      const int j = a0, k = a1;
      T a[N], d[N];
#pragma unroll
      for (int m = 0; m < N; m++) {
        NodeGeom<T, 3> ng = eg;
        if (!AFF && active) node_geom<T, 3>(g, base + k * NN + j * N + m, ng);
        const T mass = B.W[k] * B.W[j] * B.W[m] * ng.J;
        a[m] = mass * (sdx[k * PLANE + j * P + m] * (ng.X[0] * ng.X[0]));
      }
      line_DT<T, N>(B.D, a, d);
#pragma unroll
      for (int i = 0; i < N; i++) sdx[k * PLANE + j * P + i] = d[i];
    }
    // y-lines of Dy^T (M G1 dy), in place
    {
      const int i = a0, k = a1;
      T a[N], d[N];
#pragma unroll
      for (int m = 0; m < N; m++) {
        NodeGeom<T, 3> ng = eg;
        if (!AFF && active) node_geom<T, 3>(g, base + k * NN + m * N + i, ng);
        const T mass = B.W[k] * B.W[m] * B.W[i] * ng.J;
        a[m] = mass * (sdy[k * PLANE + m * P + i] * (ng.X[1] * ng.X[1]));
      }
      line_DT<T, N>(B.D, a, d);
#pragma unroll
      for (int j = 0; j < N; j++) sdy[k * PLANE + j * P + i] = d[j];
    }
    __syncthreads();
    {
      const int i = a0, j = a1;
      T d[N];
      line_DT<T, N>(B.D, rz, d);
      if (active) {
#pragma unroll
        for (int k = 0; k < N; k++) {
          const int sidx = k * PLANE + j * P + i;
          const int64_t node = base + k * NN + j * N + i;
          T L = (sdx[sidx] + sdy[sidx]) + d[k];
          if (nu != T(1)) L *= nu;
          T rhs = T(-1) * L + T(-1) * radv[k];
          const T K = imass[node] * rhs;
          if (MODE == MODE_EULER) {
            // component pointers by selection (no local-memory copy of epi)
            const T *ui = c == 0 ? epi.uin[0] : (c == 1 ? epi.uin[1] : epi.uin[2]);
            const T *yc = c == 0 ? epi.y[0] : (c == 1 ? epi.y[1] : epi.y[2]);
            const T *y2c = c == 0 ? epi.y2[0] : (c == 1 ? epi.y2[1] : epi.y2[2]);
            const T uv = epi.uin_is_u ? col(c, k, sidx) : ui[node];
            oc[node] = rk_euler_point(K, epi.dt, uv, epi.a, yc, epi.b, epi.a2, y2c, epi.b2,
                                           node);
          } else {
            oc[node] = K;
          }
        }
      }
    }
    __syncthreads();
  }
}

// 2-d variant, one thread per node.
template <typename T, int N, int EPB, int EQN, int MODE>
__global__ void __launch_bounds__(N *N *EPB)
    k_dudt2d(const __grid_constant__ Basis<T, N> B, const Geom<T> g, int64_t ne, T nu,
             const T *__restrict__ f0, const T *__restrict__ f1, const T *__restrict__ f2,
             const T *__restrict__ f3, const T *__restrict__ imass, T *__restrict__ o0,
             T *__restrict__ o1, T *__restrict__ o2, const RKEpi<T> epi) {
  (void)epi;  // the 2-d kernel has no fused update (MODE_EULER is 3-d only)
  constexpr int NF = EQN == GF_EQN_ADVECT ? 3 : (EQN == GF_EQN_BURGERS ? 2 : 1);
  constexpr int NC = EQN == GF_EQN_BURGERS ? 2 : 1;
  constexpr int P = Pad<N>::P, AREA = N * P, NN = N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw) + threadIdx.y * (NF + 2) * AREA;
  T *sgx = s + NF * AREA, *sgy = s + (NF + 1) * AREA;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int i = t % N, j = t / N;
  const int64_t node = e * NN + t;
  const T *fin[3] = {f0, f1, f2};
  T *fout[2] = {o0, o1};
  (void)f3;
  NodeGeom<T, 2> ng;
  ng.X[0] = ng.X[1] = ng.J = T(0);
  if (active) {
    elem_geom<T, 2>(g, e, ng);
    node_geom<T, 2>(g, node, ng);
  }
#pragma unroll
  for (int f = 0; f < NF; f++) s[f * AREA + j * P + i] = active ? fin[f][node] : T(0);
  const T mass = B.W[j] * B.W[i] * ng.J;
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < NC; c++) {
    const T *su = s + c * AREA;
    T dx = B.D[i] * su[j * P];
    T dy = B.D[j] * su[i];
#pragma unroll
    for (int m = 1; m < N; m++) {
      dx = fma(B.D[i + m * N], su[j * P + m], dx);
      dy = fma(B.D[j + m * N], su[m * P + i], dy);
    }
    T adv = T(0);
    if (EQN != GF_EQN_HEAT) {
      const int cb = EQN == GF_EQN_ADVECT ? 1 : 0;
      T po = (dx * ng.X[0]) * s[(cb + 0) * AREA + j * P + i];
      po += (dy * ng.X[1]) * s[(cb + 1) * AREA + j * P + i];
      adv = po * mass;
    }
    if (MODE == MODE_ADVECT) {
      if (active) fout[c][node] = adv;
      continue;
    }
    sgx[j * P + i] = mass * (dx * (ng.X[0] * ng.X[0]));
    sgy[j * P + i] = mass * (dy * (ng.X[1] * ng.X[1]));
    __syncthreads();
    T ox = B.D[i * N] * sgx[j * P];
    T oy = B.D[j * N] * sgy[i];
#pragma unroll
    for (int m = 1; m < N; m++) {
      ox = fma(B.D[m + i * N], sgx[j * P + m], ox);
      oy = fma(B.D[m + j * N], sgy[m * P + i], oy);
    }
    __syncthreads();
    if (active) {
      T L = ox + oy;
      if (nu != T(1)) L *= nu;
      T rhs = T(-1) * L + T(-1) * adv;
      fout[c][node] = imass[node] * rhs;
    }
  }
}

}  // namespace gfk

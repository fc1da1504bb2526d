// k_helm_k1.cuh -- 3-d Helmholtz apply for affine elements with a scalar
// Laplacian coefficient (GGridBox and every other grid whose elements are
// parallelepipeds: dXi/dX and Jac constant per element).
//
// GHelmholtz::reg_prod (sem/ghelmholtz.ipp:309-378) computes, per
// direction d, D_d^T (M G_d D_d u) with M = W_i W_j W_k Jac and
// G_d = (dXi_d/dX_d)^2.  For affine elements G_d and Jac are constant in
// the element, so along a line in direction d the chain D^T diag(W) D is a
// fixed 1-d matrix
//     K1 = D^T diag(W) D            (symmetric, centro-symmetric)
// times a per-line constant (e.g. Jac G_x W_j W_k for an x-line).  One
// contraction per direction replaces the two of the reference (D, then
// D^T): 3 N fused multiply-adds per node instead of 6 N.  K1 is applied in
// even-odd form (K1(N-1-i, N-1-m) = K1(i,m)), which halves it again:
//     e_m = a_m + a_{N-1-m},  o_m = a_m - a_{N-1-m}          (m < N/2)
//     S_i = sum_m Ke(i,m) e_m,  A_i = sum_m Ko(i,m) o_m        (i < N/2)
//     y_i = S_i + A_i,  y_{N-1-i} = S_i - A_i
// with Ke/Ko = (K1(i,m) +- K1(i,N-1-m)) / 2 (and the middle row/column for
// odd N).  The (S_i, A_i) accumulators form one pair: in FP32 they run on
// the packed FP32x2 FMA of sm_100 (one instruction per two FMAs).
//
// Work per element: the z-lines (one per thread) are loaded into
// registers and shared memory; x- and y-lines are read from shared memory,
// contracted and written back; the z-line thread contracts its own line
// and sums the three directions and the mass term.
#pragma once
#include "k_tensor.cuh"

namespace gfk {

template <typename T> struct Pair2;
template <> struct Pair2<float> { using type = float2; };
template <> struct Pair2<double> { using type = double2; };

// acc = a * b + acc (componentwise)
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 pfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) {
  return make_double2(a.x * b.x, a.y * b.y);
}

// Even-odd form of K1 = D^T diag(W) D plus the GLL weights.  K1 itself is
// built once per problem (gf_k1_matrix, api_setup.cu).
template <typename T, int N>
struct K1Basis {
  static constexpr int H = N / 2, MID = (N - 1) / 2;
  typename Pair2<T>::type KP[H * H > 0 ? H * H : 1];  // {Ke(i,m), Ko(i,m)}, i,m < H
  T Kcol[H > 0 ? H : 1];  // odd N: K1(i, MID), i < H
  T Krow[H > 0 ? H : 1];  // odd N: K1(MID, m), m < H
  T Kmm;                  // odd N: K1(MID, MID)
  T W[N];
};

template <typename T, int N>
inline K1Basis<T, N> make_k1basis(const gf_problem *p) {
  constexpr int H = N / 2, MID = (N - 1) / 2;
  const double *K = p->K1;  // K(l,m) = K[l + m*N]
  auto k = [&](int l, int m) { return K[l + m * N]; };
  K1Basis<T, N> b{};
  for (int i = 0; i < H; i++)
    for (int m = 0; m < H; m++) {
      b.KP[i * H + m].x = (T)(0.5 * (k(i, m) + k(i, N - 1 - m)));
      b.KP[i * H + m].y = (T)(0.5 * (k(i, m) - k(i, N - 1 - m)));
    }
  if (N % 2) {
    for (int i = 0; i < H; i++) {
      b.Kcol[i] = (T)k(i, MID);
      b.Krow[i] = (T)k(MID, i);
    }
    b.Kmm = (T)k(MID, MID);
  }
  for (int i = 0; i < N; i++) b.W[i] = (T)p->W[i];
  return b;
}

// y = c * K1 a along one line
template <typename T, int N>
__device__ __forceinline__ void line_K1(const K1Basis<T, N> &B, const T (&a)[N], T c, T (&y)[N]) {
  using P2 = typename Pair2<T>::type;
  constexpr int H = N / 2, MID = (N - 1) / 2;
  P2 eo[H > 0 ? H : 1];
#pragma unroll
  for (int m = 0; m < H; m++) {
    eo[m].x = a[m] + a[N - 1 - m];
    eo[m].y = a[m] - a[N - 1 - m];
  }
#pragma unroll
  for (int i = 0; i < H; i++) {
    P2 acc = pmul(B.KP[i * H], eo[0]);
#pragma unroll
    for (int m = 1; m < H; m++) acc = pfma(B.KP[i * H + m], eo[m], acc);
    if (N % 2) acc.x = fma(B.Kcol[i], a[MID], acc.x);
    const T s = acc.x * c;
    y[i] = fma(acc.y, c, s);
    y[N - 1 - i] = fma(-acc.y, c, s);
  }
  if (N % 2) {
    T s = B.Kmm * a[MID];
#pragma unroll
    for (int m = 0; m < H; m++) s = fma(B.Krow[m], eo[m].x, s);
    y[MID] = s * c;
  }
}

template <int N> constexpr int epb_k1() {
  return (256 / (N * N)) < 1 ? 1 : (256 / (N * N));
}

// uo = p * sum_d D_d^T (M G_d D_d u) + q M u   (qvec: per-node q)
// for affine elements; T arithmetic, LD::value_type input, TO output.
template <typename T, int N, int EPB, class LD, typename TO = T>
__global__ void __launch_bounds__(N *N *EPB)
    k_helm3d_k1(const __grid_constant__ K1Basis<T, N> B, const T *__restrict__ egeom, int64_t ne,
                T p, T q, const T *__restrict__ qvec, int use_mass, const LD ld,
                TO *__restrict__ uo, const double *__restrict__ stop) {
  if (stop && stop[0] != 0.0) return;
  constexpr int P = Pad<N>::P, PLANE = N * P, VOL = N * PLANE, NN = N * N, NNN = N * N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *su = reinterpret_cast<T *>(smem_raw) + threadIdx.y * 2 * VOL;
  T *sr = su + VOL;
  // FP32 at N = 8: rows of 8 at stride 8 in planes of 72 words, the two
  // 16-byte halves of rows 4..7 swapped (an XOR swizzle), so that an x-line
  // moves as two 128-bit accesses and both these and the scalar y-/z-line
  // accesses are free of bank conflicts; otherwise rows at stride P.
  constexpr bool VX = sizeof(T) == 4 && N == 8;
  constexpr int RS = VX ? N : P;
  auto at = [](int k, int r, int c) {
    return k * PLANE + r * RS + (VX ? (c ^ (r & 4)) : c);
  };
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int a0 = t % N, a1 = t / N;
  const int64_t base = e * NNN;

  // per-line constants: x-line (j=a0,k=a1), y-line (i=a0,k=a1), z-line
  // (i=a0,j=a1) all carry W_a0 W_a1
  T cx = T(0), cy = T(0), cz = T(0), cm = T(0);
  if (active) {
    const T *ge = egeom + e * 4;
    const T J = ge[3], w2 = B.W[a0] * B.W[a1], pj = p * J * w2;
    cx = pj * (ge[0] * ge[0]);
    cy = pj * (ge[1] * ge[1]);
    cz = pj * (ge[2] * ge[2]);
    cm = (qvec ? T(1) : q) * J * w2;
  }

  T ru[N];
  if (active) {
    typename LD::value_type lv[N];
    ld.template zline<N>(e, a0, a1, lv);
#pragma unroll
    for (int k = 0; k < N; k++) ru[k] = (T)lv[k];
  } else {
#pragma unroll
    for (int k = 0; k < N; k++) ru[k] = T(0);
  }
#pragma unroll
  for (int k = 0; k < N; k++) su[at(k, a1, a0)] = ru[k];
  __syncthreads();
  T ax[N], ay[N];
  if constexpr (VX) {
    // logical half h of row a0 is physical half h ^ sw; each thread takes
    // its own first half first, which keeps each quarter warp on 32 banks
    const int sw = (a0 >> 2) & 1;
    const float4 *row = reinterpret_cast<const float4 *>(su + a1 * PLANE + a0 * RS);
    const float4 h0 = row[sw], h1 = row[sw ^ 1];
    ax[0] = h0.x, ax[1] = h0.y, ax[2] = h0.z, ax[3] = h0.w;
    ax[4] = h1.x, ax[5] = h1.y, ax[6] = h1.z, ax[7] = h1.w;
  } else {
#pragma unroll
    for (int m = 0; m < N; m++) ax[m] = su[at(a1, a0, m)];
  }
#pragma unroll
  for (int m = 0; m < N; m++) ay[m] = su[at(a1, m, a0)];
  __syncthreads();
  {
    T y[N];
    line_K1<T, N>(B, ax, cx, y);
    if constexpr (VX) {
      const int sw = (a0 >> 2) & 1;
      float4 *row = reinterpret_cast<float4 *>(su + a1 * PLANE + a0 * RS);
      row[sw] = make_float4(y[0], y[1], y[2], y[3]);
      row[sw ^ 1] = make_float4(y[4], y[5], y[6], y[7]);
    } else {
#pragma unroll
      for (int i = 0; i < N; i++) su[at(a1, a0, i)] = y[i];
    }
    line_K1<T, N>(B, ay, cy, y);
#pragma unroll
    for (int j = 0; j < N; j++) sr[at(a1, j, a0)] = y[j];
  }
  T yz[N];
  line_K1<T, N>(B, ru, cz, yz);
  __syncthreads();
  if (active) {
#pragma unroll
    for (int k = 0; k < N; k++) {
      const int s = at(k, a1, a0);
      T o = (su[s] + sr[s]) + yz[k];
      if (use_mass) {
        const int64_t node = base + k * NN + a1 * N + a0;
        T mk = cm * B.W[k];
        if (qvec) mk *= qvec[node];
        o = fma(mk, ru[k], o);
      }
      uo[base + k * NN + a1 * N + a0] = (TO)o;
    }
  }
}

}  // namespace gfk

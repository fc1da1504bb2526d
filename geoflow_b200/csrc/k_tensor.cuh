// k_tensor.cuh -- element-local sum-factorised kernels (sm_100a).
//
// One element's n^3 (n^2 in 2-d) block is staged in shared memory.  Each
// thread owns one 1-d line of the element in turn: an x-line, a y-line and
// a z-line, so that every 1-d contraction y = D a (or D^T a) runs on a line
// held in registers, with D read from the kernel parameter block (uniform
// across the warp, so it feeds the FMAs straight from the constant bank).
// Each node therefore costs one shared-memory load per direction instead of
// n.  Rows are padded to an odd length so that x-line reads by consecutive
// threads fall in distinct banks.
//
// These kernels implement the arithmetic of GHelmholtz::reg_prod
// (sem/ghelmholtz.ipp:309-378): gdu_k = Mass (G_kk (D_k u)), uo =
// sum_k D_k^T gdu_k, times a scalar p, plus q M u.
#pragma once
#include "gf_common.cuh"
#include "k_maps.cuh"

namespace gfk {

template <int N> struct Pad { static constexpr int P = (N % 2) ? N : N + 1; };

// d[i] = sum_m D(i,m) a[m]
template <typename T, int N>
__device__ __forceinline__ void line_D(const T *__restrict__ D, const T (&a)[N], T (&d)[N]) {
#pragma unroll
  for (int i = 0; i < N; i++) {
    T s = D[i] * a[0];
#pragma unroll
    for (int m = 1; m < N; m++) s = fma(D[i + m * N], a[m], s);
    d[i] = s;
  }
}

// d[i] = sum_m D(m,i) a[m]
template <typename T, int N>
__device__ __forceinline__ void line_DT(const T *__restrict__ D, const T (&a)[N], T (&d)[N]) {
#pragma unroll
  for (int i = 0; i < N; i++) {
    T s = D[i * N] * a[0];
#pragma unroll
    for (int m = 1; m < N; m++) s = fma(D[m + i * N], a[m], s);
    d[i] = s;
  }
}

template <int N> constexpr int epb3() {
  return N <= 2 ? 32 : ((192 / (N * N)) < 1 ? 1 : (192 / (N * N)));
}
template <int N> constexpr int epb2() {
  return (256 / (N * N)) < 1 ? 1 : (256 / (N * N));
}

// Per-node geometric factors of element e at local node a.
template <typename T, int DIM>
struct NodeGeom {
  T X[DIM];  // dXidX_k
  T J;       // Jacobian
};

template <typename T, int DIM>
__device__ __forceinline__ void elem_geom(const Geom<T> &g, int64_t e, NodeGeom<T, DIM> &out) {
  if (g.egeom) {
    const T *ge = g.egeom + e * (DIM + 1);
#pragma unroll
    for (int k = 0; k < DIM; k++) out.X[k] = ge[k];
    out.J = ge[DIM];
  }
}

template <typename T, int DIM>
__device__ __forceinline__ void node_geom(const Geom<T> &g, int64_t node, NodeGeom<T, DIM> &out) {
  if (!g.egeom) {
#pragma unroll
    for (int k = 0; k < DIM; k++) out.X[k] = g.ngeom[k * g.nlocal + node];
    out.J = g.ngeom[DIM * g.nlocal + node];
  }
}

// ---------------------------------------------------------------------
// 3-d Helmholtz apply: uo = p * sum_k Dk^T M Gk Dk u + q M u
// ---------------------------------------------------------------------
// LD is the input loader (k_maps.cuh): the element-local vector itself, or
// a unique-node vector gathered through the box lattice or node_class.
// T is the arithmetic type; the input is stored as LD::value_type and the
// output as TO (FP32 storage with FP64 arithmetic keeps the apply's
// rounding at the storage level, which the mixed-precision CG relies on).
template <typename T, int N, int EPB, class LD, typename TO = T>
__global__ void __launch_bounds__(N *N *EPB)
    k_helm3d(const __grid_constant__ Basis<T, N> B, const Geom<T> g, int64_t ne, T p,
             const T *__restrict__ pvec, T q, const T *__restrict__ qvec, int use_mass,
             const LD ld, TO *__restrict__ uo, const double *__restrict__ stop) {
  if (stop && stop[0] != 0.0) return;
  constexpr int P = Pad<N>::P, PLANE = N * P, VOL = N * PLANE, NN = N * N, NNN = N * N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw) + threadIdx.y * 3 * VOL;
  T *su = s, *sgx = s + VOL, *sgy = s + 2 * VOL;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int a0 = t % N, a1 = t / N;
  const int64_t base = e * NNN;

  NodeGeom<T, 3> eg;
  eg.X[0] = eg.X[1] = eg.X[2] = eg.J = T(0);
  if (active) elem_geom<T, 3>(g, e, eg);

  // stage 0: load z-line (i=a0, j=a1) into registers and shared memory
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
  for (int k = 0; k < N; k++) su[k * PLANE + a1 * P + a0] = ru[k];
  __syncthreads();

  // stage 1: x-line (j=a0, k=a1)
  {
    const int j = a0, k = a1;
    T a[N], d[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = su[k * PLANE + j * P + m];
    line_D<T, N>(B.D, a, d);
#pragma unroll
    for (int i = 0; i < N; i++) {
      NodeGeom<T, 3> ng = eg;
      const int64_t node = base + k * NN + j * N + i;
      if (active) node_geom<T, 3>(g, node, ng);
      T gv = d[i] * (ng.X[0] * ng.X[0]);
      if (pvec && active) gv *= pvec[node];
      T mass = B.W[k] * B.W[j] * B.W[i] * ng.J;
      sgx[k * PLANE + j * P + i] = mass * gv;
    }
  }
  // stage 2: y-line (i=a0, k=a1)
  {
    const int i = a0, k = a1;
    T a[N], d[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = su[k * PLANE + m * P + i];
    line_D<T, N>(B.D, a, d);
#pragma unroll
    for (int j = 0; j < N; j++) {
      NodeGeom<T, 3> ng = eg;
      const int64_t node = base + k * NN + j * N + i;
      if (active) node_geom<T, 3>(g, node, ng);
      T gv = d[j] * (ng.X[1] * ng.X[1]);
      if (pvec && active) gv *= pvec[node];
      T mass = B.W[k] * B.W[j] * B.W[i] * ng.J;
      sgy[k * PLANE + j * P + i] = mass * gv;
    }
  }
  // stage 3: z-line (i=a0, j=a1) in registers
  T rgz[N];
  {
    const int i = a0, j = a1;
    T d[N];
    line_D<T, N>(B.D, ru, d);
#pragma unroll
    for (int k = 0; k < N; k++) {
      NodeGeom<T, 3> ng = eg;
      const int64_t node = base + k * NN + j * N + i;
      if (active) node_geom<T, 3>(g, node, ng);
      T gv = d[k] * (ng.X[2] * ng.X[2]);
      if (pvec && active) gv *= pvec[node];
      T mass = B.W[k] * B.W[j] * B.W[i] * ng.J;
      rgz[k] = mass * gv;
    }
  }
  __syncthreads();
  // stage 4: x-lines of Dx^T, in place
  {
    const int j = a0, k = a1;
    T a[N], d[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = sgx[k * PLANE + j * P + m];
    line_DT<T, N>(B.D, a, d);
#pragma unroll
    for (int i = 0; i < N; i++) sgx[k * PLANE + j * P + i] = d[i];
  }
  // stage 5: y-lines of Dy^T, in place
  {
    const int i = a0, k = a1;
    T a[N], d[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = sgy[k * PLANE + m * P + i];
    line_DT<T, N>(B.D, a, d);
#pragma unroll
    for (int j = 0; j < N; j++) sgy[k * PLANE + j * P + i] = d[j];
  }
  __syncthreads();
  // stage 6: z-lines, combine, mass term, store
  {
    const int i = a0, j = a1;
    T d[N];
    line_DT<T, N>(B.D, rgz, d);
    if (active) {
#pragma unroll
      for (int k = 0; k < N; k++) {
        const int64_t node = base + k * NN + j * N + i;
        T o = (sgx[k * PLANE + j * P + i] + sgy[k * PLANE + j * P + i]) + d[k];
        if (!pvec) o *= p;
        if (use_mass) {
          NodeGeom<T, 3> ng = eg;
          node_geom<T, 3>(g, node, ng);
          T mu = (B.W[k] * B.W[j] * B.W[i] * ng.J) * ru[k];
          mu *= qvec ? qvec[node] : q;
          o += mu;
        }
        uo[node] = (TO)o;
      }
    }
  }
}

// ---------------------------------------------------------------------
// 2-d Helmholtz apply (one thread per node)
// ---------------------------------------------------------------------
template <typename T, int N, int EPB, class LD>
__global__ void __launch_bounds__(N *N *EPB)
    k_helm2d(const __grid_constant__ Basis<T, N> B, const Geom<T> g, int64_t ne, T p,
             const T *__restrict__ pvec, T q, const T *__restrict__ qvec, int use_mass,
             const LD ld, T *__restrict__ uo, const double *__restrict__ stop) {
  if (stop && stop[0] != 0.0) return;
  constexpr int P = Pad<N>::P, AREA = N * P, NN = N * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw) + threadIdx.y * 3 * AREA;
  T *su = s, *sgx = s + AREA, *sgy = s + 2 * AREA;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int i = t % N, j = t / N;
  const int64_t node = e * NN + t;
  NodeGeom<T, 2> ng;
  ng.X[0] = ng.X[1] = ng.J = T(0);
  T uv = T(0), pv = T(1);
  if (active) {
    elem_geom<T, 2>(g, e, ng);
    node_geom<T, 2>(g, node, ng);
    uv = ld.template point2<N>(e, i, j);
    if (pvec) pv = pvec[node];
  }
  su[j * P + i] = uv;
  __syncthreads();
  T dx = B.D[i] * su[j * P];
  T dy = B.D[j] * su[i];
#pragma unroll
  for (int m = 1; m < N; m++) {
    dx = fma(B.D[i + m * N], su[j * P + m], dx);
    dy = fma(B.D[j + m * N], su[m * P + i], dy);
  }
  const T mass = B.W[j] * B.W[i] * ng.J;
  T gx = dx * (ng.X[0] * ng.X[0]);
  T gy = dy * (ng.X[1] * ng.X[1]);
  if (pvec) {
    gx *= pv;
    gy *= pv;
  }
  sgx[j * P + i] = mass * gx;
  sgy[j * P + i] = mass * gy;
  __syncthreads();
  T ox = B.D[i * N] * sgx[j * P];
  T oy = B.D[j * N] * sgy[i];
#pragma unroll
  for (int m = 1; m < N; m++) {
    ox = fma(B.D[m + i * N], sgx[j * P + m], ox);
    oy = fma(B.D[m + j * N], sgy[m * P + i], oy);
  }
  if (active) {
    T o = ox + oy;
    if (!pvec) o *= p;
    if (use_mass) {
      T mu = mass * uv;
      mu *= qvec ? qvec[node] : q;
      o += mu;
    }
    uo[node] = o;
  }
}

// ---------------------------------------------------------------------
// Single-direction reference derivative (GGrid::compute_grefderiv) and
// its physical form (GGrid::deriv): one thread per node.
// dotrans selects D^T; phys multiplies by dXidX_idir.
// ---------------------------------------------------------------------
template <typename T, int N, int DIM, int EPB>
__global__ void __launch_bounds__(N *N *(DIM == 3 ? 1 : EPB))
    k_grefderiv(const __grid_constant__ Basis<T, N> B, const Geom<T> g, int64_t ne,
                const T *__restrict__ u, int idir, int dotrans, int phys, int accum,
                T *__restrict__ du) {
  // 3-d: blockDim = (N*N) threads per element-plane loop; 2-d: (N*N, EPB)
  constexpr int NN = N * N, NE = (DIM == 3) ? NN * N : NN;
  constexpr int BPE = (DIM == 3) ? 1 : EPB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *su = reinterpret_cast<T *>(smem_raw) + threadIdx.y * NE;
  const int64_t e = (int64_t)blockIdx.x * BPE + threadIdx.y;
  const bool active = e < ne;
  const int64_t base = e * NE;
  for (int a = threadIdx.x; a < NE; a += NN) su[a] = active ? u[base + a] : T(0);
  __syncthreads();
  if (!active) return;
  NodeGeom<T, DIM> eg;
#pragma unroll
  for (int k = 0; k < DIM; k++) eg.X[k] = T(0);
  eg.J = T(0);
  elem_geom<T, DIM>(g, e, eg);
  for (int a = threadIdx.x; a < NE; a += NN) {
    int i = a % N, j = (a / N) % N, k = (DIM == 3) ? a / NN : 0;
    int c = idir == 1 ? i : (idir == 2 ? j : k);
    int stride = idir == 1 ? 1 : (idir == 2 ? N : NN);
    int b0 = a - c * stride;
    T s = T(0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      T Dv = dotrans ? B.D[m + c * N] : B.D[c + m * N];
      s = (m == 0) ? Dv * su[b0] : fma(Dv, su[b0 + m * stride], s);
    }
    if (phys) {
      NodeGeom<T, DIM> ng = eg;
      node_geom<T, DIM>(g, base + a, ng);
      s *= ng.X[idir - 1];
    }
    du[base + a] = accum ? du[base + a] + s : s;
  }
}

}  // namespace gfk

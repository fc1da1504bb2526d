// k_def.cuh -- operators on deformed (GE_DEFORMED) and 2-d embedded
// (GE_2DEMBEDDED) elements, where the metric is a full per-node matrix:
//   GHelmholtz::def_prod / embed_prod (sem/ghelmholtz.ipp:109-293)
//     uo = p sum_j D_j^T (sum_i G_ij D_i u) + q M u,
//     G_ij = sum_k dXi_i/dX_k dXi_j/dX_k W Jac   (def_init, 416-519)
//   GGrid::deriv, deformed branch (grid/ggrid.ipp:1177-1186)
//     du/dx_k = sum_j dXi_j/dX_k D_j u,  k < nxy
//   GAdvect::apply (sem/gadvect.ipp:58-100) with nxy velocity components
//   GBurgers::dudt_impl (pdes/gburgers.ipp:203-257) built from them.
// One element per block; the element's values, its reference gradient and
// the metric-weighted gradient live in shared memory, and threads stride
// over the element's nodes in each pass.  The reference gradient is
// computed once and shared by the diffusion and advection terms.
#pragma once
#include "k_maps.cuh"
#include "k_tensor.cuh"

namespace gfk {

template <typename T>
struct DefGeom {
  const T *X;  // dim*nxy planes, plane i*nxy + k = dXi_i/dX_k
  const T *G;  // packed symmetric metric with W and Jac: (00,01[,02],11[,12],22)
  const T *J;  // Jacobian plane
  int nxy;     // physical coordinates (dim, or 3 on an embedded surface)
  int64_t nlocal;
};

__device__ __forceinline__ int gpack(int i, int j, int dim) {
  if (i > j) {
    const int t = i;
    i = j;
    j = t;
  }
  return dim == 2 ? (i == 0 ? j : 2) : (i == 0 ? j : (i == 1 ? 2 + j : 5));
}

template <typename T> inline DefGeom<T> def_of(const gf_problem *p);
template <> inline DefGeom<double> def_of<double>(const gf_problem *p) {
  return DefGeom<double>{p->dgeom_d, p->gmet_d, p->ngeom_d + (int64_t)p->dim * p->nlocal, p->nxy,
                         p->nlocal};
}
template <> inline DefGeom<float> def_of<float>(const gf_problem *p) {
  return DefGeom<float>{p->dgeom_f, p->gmet_f, p->ngeom_f + (int64_t)p->dim * p->nlocal, p->nxy,
                        p->nlocal};
}

enum { DEF_HELM = 0, DEF_DUDT = 1, DEF_ADVECT = 2, DEF_DERIV = 3 };

// mode DEF_HELM: uo = p L u (+ q M u); DEF_DUDT: uo = Minv(-nu L u - adv)
// (heat when nv == 0); DEF_ADVECT: uo = adv = M sum_k c_k du/dx_k;
// DEF_DERIV: uo = du/dx_{idir}.  nv velocity components c0..c2.
// The threads that share one element: the whole block (k_def), or a group
// of lanes of one warp (the ensemble kernels, api_ensemble.cu).
struct BlockTeam {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct LaneTeam {
  int r, n;
  unsigned mask;  // the team's lanes
  __device__ __forceinline__ int rank() const { return r; }
  __device__ __forceinline__ int size() const { return n; }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// Where an element body writes node values: a plain array (OutPtr), or a
// policy that finishes the value there (the ensemble's stage epilogue).
template <typename TO>
struct OutPtr {
  TO *__restrict__ p;
  __device__ __forceinline__ void operator()(int64_t node, TO v) const { p[node] = v; }
};

// One element e of k_def, by the threads of team tm (the body shared by
// k_def and the ensemble kernels).  BB is a basis with members D[N*N] and
// W[N]; smem holds (1 + 2 DIM) N^DIM values of T.  Each node's arithmetic
// is the same whichever thread of whichever team computes it.
template <typename T, int N, int DIM, class LD, typename TO, class BB, class TM, class OUT>
__device__ __forceinline__ void def_element(const TM &tm, const BB &B, const DefGeom<T> &g,
                                            int64_t e, int mode,
                                            T p, const T *__restrict__ pvec, T q,
                                            const T *__restrict__ qvec, int use_mass, const LD &ld,
                                            int nv, const T *__restrict__ c0,
                                            const T *__restrict__ c1, const T *__restrict__ c2,
                                            int idir, const T *__restrict__ imass,
                                            const OUT &uo, T *smem) {
  constexpr int NN = N * N, NE = DIM == 3 ? NN * N : NN;
  T *su = smem;
  T *sd = su + NE;        // DIM planes: D_j u
  T *sg = sd + DIM * NE;  // DIM planes: sum_i G_ij D_i u
  const int64_t base = e * NE;
  const T *cv[3] = {c0, c1, c2};
  const int64_t nl = g.nlocal;
  // load
  if (DIM == 3) {
    for (int ij = tm.rank(); ij < NN; ij += tm.size()) {
      typename LD::value_type lv[N];
      ld.template zline<N>(e, ij % N, ij / N, lv);
#pragma unroll
      for (int k = 0; k < N; k++) su[k * NN + ij] = (T)lv[k];
    }
  } else {
    for (int a = tm.rank(); a < NN; a += tm.size())
      su[a] = (T)ld.template point2<N>(e, a % N, a / N);
  }
  tm.sync();
  const int st[3] = {1, N, NN};
  // reference gradient D_j u
  for (int a = tm.rank(); a < NE; a += tm.size()) {
    const int li[3] = {a % N, (a / N) % N, DIM == 3 ? a / NN : 0};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int b0 = a - li[d] * st[d];
      T s = B.D[li[d]] * su[b0];
#pragma unroll
      for (int m = 1; m < N; m++) s = fma(B.D[li[d] + m * N], su[b0 + m * st[d]], s);
      sd[d * NE + a] = s;
    }
  }
  tm.sync();
  // pointwise metric terms
  for (int a = tm.rank(); a < NE; a += tm.size()) {
    const int64_t node = base + a;
    if (mode == DEF_DERIV) {
      T du = sd[a] * g.X[(0 * g.nxy + idir - 1) * nl + node];
      for (int j = 1; j < DIM; j++) du += sd[j * NE + a] * g.X[(j * g.nxy + idir - 1) * nl + node];
      uo(node, (TO)du);
      continue;
    }
    if (mode != DEF_ADVECT) {
#pragma unroll
      for (int j = 0; j < DIM; j++) {
        T gj = T(0);
#pragma unroll
        for (int i = 0; i < DIM; i++) gj += sd[i * NE + a] * g.G[gpack(i, j, DIM) * nl + node];
        if (mode == DEF_HELM && pvec) gj *= pvec[node];
        sg[j * NE + a] = gj;
      }
    }
    if (mode == DEF_ADVECT || (mode == DEF_DUDT && nv > 0)) {
      const int li[3] = {a % N, (a / N) % N, DIM == 3 ? a / NN : 0};
      T mass = B.W[li[0]] * B.W[li[1]];
      if (DIM == 3) mass *= B.W[li[2]];
      mass *= g.J[node];
      T po = T(0);
      for (int k = 0; k < nv; k++) {
        T dk = sd[a] * g.X[(0 * g.nxy + k) * nl + node];
        for (int j = 1; j < DIM; j++) dk += sd[j * NE + a] * g.X[(j * g.nxy + k) * nl + node];
        dk *= cv[k][node];
        po = k == 0 ? dk : po + dk;
      }
      po *= mass;
      if (mode == DEF_ADVECT) {
        uo(node, (TO)po);
        continue;
      }
      su[a] = po;  // u itself is no longer needed by the rhs
    }
  }
  if (mode == DEF_ADVECT || mode == DEF_DERIV) return;
  tm.sync();
  // transposed divergence sum_j D_j^T g_j, then the mode's combination
  for (int a = tm.rank(); a < NE; a += tm.size()) {
    const int64_t node = base + a;
    const int li[3] = {a % N, (a / N) % N, DIM == 3 ? a / NN : 0};
    T o = T(0);
#pragma unroll
    for (int j = 0; j < DIM; j++) {
      const int b0 = a - li[j] * st[j];
      T s = B.D[li[j] * N] * sg[j * NE + b0];
#pragma unroll
      for (int m = 1; m < N; m++) s = fma(B.D[m + li[j] * N], sg[j * NE + b0 + m * st[j]], s);
      o = j == 0 ? s : o + s;
    }
    if (mode == DEF_HELM) {
      if (!pvec) o *= p;
      if (use_mass) {
        T mass = B.W[li[0]] * B.W[li[1]];
        if (DIM == 3) mass *= B.W[li[2]];
        T t = (mass * g.J[node]) * su[a];
        t *= qvec ? qvec[node] : q;
        o += t;
      }
      uo(node, (TO)o);
    } else {  // DEF_DUDT
      o *= p;  // p = nu
      const T r = nv > 0 ? T(-1) * o + T(-1) * su[a] : T(-1) * o;
      uo(node, (TO)(imass[node] * r));
    }
  }
}

// ---- pure advection with a prescribed velocity and no diffusion ----
// GBurgers::dudt_impl's pure-advection branch (pdes/gburgers.ipp:237-245)
// with nu = 0 reduces to dudt = -M^-1 M sum_k c_k du/dx_k
//   = b_0 D_0 u + b_1 D_1 u,   b_j = -(imass M) sum_k c_k dXi_j/dX_k,
// and c is fixed over a step_b advance, so the steppers form b_0, b_1 once
// per advance (adv_coef_point) and every RHS call reads 2 planes per node
// instead of the 2 nxy metric planes, nxy velocity components, Jac, the
// metric G and the inverse mass.  (The diffusion term nu L u vanishes at
// nu = 0 but for the sign of a zero.)  Rounding differs from the general
// kernel's order; both steppers use these same functions, so the ensemble
// and gf_rk_advance agree bit for bit.
template <typename T>
__device__ __forceinline__ void adv_coef_point(int64_t node, int li0, int li1, const T *W,
                                               const DefGeom<T> &g, const T *c0, const T *c1,
                                               const T *c2, const T *imass, T &b0, T &b1) {
  const int64_t nl = g.nlocal;
  const T *cv[3] = {c0, c1, c2};
  T a[2];
#pragma unroll
  for (int j = 0; j < 2; j++) {
    T s = g.X[(j * g.nxy + 0) * nl + node] * cv[0][node];
    for (int k = 1; k < g.nxy; k++) s = fma(g.X[(j * g.nxy + k) * nl + node], cv[k][node], s);
    a[j] = s;
  }
  T mass = W[li0] * W[li1];
  mass *= g.J[node];
  const T f = -(imass[node] * mass);
  b0 = f * a[0];
  b1 = f * a[1];
}

// One 2-d element of the advection right-hand side from the coefficient
// planes (team tm; smem holds N^2 values).
template <typename T, int N, class LD, class BB, class TM, class OUT>
__device__ __forceinline__ void adv_element(const TM &tm, const BB &B, int64_t e, const LD &ld,
                                            const T *__restrict__ b0, const T *__restrict__ b1,
                                            const OUT &out, T *su) {
  constexpr int NN = N * N;
  const int64_t base = e * NN;
#pragma unroll 4
  for (int a = tm.rank(); a < NN; a += tm.size())
    su[a] = (T)ld.template point2<N>(e, a % N, a / N);
  tm.sync();
#pragma unroll 4
  for (int a = tm.rank(); a < NN; a += tm.size()) {
    const int i = a % N, j = a / N;
    const T c0 = b0[base + a], c1 = b1[base + a];
    T d0 = B.D[i] * su[j * N];
    T d1 = B.D[j] * su[i];
#pragma unroll
    for (int m = 1; m < N; m++) {
      d0 = fma(B.D[i + m * N], su[j * N + m], d0);
      d1 = fma(B.D[j + m * N], su[m * N + i], d1);
    }
    out(base + a, fma(c1, d1, c0 * d0));
  }
}

template <typename T, int N, int DIM, class LD, typename TO>
__global__ void __launch_bounds__(256)
    k_def(const __grid_constant__ Basis<T, N> B, const DefGeom<T> g, int64_t ne, int mode, T p,
          const T *__restrict__ pvec, T q, const T *__restrict__ qvec, int use_mass, const LD ld,
          int nv, const T *__restrict__ c0, const T *__restrict__ c1, const T *__restrict__ c2,
          int idir, const T *__restrict__ imass, TO *__restrict__ uo,
          const double *__restrict__ stop) {
  if (stop && stop[0] != 0.0) return;
  extern __shared__ __align__(16) unsigned char smem_def[];
  const int64_t e = blockIdx.x;
  if (e >= ne) return;
  def_element<T, N, DIM, LD, TO>(BlockTeam{}, B, g, e, mode, p, pvec, q, qvec, use_mass, ld, nv, c0,
                                 c1, c2, idir, imass, OutPtr<TO>{uo},
                                 reinterpret_cast<T *>(smem_def));
}

// The coefficient planes of adv_element on one 2-d problem (one thread per
// node).
template <typename T, int N>
__global__ void k_adv_coef(const __grid_constant__ Basis<T, N> B, const DefGeom<T> g,
                           const T *__restrict__ c0, const T *__restrict__ c1,
                           const T *__restrict__ c2, const T *__restrict__ imass,
                           T *__restrict__ b0, T *__restrict__ b1) {
  for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < g.nlocal;
       node += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(node % (N * N));
    adv_coef_point<T>(node, a % N, a / N, B.W, g, c0, c1, c2, imass, b0[node], b1[node]);
  }
}

// adv_element on one 2-d problem: one element per warp, four per block.
template <typename T, int N, class LD>
__global__ void __launch_bounds__(128)
    k_adv_def(const __grid_constant__ Basis<T, N> B, int64_t ne, const LD ld,
              const T *__restrict__ b0, const T *__restrict__ b1, T *__restrict__ out) {
  __shared__ T su[4][N * N];
  const int w = threadIdx.x >> 5;
  const int64_t e = (int64_t)blockIdx.x * 4 + w;
  if (e >= ne) return;  // whole warps
  adv_element<T, N>(LaneTeam{(int)(threadIdx.x & 31), 32, 0xffffffffu}, B, e, ld, b0, b1,
                    OutPtr<T>{out}, su[w]);
}

}  // namespace gfk

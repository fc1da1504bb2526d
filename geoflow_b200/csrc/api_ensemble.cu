// api_ensemble.cu -- ensembles of independent problems advanced together:
// one persistent launch per RK stage (2-d deformed and embedded members,
// e.g. icosahedral-sphere advection cases) or per CG iteration (2-d box
// Helmholtz members: FP32 iterations, FP64 residuals and refinement).  The
// reference runs one problem per process; nothing here has a reference
// counterpart beyond the per-member arithmetic named below.
//
// Work lists.  Element work is cut into chunks of one warp: the warp splits
// into teams of `team` lanes (8, 16 or 32), one element per team, so a
// chunk holds 32/team elements of one member.  The chunks of all members
// are numbered consecutively and the warps of the grid take them round
// robin, which spreads every member evenly over the GPU whatever its size
// and order.  Node work is numbered the same way: one thread per
// gather-scatter class of every member (RK), or warp slices of 256 lattice
// nodes of every member (CG), so a slice's warp owns the same nodes in
// every phase and writes one partial sum per slice.
//
// Phases inside one launch are separated by a grid barrier (an arrival
// count and a generation word; the spin is bounded and records a timeout
// instead of waiting for ever).  The kernels are launched cooperatively,
// so all blocks are resident.  The last block to reach a reducing barrier
// folds each member's slice partials in slice order and forms the member's
// CG scalars before it releases the others: the scalars are deterministic
// and do not depend on the launch shape.
//
// Arithmetic.  An RK member's element body is def_element (k_def.cuh), its
// folds are those of k_dss_rk_split / k_dss_split and its stage sums those of
// step_b (rk_stage_point), so each member advances bit for bit as
// gf_rk_advance advances it alone.  A CG member runs GCG::solve_impl's DFM
// iteration (solvers/gcg.ipp:239-382) with a Jacobi preconditioner on the
// unique lattice nodes: FP32 vectors and applies, FP64 dot products, and
// restarted refinement, x += d and r = mask DSS_Sum(b - A x) in FP64 each
// time an FP32 run has reduced its residual by inner_tol.  The CG member is
// the masked (homogeneous Dirichlet) solve, solve_impl (2) with xb = 0: the
// form without xb leaves bbv_ unset and masks nothing.
//
// Tile shapes (threads per block, blocks per SM, team width per order) are
// chosen by gf_ensemble_tune, which times the element phase of candidate
// shapes on the ensemble's own data.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gf_common.cuh"
#include "k_def.cuh"
#include "k_dss.cuh"
#include "k_vec.cuh"
#include "rk_common.cuh"

using namespace gfk;

namespace {

constexpr int EN_MINN = 3, EN_MAXN = 10;  // members of order 2..9
constexpr int EN_MAXMEM = 64;
constexpr unsigned EN_SPIN_LIMIT = 1u << 21;
constexpr int EN_WS = 256;  // lattice nodes per warp slice (CG)

enum { EN_REFINE = 0, EN_INNER = 1, EN_DONE = 2 };

struct EnMember {
  int N, nxy, team, epw;
  int64_t ne, nlocal, nclass, nL;
  int64_t chunk0, nchunk, class0;
  double D[EN_MAXN * EN_MAXN], W[EN_MAXN], K1d[EN_MAXN];
  // deformed / embedded geometry, [0] FP64 and [1] FP32
  const void *X[2], *G[2], *J[2], *imass[2];
  const int32_t *class_ptr, *members;
  const int32_t *sh_ptr, *sh_members;  // classes of several members (shared nodes)
  int64_t nshared;
  const float *imult32;                 // 1/multiplicity per node (1: a singleton class)
  // RK state: u[0] the caller's, u[1] scratch; slopes; final-stage input
  void *u[2], *K[3], *uf;
  void *advb[2];  // advection fast path: adv_element's coefficient planes
  const void *c[3];
  double coef[4][3], ch[4];
  // box lattice (CG)
  BoxWalk walk;
  int ne0;
  const uint8_t *maskL8;
  const double *egeom64;
  const float *egeom32;
  const double *bE;
  double *xE, *bL, *xL, *r64, *dinv64, *aE;
  float *dL, *r32, *w32, *q32, *dinv32;
  double *w64, *q64;  // the FP64 solve's search direction and A w
};

struct EnCG {
  double rho, alpha, beta, rnorm, rnorm64, rtol, itol, bnorm, nd;
  int next, iters, sweeps, status;
};

struct EnCtl {
  unsigned count, gen, err, launches;
  int any_active;
  int nonfinite[EN_MAXMEM];
};

struct EnArgs {
  EnMember *mem;
  int nmem;
  const int64_t *chunk_pref, *class_pref;  // nmem + 1 each
  const int64_t *sh_pref;                  // RK: shared-class prefix, nmem + 1
  int64_t nchunk, nclass, nsh;
  EnCtl *ctl;
  EnCG *cg;
  double *partials;  // [nmem][2][gridDim.x]
  int wbytes;        // dynamic shared bytes per warp
  // RK
  int ns, par, eqn, fast;
  double nu;
  // CG
  double p, q, tol, inner_tol;
  int normtype, maxit, max_refine, relative, all_inner;
  int fp64;
  unsigned launch_cap;
  cudaGraphConditionalHandle cond;
  int has_cond;
};

// ---- grid barrier -------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Every block calls it; `last` runs in the last block to arrive, with the
// whole block, before the others are released.
template <class F>
__device__ __forceinline__ void en_barrier(EnCtl *ctl, F last) {
  __shared__ unsigned s_last, s_gen;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire(&ctl->gen);
    __threadfence();
    const unsigned t = atomicAdd(&ctl->count, 1u);
    s_last = (t == gridDim.x - 1);
    s_gen = g;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    last();
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicExch(&ctl->count, 0u);
      __threadfence();
      atomicAdd(&ctl->gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    unsigned it = 0;
    while (ld_acquire(&ctl->gen) == s_gen) {
      if (++it > EN_SPIN_LIMIT || ld_acquire(&ctl->err)) {
        atomicExch(&ctl->err, 1u);
        break;
      }
      if (it > 64) __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
}

struct NoWork {
  __device__ void operator()() const {}
};

// largest m with pref[m] <= x
__device__ __forceinline__ int en_find(const int64_t *pref, int n, int64_t x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void en_load_pref(const int64_t *g, int64_t *s, int n) {
  for (int i = threadIdx.x; i <= n; i += blockDim.x) s[i] = g[i];
}

__device__ __forceinline__ unsigned team_mask(int team, int tid) {
  return team == 32 ? 0xffffffffu : (((1u << team) - 1u) << (tid * team));
}

// words of a warp's basis region (D then W), rounded to 16 bytes
template <typename T>
__host__ __device__ __forceinline__ int en_basis_words(int N) {
  const int w = N * N + N, per16 = 16 / (int)sizeof(T);
  return (w + per16 - 1) / per16 * per16;
}

template <typename T>
struct SBasis {
  const T *D, *W;
};

// ---- RK members -----------------------------------------------------------
template <typename T>
struct LoadStage {  // the step_b stage input at the element's nodes
  using value_type = T;
  const T *uin, *K0, *K1, *K2;
  T b0, b1, b2;
  int nk;
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = pt(e * (N * N * N) + (int64_t)k * N * N + j * N + i);
  }
  __device__ __forceinline__ T pt(int64_t i) const {
    return rk_stage_point(uin[i], nk, K0, K1, K2, b0, b1, b2, i);
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    return pt(e * (N * N) + j * N + i);
  }
};

template <typename T>
struct LoadL2 {  // an element-local vector written earlier in this launch
  using value_type = T;
  const T *u;
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = __ldcg(u + e * (N * N * N) + (int64_t)k * N * N + j * N + i);
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    return __ldcg(u + e * (N * N) + j * N + i);
  }
};

// The final stage's input at an element node: the stage sum (folded as a
// class of one member) where the node is its class's only member, else the
// folded value the stage-input pass left in uf.
template <typename T>
struct LoadFinal {
  using value_type = T;
  const float *imult;
  const T *uf, *uin, *K0, *K1, *K2;
  T b0, b1, b2;
  int nk;
  __device__ __forceinline__ T at(int64_t i) const {
    if (imult[i] == 1.0f)
      return __fadd_rn_t(T(0), rk_stage_point(uin[i], nk, K0, K1, K2, b0, b1, b2, i)) / T(1);
    return __ldcg(uf + i);
  }
  template <int N>
  __device__ __forceinline__ void zline(int64_t e, int i, int j, T (&out)[N]) const {
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = at(e * (N * N * N) + (int64_t)k * N * N + j * N + i);
  }
  template <int N>
  __device__ __forceinline__ T point2(int64_t e, int i, int j) const {
    return at(e * (N * N) + j * N + i);
  }
};

// The stage epilogue at an element node.  A node that is its class's only
// member is finished here (its fold is (0 + v) / 1: K = that, and uout +=
// c h K, or in the last stage uout = Smooth(uout + c h K)); a node of a
// shared class keeps the raw slope for the fold after the barrier.  The
// arithmetic is that of k_dss_rk_split, node for node.
template <typename T>
struct OutStage {
  const float *imult;
  T *K;
  const T *src;
  T *uout;
  T ch;
  int fin;
  int *nonfinite;
  __device__ __forceinline__ void operator()(int64_t i, T v) const {
    if (imult[i] != 1.0f) {
      K[i] = v;
      return;
    }
    const T acc = __fadd_rn_t(T(0), v) / T(1);
    if (!fin) {
      K[i] = acc;
      uout[i] = rk_accum_point(src[i], acc, ch);
    } else {
      const T acc2 = __fadd_rn_t(T(0), rk_accum_point(src[i], acc, ch)) / T(1);
      uout[i] = acc2;
      if (!isfinite((double)acc2)) *nonfinite = 1;
    }
  }
};

template <typename T, int N>
__device__ void en_rhs_elem(const LaneTeam &tm, const EnArgs &a, int mi, const EnMember &M,
                            int64_t e, const SBasis<T> &B, T *slice, bool fin, int stage, T nu,
                            bool fast) {
  const int par = a.par;
  T *uout = (T *)M.u[1 - par];
  const OutStage<T> out{M.imult32,
                        (T *)M.K[fin ? 0 : stage],
                        stage == 0 ? (const T *)M.u[par] : uout,
                        uout,
                        (T)M.ch[stage],
                        fin,
                        &a.ctl->nonfinite[mi]};
  const LoadStage<T> lds{(const T *)M.u[par], (const T *)M.K[0], (const T *)M.K[1],
                         (const T *)M.K[2], (T)M.coef[stage][0], (T)M.coef[stage][1],
                         (T)M.coef[stage][2], stage};
  const LoadFinal<T> ldf{M.imult32, (const T *)M.uf, lds.uin, lds.K0, lds.K1, lds.K2,
                         lds.b0, lds.b1, lds.b2, stage};
  if (fast) {  // prescribed velocity, nu = 0: adv_element on the coefficient planes
    const T *b0 = (const T *)M.advb[0], *b1 = (const T *)M.advb[1];
    if (fin)
      adv_element<T, N>(tm, B, e, ldf, b0, b1, out, slice);
    else
      adv_element<T, N>(tm, B, e, lds, b0, b1, out, slice);
    return;
  }
  constexpr int pr = sizeof(T) == 4 ? 1 : 0;
  const DefGeom<T> g{(const T *)M.X[pr], (const T *)M.G[pr], (const T *)M.J[pr], M.nxy,
                     M.nlocal};
  const T *imass = (const T *)M.imass[pr];
  const int nv = a.eqn == GF_EQN_ADVECT ? M.nxy : 0;
  const T *c0 = (const T *)M.c[0], *c1 = (const T *)M.c[1], *c2 = (const T *)M.c[2];
  if (fin)
    def_element<T, N, 2, LoadFinal<T>, T>(tm, B, g, e, DEF_DUDT, nu, nullptr, T(0), nullptr, 0,
                                          ldf, nv, c0, c1, c2, 0, imass, out, slice);
  else
    def_element<T, N, 2, LoadStage<T>, T>(tm, B, g, e, DEF_DUDT, nu, nullptr, T(0), nullptr, 0,
                                          lds, nv, c0, c1, c2, 0, imass, out, slice);
}

// Element phase of an RK stage: K_stage = dudt(stage input), or for the
// final stage K_0 = dudt(uf).
template <typename T>
__device__ void en_rk_elements(const EnArgs &a, const int64_t *cpref, bool from_uf, int stage) {
  extern __shared__ __align__(16) unsigned char en_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  T *ws = reinterpret_cast<T *>(en_smem + (size_t)wib * a.wbytes);
  const int64_t nw = (int64_t)gridDim.x * wpb;
  const T nu = (T)a.nu;
  const bool fast = a.fast != 0;
  int cur = -1;
  for (int64_t ch = (int64_t)blockIdx.x * wpb + wib; ch < a.nchunk; ch += nw) {
    const int mi = en_find(cpref, a.nmem, ch);
    const EnMember &M = a.mem[mi];
    const int N = M.N;
    if (mi != cur) {
      for (int i = lane; i < N * N; i += 32) ws[i] = (T)M.D[i];
      for (int i = lane; i < N; i += 32) ws[N * N + i] = (T)M.W[i];
      __syncwarp();
      cur = mi;
    }
    const int team = M.team, tid = lane / team;
    const int64_t e = (ch - M.chunk0) * M.epw + tid;
    if (e < M.ne) {
      const LaneTeam tm{lane - tid * team, team, team_mask(team, tid)};
      const SBasis<T> B{ws, ws + N * N};
      T *slice = ws + en_basis_words<T>(N) + tid * 5 * N * N;
      switch (N) {
        case 3: en_rhs_elem<T, 3>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 4: en_rhs_elem<T, 4>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 5: en_rhs_elem<T, 5>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 6: en_rhs_elem<T, 6>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 7: en_rhs_elem<T, 7>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 8: en_rhs_elem<T, 8>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        case 9: en_rhs_elem<T, 9>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
        default: en_rhs_elem<T, 10>(tm, a, mi, M, e, B, slice, from_uf, stage, nu, fast); break;
      }
    }
    __syncwarp();
  }
}

// The node work of an RK stage after its element phase: the classes of
// several members (shared nodes; a class of one member is finished by the
// element phase), one thread each from the problem's shared-class list
// (sh_ptr / sh_members, members in ascending local id), numbered over all
// members (prefix spref).  The fold is that of k_dss_rk_split: from 0, in
// member order, divided by the count.
template <class FC>
__device__ __forceinline__ void en_rk_items(const EnArgs &a, const int64_t *spref, FC cls) {
  const int64_t nt = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.nsh; j += nt) {
    const int mi = en_find(spref, a.nmem, j);
    const EnMember &M = a.mem[mi];
    const int64_t cl = j - spref[mi];
    cls(mi, M, M.sh_ptr[cl], M.sh_ptr[cl + 1]);
  }
}

// Final-stage input at the shared nodes: uf = Smooth(stage sum over the
// ns-1 earlier slopes) (the element phase forms it at the other nodes).
template <typename T>
__device__ void en_rk_stage_input(const EnArgs &a, const int64_t *spref, int stage) {
  en_rk_items(
      a, spref,
      [&](int, const EnMember &M, int32_t b0, int32_t e0) {
        const T *uin = (const T *)M.u[a.par];
        const T *K0 = (const T *)M.K[0], *K1 = (const T *)M.K[1], *K2 = (const T *)M.K[2];
        const T c0 = (T)M.coef[stage][0], c1 = (T)M.coef[stage][1], c2 = (T)M.coef[stage][2];
        T acc = T(0);
        for (int32_t k = b0; k < e0; k++) {
          const int64_t m = M.sh_members[k];
          acc = __fadd_rn_t(acc, rk_stage_point(uin[m], stage, K0, K1, K2, c0, c1, c2, m));
        }
        acc = acc / (T)(e0 - b0);
        T *uf = (T *)M.uf;
        for (int32_t k = b0; k < e0; k++) uf[M.sh_members[k]] = acc;
      });
}

// Fold of a stage at the shared nodes: Smooth K_stage and uout += c h K
// (stages before the last), or for the last stage uout = Smooth(uout + c h
// Smooth(K_0)) (the element phase finishes the other nodes).
template <typename T>
__device__ void en_rk_fold(const EnArgs &a, const int64_t *spref, int stage) {
  const bool fin = stage == a.ns - 1;
  en_rk_items(
      a, spref,
      [&](int mi, const EnMember &M, int32_t b0, int32_t e0) {
        const T cnt = (T)(e0 - b0), ch = (T)M.ch[stage];
        T *uout = (T *)M.u[1 - a.par];
        const T *src = stage == 0 ? (const T *)M.u[a.par] : uout;
        T *Kx = (T *)M.K[fin ? 0 : stage];
        const int32_t *mem = M.sh_members;
        T acc = T(0);
        for (int32_t k = b0; k < e0; k++) acc = __fadd_rn_t(acc, __ldcg(Kx + mem[k]));
        acc = acc / cnt;
        if (!fin) {
          for (int32_t k = b0; k < e0; k++) {
            const int64_t m = mem[k];
            Kx[m] = acc;
            uout[m] = rk_accum_point(src[m], acc, ch);
          }
        } else {
          T acc2 = T(0);
          for (int32_t k = b0; k < e0; k++)
            acc2 = __fadd_rn_t(acc2, rk_accum_point(src[mem[k]], acc, ch));
          acc2 = acc2 / cnt;
          for (int32_t k = b0; k < e0; k++) uout[mem[k]] = acc2;
          if (!isfinite((double)acc2)) a.ctl->nonfinite[mi] = 1;
        }
      });
}

// One RK stage of every member (step_b of GExRKStepper, gexrk_stepper.ipp:
// 252-341): stages before the last are RHS | fold; the last is stage input
// and Smooth | RHS | fold.  (FP32 fits 64 registers, two 512-thread blocks
// per SM; FP64 takes 110, one block, rather than spill.)
template <typename T>
__global__ void __launch_bounds__(512, sizeof(T) == 8 ? 1 : 2)
    k_en_rk_stage(EnArgs a, int stage) {
  __shared__ int64_t s_cpref[EN_MAXMEM + 1], s_spref[EN_MAXMEM + 1];
  en_load_pref(a.chunk_pref, s_cpref, a.nmem);
  en_load_pref(a.sh_pref, s_spref, a.nmem);
  __syncthreads();
  const bool fin = stage == a.ns - 1;
  if (fin) {
    en_rk_stage_input<T>(a, s_spref, stage);
    en_barrier(a.ctl, NoWork{});
  }
  en_rk_elements<T>(a, s_cpref, fin, stage);
  en_barrier(a.ctl, NoWork{});
  en_rk_fold<T>(a, s_spref, stage);
}

// element phase alone (the autotuner's timing kernel): stage 0 of step_b
template <typename T>
__global__ void __launch_bounds__(512) k_en_rk_tune(EnArgs a) {
  __shared__ int64_t s_cpref[EN_MAXMEM + 1];
  en_load_pref(a.chunk_pref, s_cpref, a.nmem);
  __syncthreads();
  en_rk_elements<T>(a, s_cpref, false, 0);
}

// ---- CG members (2-d box lattices) -----------------------------------------
// One affine element's Helmholtz apply p L u + q M u (the arithmetic of
// k_helm2d, GHelmholtz::reg_prod, sem/ghelmholtz.ipp:309-378) by a team,
// input gathered from the lattice by ld(c), output element-local.
template <typename T, int N, class LD>
__device__ __forceinline__ void en_box_apply(const LaneTeam &tm, const EnMember &M, int64_t e,
                                             const T *D, const T *W, T *s, const LD &ld, T p,
                                             T q, T *__restrict__ out) {
  constexpr int NN = N * N;
  T *su = s, *sgx = s + NN, *sgy = s + 2 * NN;
  const T *eg = sizeof(T) == 8 ? (const T *)M.egeom64 : (const T *)M.egeom32;
  const T X0 = eg[e * 3], X1 = eg[e * 3 + 1], J = eg[e * 3 + 2];
  const int ey = (int)(e / M.ne0), ex = (int)(e - (int64_t)ey * M.ne0);
  const BoxWalk &w = M.walk;
#pragma unroll 4
  for (int a = tm.rank(); a < NN; a += tm.size()) {
    const int i = a % N, j = a / N;
    int gx = ex * (N - 1) + i, gy = ey * (N - 1) + j;
    if (w.per[0] && gx == w.M[0]) gx = 0;
    if (w.per[1] && gy == w.M[1]) gy = 0;
    su[a] = ld((int64_t)gy * w.M[0] + gx);
  }
  tm.sync();
  for (int a = tm.rank(); a < NN; a += tm.size()) {
    const int i = a % N, j = a / N;
    T dx = D[i] * su[j * N];
    T dy = D[j] * su[i];
#pragma unroll
    for (int m = 1; m < N; m++) {
      dx = fma(D[i + m * N], su[j * N + m], dx);
      dy = fma(D[j + m * N], su[m * N + i], dy);
    }
    const T mass = W[j] * W[i] * J;
    sgx[a] = mass * (dx * (X0 * X0));
    sgy[a] = mass * (dy * (X1 * X1));
  }
  tm.sync();
  for (int a = tm.rank(); a < NN; a += tm.size()) {
    const int i = a % N, j = a / N;
    T ox = D[i * N] * sgx[j * N];
    T oy = D[j * N] * sgy[i];
#pragma unroll
    for (int m = 1; m < N; m++) {
      ox = fma(D[m + i * N], sgx[j * N + m], ox);
      oy = fma(D[m + j * N], sgy[m * N + i], oy);
    }
    T o = ox + oy;
    o *= p;
    T mu = W[j] * W[i] * J * su[a];
    mu *= q;
    o += mu;
    out[e * NN + a] = o;
  }
}

struct LdW {  // FP32 search direction
  const float *w;
  __device__ __forceinline__ float operator()(int64_t c) const { return w[c]; }
};
struct LdW64 {  // FP64 search direction
  const double *w;
  __device__ __forceinline__ double operator()(int64_t c) const { return w[c]; }
};
struct LdX {  // FP64 solution plus the FP32 correction not yet added
  const double *x;
  const float *d;
  __device__ __forceinline__ double operator()(int64_t c) const { return x[c] + (double)d[c]; }
};

template <int N>
__device__ void en_cg_elem(const LaneTeam &tm, const EnMember &M, int64_t e, int mode, bool f64,
                           const float *Df, const float *Wf, const double *Dd, const double *Wd,
                           void *slice, double p, double q) {
  if (mode == EN_INNER && !f64)
    en_box_apply<float, N>(tm, M, e, Df, Wf, (float *)slice, LdW{M.w32}, (float)p, (float)q,
                           (float *)M.aE);
  else if (mode == EN_INNER)
    en_box_apply<double, N>(tm, M, e, Dd, Wd, (double *)slice, LdW64{M.w64}, p, q, M.aE);
  else
    en_box_apply<double, N>(tm, M, e, Dd, Wd, (double *)slice, LdX{M.xL, M.dL}, p, q, M.aE);
}

// words (doubles) of a CG warp's basis region: D and W in FP64 and FP32
__host__ __device__ __forceinline__ int en_cg_basis_doubles(int N) {
  return en_basis_words<double>(N) + (en_basis_words<float>(N) + 1) / 2;
}

__device__ void en_cg_elements(const EnArgs &a, const int64_t *cpref, const int *mode) {
  extern __shared__ __align__(16) unsigned char en_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double *ws = reinterpret_cast<double *>(en_smem + (size_t)wib * a.wbytes);
  const int64_t nw = (int64_t)gridDim.x * wpb;
  int cur = -1;
  const bool f64 = a.fp64 != 0;
  for (int64_t ch = (int64_t)blockIdx.x * wpb + wib; ch < a.nchunk; ch += nw) {
    const int mi = en_find(cpref, a.nmem, ch);
    const int md = a.all_inner ? EN_INNER : mode[mi];
    if (md == EN_DONE) continue;  // warp-uniform
    const EnMember &M = a.mem[mi];
    const int N = M.N;
    double *Dd = ws, *Wd = ws + N * N;
    float *Df = reinterpret_cast<float *>(ws + en_basis_words<double>(N)), *Wf = Df + N * N;
    if (mi != cur) {
      for (int i = lane; i < N * N; i += 32) {
        Dd[i] = M.D[i];
        Df[i] = (float)M.D[i];
      }
      for (int i = lane; i < N; i += 32) {
        Wd[i] = M.W[i];
        Wf[i] = (float)M.W[i];
      }
      __syncwarp();
      cur = mi;
    }
    const int team = M.team, tid = lane / team;
    const int64_t e = (ch - M.chunk0) * M.epw + tid;
    if (e < M.ne) {
      const LaneTeam tm{lane - tid * team, team, team_mask(team, tid)};
      void *slice = ws + en_cg_basis_doubles(N) + (size_t)tid * 3 * N * N;
      switch (N) {
        case 3: en_cg_elem<3>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 4: en_cg_elem<4>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 5: en_cg_elem<5>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 6: en_cg_elem<6>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 7: en_cg_elem<7>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 8: en_cg_elem<8>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        case 9: en_cg_elem<9>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
        default: en_cg_elem<10>(tm, M, e, md, f64, Df, Wf, Dd, Wd, slice, a.p, a.q); break;
      }
    }
    __syncwarp();
  }
}

// Block partials: every warp folds its lanes (fixed tree), then the warps'
// values are folded in warp order; partials[(mi*2 + k)*gridDim.x + block].
__device__ __forceinline__ double en_warp_fold(double v, bool max) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = max ? fmax(v, w) : v + w;
  }
  return v;
}

// The CG's lattice work in warp slices: slice s of member m covers the
// lattice nodes [s EN_WS, min((s+1) EN_WS, nL)); the slices of all members
// are numbered consecutively (prefix spref) and the grid's warps take them
// round robin, so a slice's warp is the same in every phase of a launch and
// reads back its own writes.  f(mi, M, c, hi, a0, a1) runs the calling
// lane's nodes c, c + 32, ... < hi; with `part` the warp's folded sums of
// slice s go to partials[2 s] and partials[2 s + 1].
template <class F>
__device__ __forceinline__ void en_ws_loop(const EnArgs &a, const int64_t *spref, const int *act,
                                           bool part, bool max1, F f) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * wpb;
  for (int64_t ws = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); ws < a.nclass; ws += nw) {
    const int mi = en_find(spref, a.nmem, ws);
    if (!act[mi]) continue;  // warp-uniform
    const EnMember &M = a.mem[mi];
    const int64_t lo = (ws - spref[mi]) * EN_WS;
    const int64_t hi = lo + EN_WS < M.nL ? lo + EN_WS : M.nL;
    double a0 = 0.0, a1 = 0.0;
    f(mi, M, lo + lane, hi, a0, a1);
    if (part) {
      a0 = en_warp_fold(a0, false);
      a1 = en_warp_fold(a1, max1);
      if (lane == 0) {
        a.partials[2 * ws] = a0;
        a.partials[2 * ws + 1] = a1;
      }
    }
  }
}

// In the last block: the two totals of member mi over its slices (one
// warp), valid in all lanes.  Lane l folds slices l, l + 32, ... in order
// (four loads issued ahead of the adds), then the lanes fold in a fixed
// tree: deterministic for a given member layout.
__device__ __forceinline__ void en_acc_total(const EnArgs &a, const int64_t *spref, int mi,
                                             bool max1, double &t0, double &t1) {
  const int lane = threadIdx.x & 31;
  const int64_t s0 = spref[mi], s1 = spref[mi + 1];
  double v0 = 0.0, v1 = 0.0;
  int64_t s = s0 + lane;
  for (; s + 96 < s1; s += 128) {
    double x[4], y[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      x[k] = __ldcg(a.partials + 2 * (s + 32 * k));
      y[k] = __ldcg(a.partials + 2 * (s + 32 * k) + 1);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v0 += x[k];
      v1 = max1 ? fmax(v1, y[k]) : v1 + y[k];
    }
  }
  for (; s < s1; s += 32) {
    v0 += __ldcg(a.partials + 2 * s);
    const double y = __ldcg(a.partials + 2 * s + 1);
    v1 = max1 ? fmax(v1, y) : v1 + y;
  }
  t0 = en_warp_fold(v0, false);
  t1 = en_warp_fold(v1, max1);
}

__device__ __forceinline__ double en_norm(const EnArgs &a, const EnCG &s, double t) {
  return a.normtype == GF_NORM_INF ? t : sqrt(t / s.nd);
}

// norm contribution of a lattice value r with `cnt` element copies
__device__ __forceinline__ void en_nacc(bool inf, double &acc, int cnt, double r) {
  acc = inf ? fmax(acc, fabs(r)) : acc + (double)cnt * r * r;
}

// One CG iteration of every member still running (see the file comment).
// A member is in one of three states: INNER (one PCG iteration: FP32
// vectors in the mixed solve, FP64 in the FP64 solve), REFINE (the FP64
// residual r = mask DSS_Sum(b - A (x + d)) with x += d, then the restart of
// the FP32 run; the FP64 solve passes here once, at its start) or DONE.  a.all_inner (the autotuner) runs every member as INNER
// and leaves the states alone.
__global__ void __launch_bounds__(512) k_en_cg_iter(EnArgs a) {
  __shared__ int64_t s_cpref[EN_MAXMEM + 1], s_spref[EN_MAXMEM + 1];
  __shared__ int s_mode[EN_MAXMEM], s_act[EN_MAXMEM], s_act3[EN_MAXMEM];
  en_load_pref(a.chunk_pref, s_cpref, a.nmem);
  en_load_pref(a.class_pref, s_spref, a.nmem);
  for (int i = threadIdx.x; i < a.nmem; i += blockDim.x) {
    s_mode[i] = a.all_inner ? EN_INNER : __ldcg(&a.cg[i].next);
    s_act[i] = s_mode[i] != EN_DONE;
  }
  __syncthreads();
  const bool inf = a.normtype == GF_NORM_INF, f64 = a.fp64 != 0;
  const bool tune = a.all_inner != 0;
  // 1. element applies: INNER q_E = A w; REFINE a_E = A (x + d) (FP64)
  en_cg_elements(a, s_cpref, s_mode);
  en_barrier(a.ctl, NoWork{});
  // 2. assembly: INNER q = mask DSS_Sum(q_E), <w, q>; REFINE x += d,
  //    r = mask (b_L - DSS_Sum(a_E)), norm(r)
  en_ws_loop(a, s_spref, s_act, true, inf,
             [&](int mi, const EnMember &M, int64_t c, int64_t hi, double &a0, double &a1) {
               const uint8_t *__restrict__ mk = M.maskL8;
               if (s_mode[mi] == EN_INNER && !f64) {
                 const float *__restrict__ qE = (const float *)M.aE;
                 const float *__restrict__ w = M.w32;
                 float *__restrict__ q = M.q32;
#pragma unroll 4
                 for (; c < hi; c += 32) {
                   const BoxCopies k = M.walk.copies((int)c);
                   float sm = 0.f;
                   k.each([&](int m) { sm = __fadd_rn(sm, __ldcg(qE + m)); });
                   const float qv = (!mk || mk[c]) ? sm : 0.f;
                   q[c] = qv;
                   a0 += (double)w[c] * (double)qv;
                 }
               } else if (s_mode[mi] == EN_INNER) {
                 const double *__restrict__ qE = M.aE;
                 const double *__restrict__ w = M.w64;
                 double *__restrict__ q = M.q64;
#pragma unroll 4
                 for (; c < hi; c += 32) {
                   const BoxCopies k = M.walk.copies((int)c);
                   double sm = 0.0;
                   k.each([&](int m) { sm = __dadd_rn(sm, __ldcg(qE + m)); });
                   const double qv = (!mk || mk[c]) ? sm : 0.0;
                   q[c] = qv;
                   a0 += w[c] * qv;
                 }
               } else {
                 for (; c < hi; c += 32) {
                   const BoxCopies k = M.walk.copies((int)c);
                   double sm = 0.0;
                   k.each([&](int m) { sm = __dadd_rn(sm, __ldcg(M.aE + m)); });
                   M.xL[c] = M.xL[c] + (double)M.dL[c];
                   M.dL[c] = 0.f;
                   const double r = (!M.maskL8 || M.maskL8[c]) ? M.bL[c] - sm : 0.0;
                   M.r64[c] = r;
                   en_nacc(inf, a1, k.count(), r);
                 }
               }
             });
  en_barrier(a.ctl, [&] {
    const int wpb = blockDim.x >> 5, wib = threadIdx.x >> 5;
    for (int mi = wib; mi < a.nmem; mi += wpb) {
      if (!s_act[mi]) continue;
      double t0, t1;
      en_acc_total(a, s_spref, mi, inf, t0, t1);
      if ((threadIdx.x & 31) != 0) continue;
      EnCG &S = a.cg[mi];
      if (s_mode[mi] == EN_INNER) {
        S.alpha = S.rho / t0;
        if (!tune && !isfinite(S.alpha)) {
          S.status = 2;
          S.next = EN_DONE;
        }
      } else {
        const double rn = en_norm(a, S, t1);
        S.rnorm64 = rn;
        S.sweeps++;
        if (!isfinite(rn)) {
          S.status = 2;
          S.next = EN_DONE;
        } else if (!f64 && rn <= S.rtol) {
          S.status = 0;
          S.next = EN_DONE;
        } else if (S.iters >= a.maxit || S.sweeps > a.max_refine) {
          S.status = (rn <= S.rtol) ? 0 : 1;
          S.next = EN_DONE;
        }
      }
    }
  });
  for (int i = threadIdx.x; i < a.nmem; i += blockDim.x)
    s_act3[i] = s_act[i] && (tune || __ldcg(&a.cg[i].next) != EN_DONE);
  __syncthreads();
  // 3. INNER: x (FP64) or d (FP32) += alpha w, r -= alpha q, z = Dinv r,
  //    <r, z>, norm(r); REFINE (not finished): z = Dinv r (r32 = r in the
  //    mixed solve), w = z, <r, z>, norm(r)
  en_ws_loop(a, s_spref, s_act3, true, inf,
             [&](int mi, const EnMember &M, int64_t c, int64_t hi, double &a0, double &a1) {
               const EnCG &S = a.cg[mi];
               const bool inner = s_mode[mi] == EN_INNER;
               if (inner && !f64) {
                 const float al = (float)__ldcg(&S.alpha);
                 float *__restrict__ d = M.dL;
                 float *__restrict__ rr = M.r32;
                 const float *__restrict__ w = M.w32;
                 const float *__restrict__ q = M.q32;
                 const float *__restrict__ di = M.dinv32;
#pragma unroll 4
                 for (; c < hi; c += 32) {
                   d[c] = fmaf(al, w[c], d[c]);
                   const float r = fmaf(-al, q[c], rr[c]);
                   rr[c] = r;
                   const float z = di[c] * r;
                   a0 += (double)r * (double)z;
                   en_nacc(inf, a1, inf ? 1 : M.walk.copies((int)c).count(), (double)r);
                 }
               } else if (inner) {
                 const double al = __ldcg(&S.alpha);
                 double *__restrict__ x = M.xL;
                 double *__restrict__ rr = M.r64;
                 const double *__restrict__ w = M.w64;
                 const double *__restrict__ q = M.q64;
                 const double *__restrict__ di = M.dinv64;
#pragma unroll 4
                 for (; c < hi; c += 32) {
                   x[c] = fma(al, w[c], x[c]);
                   const double r = fma(-al, q[c], rr[c]);
                   rr[c] = r;
                   const double z = di[c] * r;
                   a0 += r * z;
                   en_nacc(inf, a1, inf ? 1 : M.walk.copies((int)c).count(), r);
                 }
               } else if (f64) {
                 for (; c < hi; c += 32) {
                   const double r = M.r64[c];
                   const double z = M.dinv64[c] * r;
                   M.w64[c] = z;
                   a0 += r * z;
                   en_nacc(inf, a1, inf ? 1 : M.walk.copies((int)c).count(), r);
                 }
               } else {
                 for (; c < hi; c += 32) {
                   const float r = (float)M.r64[c];
                   M.r32[c] = r;
                   const float z = M.dinv32[c] * r;
                   M.w32[c] = z;
                   a0 += (double)r * (double)z;
                   en_nacc(inf, a1, inf ? 1 : M.walk.copies((int)c).count(), (double)r);
                 }
               }
             });
  en_barrier(a.ctl, [&] {
    const int wpb = blockDim.x >> 5, wib = threadIdx.x >> 5;
    for (int mi = wib; mi < a.nmem; mi += wpb) {
      if (!s_act3[mi]) continue;
      double t0, t1;
      en_acc_total(a, s_spref, mi, inf, t0, t1);
      if ((threadIdx.x & 31) != 0) continue;
      EnCG &S = a.cg[mi];
      const double rn = en_norm(a, S, t1);
      if (tune) {
        S.beta = 0.0;
        continue;
      }
      if (s_mode[mi] == EN_INNER) {
        S.beta = t0 / S.rho;
        S.rho = t0;
        S.rnorm = rn;
        S.iters++;
        if (!isfinite(S.beta) || !isfinite(rn)) {
          S.status = 2;
          S.next = EN_DONE;
        } else if (f64) {  // GCG's loop test on the recurrence residual
          if (rn <= S.rtol) {
            S.status = 0;
            S.next = EN_DONE;
          } else if (S.iters >= a.maxit) {
            S.status = 1;
            S.next = EN_DONE;
          }
        } else if (rn <= S.itol || S.iters >= a.maxit) {
          S.next = EN_REFINE;
        }
      } else {
        // the kept direction continues with beta = rho'/rho (0 at the start)
        S.beta = 0.0;
        S.rho = t0;
        S.rnorm = rn;
        S.itol = fmax(a.inner_tol * rn, 0.25 * S.rtol);
        S.next = (rn > 0.0 && isfinite(t0)) ? EN_INNER : EN_REFINE;
        if (f64 && !(rn > 0.0)) {  // exact solution: nothing to iterate
          S.status = 0;
          S.next = EN_DONE;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && !tune) {
      int any = 0;
      for (int mi = 0; mi < a.nmem; mi++) any |= (a.cg[mi].next != EN_DONE);
      a.ctl->any_active = any;
      a.ctl->launches++;
    }
  });
  // 4. INNER: w = Dinv r + beta w
  for (int i = threadIdx.x; i < a.nmem; i += blockDim.x)
    s_act[i] = s_act3[i] && s_mode[i] == EN_INNER;
  __syncthreads();
  en_ws_loop(a, s_spref, s_act, false, inf,
             [&](int mi, const EnMember &M, int64_t c, int64_t hi, double &, double &) {
               if (f64) {
                 const double be = __ldcg(&a.cg[mi].beta);
                 double *__restrict__ w = M.w64;
                 const double *__restrict__ di = M.dinv64;
                 const double *__restrict__ r = M.r64;
#pragma unroll 4
                 for (; c < hi; c += 32) w[c] = fma(be, w[c], di[c] * r[c]);
               } else {
                 const float be = (float)__ldcg(&a.cg[mi].beta);
                 float *__restrict__ w = M.w32;
                 const float *__restrict__ di = M.dinv32;
                 const float *__restrict__ r = M.r32;
#pragma unroll 4
                 for (; c < hi; c += 32) w[c] = fmaf(be, w[c], di[c] * r[c]);
               }
             });
  if (a.has_cond && blockIdx.x == 0 && threadIdx.x == 0) {
    const bool more = __ldcg(&a.ctl->any_active) && !ld_acquire(&a.ctl->err) &&
                      ld_acquire(&a.ctl->launches) < a.launch_cap;
    cudaGraphSetConditional(a.cond, more ? 1u : 0u);
  }
}

// Solve setup: b_L = DSS_Sum(b_E), x_L = mask x_E (solve_impl (2) with
// xb = 0, gcg.ipp:362-382), the Jacobi inverse of the assembled diagonal,
// norm(b) on the element-local b, the stop threshold.
__global__ void __launch_bounds__(512) k_en_cg_init(EnArgs a) {
  __shared__ int64_t s_spref[EN_MAXMEM + 1];
  __shared__ int s_act[EN_MAXMEM];
  en_load_pref(a.class_pref, s_spref, a.nmem);
  for (int i = threadIdx.x; i < a.nmem; i += blockDim.x) s_act[i] = 1;
  __syncthreads();
  const bool inf = a.normtype == GF_NORM_INF;
  en_ws_loop(a, s_spref, s_act, true, inf,
             [&](int mi, const EnMember &M, int64_t c, int64_t hi, double &, double &a1) {
               const int N = M.N, NN = N * N;
               for (; c < hi; c += 32) {
                 const BoxCopies k = M.walk.copies((int)c);
                 double sm = 0.0, dg = 0.0, x0 = 0.0;
                 bool first = true;
                 k.each([&](int m) {
                   const double bv = M.bE[m];
                   sm = __dadd_rn(sm, bv);
                   a1 = inf ? fmax(a1, fabs(bv)) : a1 + bv * bv;
                   if (first) x0 = M.xE[m];
                   first = false;
                   const int64_t e = m / NN;
                   const int loc = (int)(m - e * NN), i = loc % N, j = loc / N;
                   const double X0 = M.egeom64[e * 3], X1 = M.egeom64[e * 3 + 1],
                                J = M.egeom64[e * 3 + 2];
                   dg += a.p * (X0 * X0 * J * M.W[j] * M.K1d[i] + X1 * X1 * J * M.W[i] * M.K1d[j]) +
                         a.q * J * M.W[i] * M.W[j];
                 });
                 M.bL[c] = sm;
                 M.xL[c] = (!M.maskL8 || M.maskL8[c]) ? x0 : 0.0;  // x = mask x + xb, xb = 0
                 M.dL[c] = 0.f;
                 M.w32[c] = 0.f;
                 M.w64[c] = 0.0;
                 const double di = dg != 0.0 ? 1.0 / dg : 1.0;
                 M.dinv64[c] = di;
                 M.dinv32[c] = (float)di;
               }
             });
  en_barrier(a.ctl, [&] {
    const int wpb = blockDim.x >> 5, wib = threadIdx.x >> 5;
    for (int mi = wib; mi < a.nmem; mi += wpb) {
      double t0, t1;
      en_acc_total(a, s_spref, mi, inf, t0, t1);
      if ((threadIdx.x & 31) != 0) continue;
      EnCG &S = a.cg[mi];
      S.bnorm = en_norm(a, S, t1);
      S.rtol = (a.relative || S.bnorm >= 1.0) ? a.tol * S.bnorm : a.tol;
      S.next = EN_REFINE;
      S.iters = S.sweeps = S.status = 0;
      S.rho = S.alpha = S.beta = 0.0;
      S.rnorm = S.rnorm64 = S.bnorm;
    }
    if (threadIdx.x == 0) {
      a.ctl->any_active = 1;
      a.ctl->launches = 0;
    }
  });
}

// x_E = x_L at every element-local node (one thread per node).
__global__ void k_en_cg_finish(EnArgs a) {
  for (int mi = 0; mi < a.nmem; mi++) {
    const EnMember &M = a.mem[mi];
    const int N = M.N, NN = N * N, P = N - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M.nlocal;
         i += (int64_t)gridDim.x * blockDim.x) {
      const int64_t e = i / NN;
      const int loc = (int)(i - e * NN);
      const int ey = (int)(e / M.ne0), ex = (int)(e - (int64_t)ey * M.ne0);
      int gx = ex * P + loc % N, gy = ey * P + loc / N;
      if (M.walk.per[0] && gx == M.walk.M[0]) gx = 0;
      if (M.walk.per[1] && gy == M.walk.M[1]) gy = 0;
      M.xE[i] = M.xL[(int64_t)gy * M.walk.M[0] + gx];
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct EnShape {
  int threads = 256, bps = 0;  // bps 0: as many as fit
  int team[EN_MAXN + 1];       // lanes per element, by point count
  bool tuned = false;
  float ms = -1.f;  // the tuner's time per launch of the chosen shape
  EnShape() {
    for (int n = 0; n <= EN_MAXN; n++) team[n] = n * n <= 16 ? 8 : (n * n <= 48 ? 16 : 32);
  }
};

struct gf_ensemble {
  gf_context *ctx = nullptr;
  std::vector<gf_problem *> probs;
  int kind = -1;  // GF_ENS_RK or GF_ENS_CG, fixed by the members
  EnShape shape[3];  // RK FP64, RK FP32, CG
  std::vector<EnMember> host;
  EnMember *mem_d = nullptr;
  int64_t *pref_d = nullptr;  // chunk prefix, then class prefix
  EnCtl *ctl_d = nullptr;
  EnCtl *ctl_h = nullptr;  // pinned
  EnCG *cg_d = nullptr;
  EnCG *cg_h = nullptr;  // pinned
  double *partials = nullptr;
  size_t partials_n = 0;
  std::vector<void *> bufs;  // per-member device buffers
  size_t buf_key = 0;        // dtype/kind the buffers were made for
  cudaStream_t cs = nullptr;  // capture stream
  // cached graphs: RK (1 and 2 steps) per dtype, CG loop
  cudaGraphExec_t rk_exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int rk_key[2][2][3] = {};  // ns, threads, blocks
  double rk_nu_key[2][2] = {};  // nu (held in the captured arguments)
  cudaGraphExec_t cg_exec = nullptr;
  int cg_key[2] = {};
  double cg_pkey[5] = {};  // p, q, tol, inner_tol, relative|normtype|maxit|max_refine
  int rk_eqn = -1;         // equation of the last RK advance (the tuner runs it)
  double rk_nu = 0.0;
  int cg_fp64 = 0;         // precision of the last CG solve (the tuner runs it)
  bool cooperative = true;
  uint64_t launches = 0;
  int last_grid = 0;
};

namespace {

int en_cap_bytes(gf_ensemble *E, int which, int team_override_n = -1, int team_override = 0) {
  // dynamic shared bytes per warp for shape `which`
  size_t wb = 0;
  for (size_t m = 0; m < E->probs.size(); m++) {
    const gf_problem *p = E->probs[m];
    const int N = p->n;
    int team = E->shape[which].team[N];
    if (N == team_override_n) team = team_override;
    const int epw = 32 / team;
    size_t b;
    if (which == 2)
      b = sizeof(double) * (en_cg_basis_doubles(N) + (size_t)epw * 3 * N * N);
    else if (which == 0)
      b = sizeof(double) * (en_basis_words<double>(N) + (size_t)epw * 5 * N * N);
    else
      b = sizeof(float) * (en_basis_words<float>(N) + (size_t)epw * 5 * N * N);
    wb = std::max(wb, b);
  }
  return (int)((wb + 15) / 16 * 16);
}

const void *en_kernel(int which) {
  if (which == 0) return (const void *)k_en_rk_stage<double>;
  if (which == 1) return (const void *)k_en_rk_stage<float>;
  return (const void *)k_en_cg_iter;
}

// Blocks of the cooperative grid for shape `which` (0 if it does not fit).
int en_grid(gf_ensemble *E, int which, int threads, int bps, int wbytes) {
  const void *k = en_kernel(which);
  const size_t smem = (size_t)wbytes * (threads / 32);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  // the tuning kernel runs the same shape; the CG setup kernel is launched
  // cooperatively on the same grid, so it must fit as well
  const void *other = which == 0   ? (const void *)k_en_rk_tune<double>
                      : which == 1 ? (const void *)k_en_rk_tune<float>
                                   : (const void *)k_en_cg_init;
  if (cudaFuncSetAttribute(other, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (which == 2) {
    int occ2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, other, threads, smem) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    occ = std::min(occ, occ2);
  }
  if (occ < 1) return 0;
  const int b = bps > 0 ? std::min(bps, occ) : occ;
  return b * E->ctx->sm_count;
}

// Chunk and class numbering for shape `which`; fills descriptor offsets and
// the prefix arrays (host), returns totals.
// Work numbering of shape `which`: element chunks (cpref); RK node items
// (kpref, all nodes) and shared classes (spref); CG lattice warp slices
// (kpref).
void en_layout(gf_ensemble *E, int which, std::vector<int64_t> &cpref, std::vector<int64_t> &kpref,
               std::vector<int64_t> &spref, int64_t &nchunk, int64_t &nclass, int64_t &nsh) {
  const int n = (int)E->probs.size();
  cpref.assign(n + 1, 0);
  kpref.assign(n + 1, 0);
  spref.assign(n + 1, 0);
  nchunk = nclass = nsh = 0;
  for (int m = 0; m < n; m++) {
    EnMember &M = E->host[m];
    M.team = E->shape[which].team[M.N];
    M.epw = 32 / M.team;
    M.chunk0 = nchunk;
    M.nchunk = (M.ne + M.epw - 1) / M.epw;
    M.class0 = nclass;
    cpref[m] = nchunk;
    kpref[m] = nclass;
    spref[m] = nsh;
    nchunk += M.nchunk;
    nclass += which == 2 ? (M.nL + EN_WS - 1) / EN_WS : M.nlocal;
    nsh += which == 2 ? 0 : M.nshared;
  }
  cpref[n] = nchunk;
  kpref[n] = nclass;
  spref[n] = nsh;
}

int en_upload(gf_ensemble *E, int which, EnArgs &a) {
  gf_context *ctx = E->ctx;
  std::vector<int64_t> cp, kp, sp;
  int64_t nchunk, nclass, nsh;
  en_layout(E, which, cp, kp, sp, nchunk, nclass, nsh);
  const int n = (int)E->probs.size();
  cudaStream_t st = ctx->stream;
  GF_CUDA(ctx, cudaMemcpyAsync(E->mem_d, E->host.data(), sizeof(EnMember) * n,
                               cudaMemcpyHostToDevice, st));
  GF_CUDA(ctx, cudaMemcpyAsync(E->pref_d, cp.data(), sizeof(int64_t) * (n + 1),
                               cudaMemcpyHostToDevice, st));
  GF_CUDA(ctx, cudaMemcpyAsync(E->pref_d + EN_MAXMEM + 1, kp.data(), sizeof(int64_t) * (n + 1),
                               cudaMemcpyHostToDevice, st));
  GF_CUDA(ctx, cudaMemcpyAsync(E->pref_d + 2 * (EN_MAXMEM + 1), sp.data(),
                               sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
  // the host arrays are pageable: finish the copies before they change
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  memset(&a, 0, sizeof(a));
  a.mem = E->mem_d;
  a.nmem = n;
  a.chunk_pref = E->pref_d;
  a.class_pref = E->pref_d + EN_MAXMEM + 1;
  a.sh_pref = E->pref_d + 2 * (EN_MAXMEM + 1);
  a.nchunk = nchunk;
  a.nclass = nclass;
  a.nsh = nsh;
  a.ctl = E->ctl_d;
  a.cg = E->cg_d;
  a.partials = E->partials;
  a.wbytes = en_cap_bytes(E, which);
  return GF_OK;
}

cudaError_t en_launch(gf_ensemble *E, const void *k, int grid, int threads, size_t smem,
                      cudaStream_t st, void **args, bool coop) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = coop ? at : nullptr;
  cfg.numAttrs = coop ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, k, args);
}

int en_check_partials(gf_ensemble *E, int64_t nslice) {
  const size_t need = (size_t)2 * std::max<int64_t>(nslice, 1);
  if (E->partials_n >= need) return GF_OK;
  if (E->partials) cudaFree(E->partials);
  E->partials = nullptr;
  GF_CUDA(E->ctx, cudaMalloc(&E->partials, sizeof(double) * need));
  E->partials_n = need;
  return GF_OK;
}

void en_drop_graphs(gf_ensemble *E) {
  for (auto &row : E->rk_exec)
    for (auto &g : row)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  if (E->cg_exec) {
    cudaGraphExecDestroy(E->cg_exec);
    E->cg_exec = nullptr;
  }
}

void en_free_bufs(gf_ensemble *E) {
  for (void *b : E->bufs) cudaFree(b);
  E->bufs.clear();
  E->buf_key = 0;
}

void *en_alloc(gf_ensemble *E, size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, std::max<size_t>(bytes, 16));
  E->bufs.push_back(p);
  return p;
}

// Scratch vectors of every member: RK (u[1], K[0..2], uf) or CG.
int en_buffers(gf_ensemble *E, int which) {
  const size_t key = (size_t)which + 1;
  if (E->buf_key == key) return GF_OK;
  en_drop_graphs(E);
  en_free_bufs(E);
  for (size_t m = 0; m < E->probs.size(); m++) {
    EnMember &M = E->host[m];
    if (which < 2) {
      const size_t b = (which == 0 ? sizeof(double) : sizeof(float)) * (size_t)M.nlocal;
      M.u[1] = en_alloc(E, b);
      for (int k = 0; k < 3; k++) M.K[k] = en_alloc(E, b);
      M.uf = en_alloc(E, b);
      M.advb[0] = en_alloc(E, b);
      M.advb[1] = en_alloc(E, b);
      if (!M.u[1] || !M.K[0] || !M.K[1] || !M.K[2] || !M.uf || !M.advb[0] || !M.advb[1])
        goto oom;
    } else {
      const size_t L = (size_t)M.nL;
      M.bL = (double *)en_alloc(E, 8 * L);
      M.xL = (double *)en_alloc(E, 8 * L);
      M.r64 = (double *)en_alloc(E, 8 * L);
      M.dinv64 = (double *)en_alloc(E, 8 * L);
      M.aE = (double *)en_alloc(E, 8 * (size_t)M.nlocal);
      M.dL = (float *)en_alloc(E, 4 * L);
      M.r32 = (float *)en_alloc(E, 4 * L);
      M.w32 = (float *)en_alloc(E, 4 * L);
      M.q32 = (float *)en_alloc(E, 4 * L);
      M.dinv32 = (float *)en_alloc(E, 4 * L);
      M.w64 = (double *)en_alloc(E, 8 * L);
      M.q64 = (double *)en_alloc(E, 8 * L);
      if (!M.bL || !M.xL || !M.r64 || !M.dinv64 || !M.aE || !M.dL || !M.r32 || !M.w32 ||
          !M.q32 || !M.dinv32 || !M.w64 || !M.q64)
        goto oom;
    }
  }
  E->buf_key = key;
  return GF_OK;
oom:
  en_free_bufs(E);
  return gf_fail(E->ctx, GF_ERR_NOMEM, "ensemble scratch allocation failed");
}

// Time `reps` launches of the tuning kernel of shape `which`; returns ms
// per launch or a negative value when the shape does not fit.
float en_time_shape(gf_ensemble *E, int which, int reps) {
  EnShape &S = E->shape[which];
  EnArgs a;
  if (en_upload(E, which, a)) return -1.f;
  const int grid = en_grid(E, which, S.threads, S.bps, a.wbytes);
  if (grid <= 0) return -1.f;
  // RK: the element phase of stage 0 (no grid barrier); CG: one whole
  // iteration of every member (cooperative: its barriers and reductions
  // depend on the block count)
  const void *k = which == 0   ? (const void *)k_en_rk_tune<double>
                  : which == 1 ? (const void *)k_en_rk_tune<float>
                               : (const void *)k_en_cg_iter;
  a.all_inner = 1;
  a.ns = 1;
  a.eqn = E->rk_eqn;
  a.nu = E->rk_nu;
  a.fp64 = E->cg_fp64;
  a.fast = E->rk_eqn == GF_EQN_ADVECT && E->rk_nu == 0.0;
  if (which == 2) {
    if (en_check_partials(E, a.nclass)) return -1.f;
    a.partials = E->partials;
    if (cudaMemsetAsync(E->ctl_d, 0, sizeof(EnCtl), E->ctx->stream) != cudaSuccess) return -1.f;
  }
  void *args[1] = {&a};
  const size_t smem = (size_t)a.wbytes * (S.threads / 32);
  cudaStream_t st = E->ctx->stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = -1.f;
  for (int r = 0; r < reps + 2; r++) {
    cudaEventRecord(e0, st);
    if (en_launch(E, k, grid, S.threads, smem, st, args, which == 2 && E->cooperative) !=
        cudaSuccess) {
      cudaGetLastError();
      best = -1.f;
      break;
    }
    E->launches++;
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 2 && (best < 0.f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

int en_which(int kind, int dtype) {
  if (kind == GF_ENS_CG) return 2;
  return dtype == GF_F32 ? 1 : 0;
}

}  // namespace

extern "C" int gf_ensemble_create(gf_ctx_t ctx, int n, const gf_problem_t *members,
                                  gf_ensemble_t *out) {
  if (!ctx || !out) return GF_ERR_ARG;
  *out = nullptr;
  GF_REQUIRE(ctx, n >= 1 && n <= EN_MAXMEM && members, "1..%d members", EN_MAXMEM);
  int kind = -1;
  for (int m = 0; m < n; m++) {
    const gf_problem *p = members[m];
    GF_REQUIRE(ctx, p && p->ctx == ctx, "member %d is not a problem of this context", m);
    GF_REQUIRE(ctx, p->dim == 2, "member %d: ensembles take 2-d members", m);
    GF_REQUIRE(ctx, p->n >= EN_MINN && p->n <= EN_MAXN, "member %d: order %d outside 2..%d", m,
               p->n - 1, EN_MAXN - 1);
    int k;
    if (p->geom >= GF_GEOM_DEFORMED) {
      GF_REQUIRE(ctx, p->dgeom_d && p->dgeom_f && p->gmet_d && p->gmet_f,
                 "member %d: deformed geometry missing", m);
      k = GF_ENS_RK;
    } else {
      BoxWalk w{};
      GF_REQUIRE(ctx, p->has_box && p->egeom_d && p->egeom_f && dss_box_walk(p, w),
                 "member %d: CG members are box grids with affine elements", m);
      k = GF_ENS_CG;
    }
    GF_REQUIRE(ctx, kind < 0 || kind == k,
               "members mix deformed (RK) and box (CG) problems; make one ensemble of each");
    kind = k;
  }
  gf_ensemble *E = new gf_ensemble;
  E->ctx = ctx;
  E->kind = kind;
  E->probs.assign(members, members + n);
  E->host.resize(n);
  for (int m = 0; m < n; m++) {
    gf_problem *p = members[m];
    EnMember &M = E->host[m];
    memset(&M, 0, sizeof(M));
    M.N = p->n;
    M.nxy = p->nxy ? p->nxy : p->dim;
    M.ne = p->ne;
    M.nlocal = p->nlocal;
    M.nclass = p->nclass;
    for (int i = 0; i < M.N * M.N; i++) M.D[i] = p->D[i];
    for (int i = 0; i < M.N; i++) {
      M.W[i] = p->W[i];
      M.K1d[i] = p->K1[i + i * M.N];
    }
    M.class_ptr = p->class_ptr;
    M.members = p->members;
    M.sh_ptr = p->sh_ptr;
    M.sh_members = p->sh_members;
    M.nshared = p->nshared;
    M.imult32 = p->imult_f;
    if (kind == GF_ENS_RK) {
      M.X[0] = p->dgeom_d;
      M.X[1] = p->dgeom_f;
      M.G[0] = p->gmet_d;
      M.G[1] = p->gmet_f;
      M.J[0] = p->ngeom_d + (int64_t)p->dim * p->nlocal;
      M.J[1] = p->ngeom_f + (int64_t)p->dim * p->nlocal;
      M.imass[0] = p->imass_d;
      M.imass[1] = p->imass_f;
    } else {
      M.walk = BoxWalk::make(p->box);
      M.ne0 = p->box.ne[0];
      M.nL = p->box.size();
      M.maskL8 = p->maskL8;
      M.egeom64 = p->egeom_d;
      M.egeom32 = p->egeom_f;
    }
  }
  cudaError_t e = cudaMalloc(&E->mem_d, sizeof(EnMember) * n);
  if (e == cudaSuccess) e = cudaMalloc(&E->pref_d, sizeof(int64_t) * 3 * (EN_MAXMEM + 1));
  if (e == cudaSuccess) e = cudaMalloc(&E->ctl_d, sizeof(EnCtl));
  if (e == cudaSuccess) e = cudaMalloc(&E->cg_d, sizeof(EnCG) * EN_MAXMEM);
  if (e == cudaSuccess) e = cudaMallocHost(&E->ctl_h, sizeof(EnCtl));
  if (e == cudaSuccess) e = cudaMallocHost(&E->cg_h, sizeof(EnCG) * EN_MAXMEM);
  if (e == cudaSuccess) e = cudaMemset(E->ctl_d, 0, sizeof(EnCtl));
  if (e == cudaSuccess) e = cudaMemset(E->cg_d, 0, sizeof(EnCG) * EN_MAXMEM);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    gf_ensemble_destroy(E);
    return gf_fail(ctx, GF_ERR_NOMEM, "ensemble allocation failed: %s", cudaGetErrorString(e));
  }
  ctx->nprob++;
  *out = E;
  return GF_OK;
}

extern "C" int gf_ensemble_destroy(gf_ensemble_t E) {
  if (!E) return GF_OK;
  en_drop_graphs(E);
  en_free_bufs(E);
  if (E->mem_d) cudaFree(E->mem_d);
  if (E->pref_d) cudaFree(E->pref_d);
  if (E->ctl_d) cudaFree(E->ctl_d);
  if (E->cg_d) cudaFree(E->cg_d);
  if (E->partials) cudaFree(E->partials);
  if (E->ctl_h) cudaFreeHost(E->ctl_h);
  if (E->cg_h) cudaFreeHost(E->cg_h);
  if (E->cs) cudaStreamDestroy(E->cs);
  if (E->ctx && E->mem_d) E->ctx->nprob--;
  delete E;
  return GF_OK;
}

extern "C" int gf_ensemble_kind(gf_ensemble_t E) { return E ? E->kind : GF_ERR_ARG; }

extern "C" uint64_t gf_ensemble_launches(gf_ensemble_t E) { return E ? E->launches : 0; }

extern "C" int gf_ensemble_shape(gf_ensemble_t E, int dtype, int *threads, int *blocks,
                                 int *team_by_n, int *tuned, double *tuned_ms) {
  if (!E) return GF_ERR_ARG;
  const int w = en_which(E->kind, dtype);
  const EnShape &S = E->shape[w];
  if (threads) *threads = S.threads;
  if (blocks) *blocks = en_grid(E, w, S.threads, S.bps, en_cap_bytes(E, w));
  if (team_by_n)
    for (int n = 0; n <= EN_MAXN; n++) team_by_n[n] = S.team[n];
  if (tuned) *tuned = S.tuned ? 1 : 0;
  if (tuned_ms) *tuned_ms = S.ms;
  return GF_OK;
}

extern "C" int gf_ensemble_set_shape(gf_ensemble_t E, int dtype, int threads, int bps,
                                     const int *team_by_n) {
  if (!E) return GF_ERR_ARG;
  gf_context *ctx = E->ctx;
  GF_REQUIRE(ctx, threads == 64 || threads == 128 || threads == 256 || threads == 512,
             "threads per block: 64, 128, 256 or 512");
  GF_REQUIRE(ctx, bps >= 0 && bps <= 32, "blocks per SM: 0 (as many as fit) .. 32");
  const int w = en_which(E->kind, dtype);
  EnShape S = E->shape[w];
  S.threads = threads;
  S.bps = bps;
  if (team_by_n)
    for (int n = EN_MINN; n <= EN_MAXN; n++) {
      GF_REQUIRE(ctx, team_by_n[n] == 8 || team_by_n[n] == 16 || team_by_n[n] == 32,
                 "team widths are 8, 16 or 32 lanes");
      S.team[n] = team_by_n[n];
    }
  const EnShape old = E->shape[w];
  E->shape[w] = S;
  if (en_grid(E, w, S.threads, S.bps, en_cap_bytes(E, w)) <= 0) {
    E->shape[w] = old;
    return gf_fail(ctx, GF_ERR_ARG, "shape does not fit on the device");
  }
  en_drop_graphs(E);
  return GF_OK;
}

// The autotuner: coordinate search over threads x blocks per SM, then the
// team width of each order present, each candidate timed on the element
// phase of this ensemble (best of `reps` launches).
extern "C" int gf_ensemble_tune(gf_ensemble_t E, int dtype, int reps) {
  if (!E) return GF_ERR_ARG;
  gf_context *ctx = E->ctx;
  const int w = en_which(E->kind, dtype);
  GF_REQUIRE(ctx, E->kind == GF_ENS_CG || dtype == GF_F32 || dtype == GF_F64, "bad dtype");
  const bool search = reps >= 0;  // reps < 0: time the current shape |reps| times, no search
  reps = reps == 0 ? 5 : (reps < 0 ? -reps : reps);
  int rc = en_buffers(E, w);
  if (rc) return rc;
  // The timing kernels read and write the ensemble's own scratch only: an
  // RK member's stage input is its scratch state u[1] and its velocity
  // components are scratch slopes (the element work does not depend on the
  // values); a CG member's search direction is its scratch w.  The caller's
  // buffers are restored afterwards.
  std::vector<EnMember> saved = E->host;
  if (E->kind == GF_ENS_RK) {
    for (auto &M : E->host) {
      M.u[0] = M.u[1];
      M.c[0] = M.K[1];
      M.c[1] = M.K[2];
      M.c[2] = M.uf;
    }
    if (E->rk_eqn < 0) E->rk_eqn = GF_EQN_ADVECT;
  }
  EnShape &S = E->shape[w];
  EnShape best = S;
  float tbest = en_time_shape(E, w, reps);
  const int thr[4] = {64, 128, 256, 512};
  const int bps[4] = {1, 2, 4, 0};
  for (int ti = 0; search && ti < 4; ti++)
    for (int bi = 0; bi < 4; bi++) {
      S = best;
      S.threads = thr[ti];
      S.bps = bps[bi];
      const float t = en_time_shape(E, w, reps);
      if (t > 0.f && (tbest < 0.f || t < tbest)) {
        tbest = t;
        best = S;
      }
    }
  bool seen[EN_MAXN + 1] = {};
  for (auto *p : E->probs) seen[p->n] = true;
  const int teams[3] = {8, 16, 32};
  for (int n = EN_MINN; search && n <= EN_MAXN; n++) {
    if (!seen[n]) continue;
    for (int k = 0; k < 3; k++) {
      S = best;
      S.team[n] = teams[k];
      const float t = en_time_shape(E, w, reps);
      if (t > 0.f && (tbest < 0.f || t < tbest)) {
        tbest = t;
        best = S;
      }
    }
  }
  best.tuned = search || best.tuned;
  best.ms = tbest;
  S = best;
  E->host = saved;
  en_drop_graphs(E);
  if (tbest < 0.f) return gf_fail(ctx, GF_ERR_CUDA, "no ensemble shape could be launched");
  return GF_OK;
}

// ---- RK --------------------------------------------------------------------
extern "C" int gf_ensemble_rk_advance(gf_ensemble_t E, int dtype, const gf_rk_traits *tr,
                                      void *const *u, const void *const *c, const double *dt,
                                      int nsteps) {
  if (!E) return GF_ERR_ARG;
  gf_context *ctx = E->ctx;
  GF_REQUIRE(ctx, E->kind == GF_ENS_RK, "this ensemble holds CG (box) members");
  GF_REQUIRE(ctx, tr && u && dt && nsteps >= 0, "traits, u and dt are required");
  GF_REQUIRE(ctx, dtype == GF_F32 || dtype == GF_F64, "unknown dtype %d", dtype);
  GF_REQUIRE(ctx, tr->eqn == GF_EQN_ADVECT || tr->eqn == GF_EQN_HEAT,
             "ensemble RK evolves advection or heat members");
  GF_REQUIRE(ctx, tr->nstate == 1, "one state component per member");
  GF_REQUIRE(ctx, tr->scheme >= GF_RK1 && tr->scheme <= GF_RK4, "ensemble RK runs step_b (RK1..RK4)");
  GF_REQUIRE(ctx, tr->eqn != GF_EQN_ADVECT || c, "advection needs the members' velocities");
  const int n = (int)E->probs.size();
  for (int m = 0; m < n; m++) {
    GF_REQUIRE(ctx, u[m], "member %d: state missing", m);
    if (tr->eqn == GF_EQN_ADVECT)
      for (int k = 0; k < E->host[m].nxy; k++)
        GF_REQUIRE(ctx, c[3 * m + k], "member %d: velocity component %d missing", m, k);
  }
  int capturing = 0;
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    GF_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    capturing = cs != cudaStreamCaptureStatusNone;
  }
  GF_REQUIRE(ctx, !capturing, "the ensemble captures its own graphs; call it outside a capture");
  if (nsteps == 0) return GF_OK;
  const int w = en_which(GF_ENS_RK, dtype);
  int rc = en_buffers(E, w);
  if (rc) return rc;
  double alpha[4], beta[4][4], cc[4];
  gfrk::butcher(tr->scheme, alpha, beta, cc);
  const int ns = tr->scheme;
  if (E->rk_eqn != tr->eqn) en_drop_graphs(E);
  E->rk_eqn = tr->eqn;
  E->rk_nu = tr->nu;
  for (int m = 0; m < n; m++) {
    EnMember &M = E->host[m];
    M.u[0] = u[m];
    for (int k = 0; k < 3; k++)
      M.c[k] = (tr->eqn == GF_EQN_ADVECT && k < M.nxy) ? c[3 * m + k] : nullptr;
    // coefficients rounded as the single-problem stepper rounds them
    for (int s = 0; s < 4; s++) {
      for (int j = 0; j < 3; j++) {
        if (dtype == GF_F32) {
          const float h = (float)dt[m];
          M.coef[s][j] = (double)((float)beta[s][j] * h);
        } else {
          M.coef[s][j] = beta[s][j] * dt[m];
        }
      }
      M.ch[s] = dtype == GF_F32 ? (double)((float)cc[s] * (float)dt[m]) : cc[s] * dt[m];
    }
  }
  EnArgs a;
  if ((rc = en_upload(E, w, a))) return rc;
  const EnShape &S = E->shape[w];
  const int grid = en_grid(E, w, S.threads, S.bps, a.wbytes);
  if (grid <= 0) return gf_fail(ctx, GF_ERR_UNSUPPORTED, "ensemble shape does not fit");
  a.ns = ns;
  a.eqn = tr->eqn;
  a.nu = tr->nu;
  a.fast = tr->eqn == GF_EQN_ADVECT && tr->nu == 0.0;
  const size_t smem = (size_t)a.wbytes * (S.threads / 32);
  const void *k = en_kernel(w);
  cudaStream_t st = ctx->stream;
  if (a.fast)  // the coefficient planes, by the single-problem stepper's kernel
    for (int m = 0; m < n; m++) {
      gf_problem *p = E->probs[m];
      EnMember &M = E->host[m];
      const int nc = M.nxy;
      int r2;
      if (dtype == GF_F32) {
        const float *cc[3] = {(const float *)M.c[0], (const float *)M.c[1],
                              nc > 2 ? (const float *)M.c[2] : nullptr};
        r2 = gfrk::adv_coef_launch<float>(p, cc, (float *)M.advb[0], (float *)M.advb[1], st);
      } else {
        const double *cc[3] = {(const double *)M.c[0], (const double *)M.c[1],
                               nc > 2 ? (const double *)M.c[2] : nullptr};
        r2 = gfrk::adv_coef_launch<double>(p, cc, (double *)M.advb[0], (double *)M.advb[1], st);
      }
      if (r2) return gf_fail(ctx, r2, "advection coefficients");
      E->launches++;
    }
  GF_CUDA(ctx, cudaMemsetAsync(E->ctl_d, 0, sizeof(EnCtl), st));
  // graphs of 2 steps (par 0 then 1) and 1 step (par 0), rebuilt when the
  // scheme or shape changes; the kernels read the descriptors from device
  // memory, so the same graph serves any bound state
  auto build = [&](int steps, cudaGraphExec_t &exec, int *key, double &nukey) -> int {
    if (exec && key[0] == ns && key[1] == S.threads && key[2] == grid && nukey == tr->nu)
      return GF_OK;
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    for (int attempt = 0; attempt < 2; attempt++) {
      const bool coop = E->cooperative;
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(E->cs, cudaStreamCaptureModeRelaxed);
      for (int s = 0; e == cudaSuccess && s < steps; s++)
        for (int stg = 0; e == cudaSuccess && stg < ns; stg++) {
          EnArgs b = a;
          b.par = s & 1;
          int sv = stg;
          void *args[2] = {&b, &sv};
          e = en_launch(E, k, grid, S.threads, smem, E->cs, args, coop);
        }
      cudaError_t e2 = cudaStreamEndCapture(E->cs, &g);
      if (e == cudaSuccess) e = e2;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e == cudaSuccess) break;
      cudaGetLastError();
      exec = nullptr;
      if (!coop) return gf_fail(ctx, GF_ERR_CUDA, "ensemble graph capture failed: %s",
                                cudaGetErrorString(e));
      E->cooperative = false;  // capture without the cooperative attribute
    }
    key[0] = ns;
    key[1] = S.threads;
    key[2] = grid;
    nukey = tr->nu;
    return GF_OK;
  };
  const int di = dtype == GF_F32 ? 1 : 0;
  if (nsteps >= 2 && (rc = build(2, E->rk_exec[di][1], E->rk_key[di][1], E->rk_nu_key[di][1])))
    return rc;
  if ((nsteps & 1) && (rc = build(1, E->rk_exec[di][0], E->rk_key[di][0], E->rk_nu_key[di][0])))
    return rc;
  for (int s = 0; s + 1 < nsteps; s += 2) {
    GF_CUDA(ctx, cudaGraphLaunch(E->rk_exec[di][1], st));
    E->launches += 2 * ns;
  }
  if (nsteps & 1) {
    GF_CUDA(ctx, cudaGraphLaunch(E->rk_exec[di][0], st));
    E->launches += ns;
    const size_t bytes = (dtype == GF_F32 ? 4 : 8) * 1;
    for (int m = 0; m < n; m++)
      GF_CUDA(ctx, cudaMemcpyAsync(E->host[m].u[0], E->host[m].u[1], bytes * E->host[m].nlocal,
                                   cudaMemcpyDeviceToDevice, st));
  }
  E->last_grid = grid;
  GF_CUDA(ctx, cudaMemcpyAsync(E->ctl_h, E->ctl_d, sizeof(EnCtl), cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  if (E->ctl_h->err) return gf_fail(ctx, GF_ERR_CUDA, "ensemble grid barrier timed out");
  for (int m = 0; m < n; m++)
    if (E->ctl_h->nonfinite[m])
      return gf_fail(ctx, GF_ERR_NONFINITE, "member %d: non-finite state after the last step", m);
  return GF_OK;
}

// ---- CG --------------------------------------------------------------------
extern "C" int gf_ensemble_cg_solve(gf_ensemble_t E, const gf_cg_traits *tr, double p, double q,
                                    const double *const *b, double *const *x, int *iters,
                                    double *final_norm, int *status) {
  if (!E) return GF_ERR_ARG;
  gf_context *ctx = E->ctx;
  GF_REQUIRE(ctx, E->kind == GF_ENS_CG, "this ensemble holds RK (deformed) members");
  GF_REQUIRE(ctx, tr && b && x, "traits, b and x are required");
  GF_REQUIRE(ctx, tr->precision == GF_CG_MIXED || tr->precision == GF_CG_FP64,
             "ensemble CG precision: GF_CG_MIXED or GF_CG_FP64");
  GF_REQUIRE(ctx, tr->precond == GF_PRECOND_JACOBI, "ensemble CG takes the Jacobi preconditioner");
  GF_REQUIRE(ctx, tr->normtype == GF_NORM_EUC || tr->normtype == GF_NORM_INF,
             "ensemble CG norms: EUC or INF");
  GF_REQUIRE(ctx, tr->maxit >= 1 && tr->tol > 0.0, "maxit >= 1 and tol > 0");
  const int n = (int)E->probs.size();
  for (int m = 0; m < n; m++) GF_REQUIRE(ctx, b[m] && x[m], "member %d: b or x missing", m);
  int rc = en_buffers(E, 2);
  if (rc) return rc;
  for (int m = 0; m < n; m++) {
    E->host[m].bE = b[m];
    E->host[m].xE = x[m];
  }
  EnArgs a;
  if ((rc = en_upload(E, 2, a))) return rc;
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    GF_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    GF_REQUIRE(ctx, cs == cudaStreamCaptureStatusNone,
               "the ensemble captures its own graphs; call it outside a capture");
  }
  const EnShape &S = E->shape[2];
  const int grid = en_grid(E, 2, S.threads, S.bps, a.wbytes);
  if (grid <= 0) return gf_fail(ctx, GF_ERR_UNSUPPORTED, "ensemble shape does not fit");
  if ((rc = en_check_partials(E, a.nclass))) return rc;
  a.partials = E->partials;
  a.p = p;
  a.q = q;
  a.tol = tr->tol;
  a.fp64 = tr->precision == GF_CG_FP64;
  a.inner_tol = tr->inner_tol > 0.0 ? tr->inner_tol : 1e-4;
  E->cg_fp64 = a.fp64;
  a.normtype = tr->normtype;
  a.maxit = tr->maxit;
  a.max_refine = tr->max_refine > 0 ? tr->max_refine : 64;
  a.relative = tr->relative;
  a.launch_cap = (unsigned)std::min<int64_t>(0x7fffffff, 2LL * tr->maxit + 4LL * a.max_refine + 16);
  for (int m = 0; m < n; m++) {
    E->cg_h[m] = EnCG{};
    E->cg_h[m].nd = (double)E->host[m].nlocal;
  }
  cudaStream_t st = ctx->stream;
  GF_CUDA(ctx, cudaMemcpyAsync(E->cg_d, E->cg_h, sizeof(EnCG) * n, cudaMemcpyHostToDevice, st));
  GF_CUDA(ctx, cudaMemsetAsync(E->ctl_d, 0, sizeof(EnCtl), st));
  const size_t smem = (size_t)a.wbytes * (S.threads / 32);
  {
    void *args[1] = {&a};
    GF_CUDA(ctx, en_launch(E, (const void *)k_en_cg_init, grid, S.threads, smem, st, args,
                           E->cooperative));
    E->launches++;
  }
  // the iteration loop: a WHILE node whose body is one cooperative launch;
  // the kernel's block 0 clears the condition once no member is running
  // the captured kernel holds p, q and the traits in its arguments
  const double pkey[5] = {p, q, a.tol, a.inner_tol,
                          (double)a.relative + 2.0 * a.normtype + 8.0 * a.fp64 +
                              32.0 * a.max_refine + 65536.0 * (double)a.maxit};
  if (!(E->cg_exec && E->cg_key[0] == S.threads && E->cg_key[1] == grid &&
        std::equal(pkey, pkey + 5, E->cg_pkey))) {
    if (E->cg_exec) cudaGraphExecDestroy(E->cg_exec);
    E->cg_exec = nullptr;
    for (int attempt = 0; attempt < 2; attempt++) {
      const bool coop = E->cooperative;
      cudaGraph_t g = nullptr, body = nullptr;
      cudaGraphConditionalHandle h = 0;
      cudaError_t e = cudaGraphCreate(&g, 0);
      if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
      cudaGraphNodeParams np = {};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
      if (e == cudaSuccess) {
        body = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(E->cs, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed);
      }
      if (e == cudaSuccess) {
        EnArgs b2 = a;
        b2.cond = h;
        b2.has_cond = 1;
        void *args[1] = {&b2};
        e = en_launch(E, (const void *)k_en_cg_iter, grid, S.threads, smem, E->cs, args, coop);
        cudaError_t e2 = cudaStreamEndCapture(E->cs, &body);
        if (e == cudaSuccess) e = e2;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&E->cg_exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e == cudaSuccess) break;
      cudaGetLastError();
      E->cg_exec = nullptr;
      if (!coop)
        return gf_fail(ctx, GF_ERR_CUDA, "ensemble CG capture failed: %s", cudaGetErrorString(e));
      E->cooperative = false;
    }
    E->cg_key[0] = S.threads;
    E->cg_key[1] = grid;
    std::copy(pkey, pkey + 5, E->cg_pkey);
  }
  GF_CUDA(ctx, cudaGraphLaunch(E->cg_exec, st));
  E->launches++;
  k_en_cg_finish<<<std::max(1, ctx->sm_count * 4), 256, 0, st>>>(a);
  GF_CHECK_LAUNCH(ctx);
  E->last_grid = grid;
  GF_CUDA(ctx, cudaMemcpyAsync(E->cg_h, E->cg_d, sizeof(EnCG) * n, cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaMemcpyAsync(E->ctl_h, E->ctl_d, sizeof(EnCtl), cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  E->launches += E->ctl_h->launches;
  if (E->ctl_h->err) return gf_fail(ctx, GF_ERR_CUDA, "ensemble grid barrier timed out");
  int worst = GF_OK;
  for (int m = 0; m < n; m++) {
    const EnCG &C = E->cg_h[m];
    if (iters) iters[m] = C.iters;
    if (final_norm) final_norm[m] = a.fp64 ? C.rnorm : C.rnorm64;
    if (status) status[m] = C.status;
    if (C.status == 2) worst = GF_ERR_NONFINITE;
    else if (C.status == 1 && worst == GF_OK) worst = GF_CG_NOCONVERGE;
    if (C.next != EN_DONE && worst == GF_OK) worst = GF_CG_NOCONVERGE;
  }
  if (worst == GF_ERR_NONFINITE) return gf_fail(ctx, worst, "ensemble CG breakdown (non-finite)");
  return worst;
}

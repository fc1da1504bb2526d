// api_cg.cu -- conjugate gradient on the assembled Helmholtz operator.
//
// Semantics follow GCG::solve_impl (solvers/gcg.ipp:239-382, the
// Deville-Fischer-Mund form): r = mask*DSS_Sum(b - A x), dots weighted by
// 1/multiplicity, the stop rule norm(r) <= (norm(b) < 1 ? tol : tol*norm(b))
// with norm(b) taken on the element-local b, and the xb lift of
// solve_impl (2).  Additions the reference lacks: a Jacobi preconditioner,
// a relative stop option and a mixed-precision solve (FP32 PCG on the
// correction, FP64 residual and iterative refinement).
//
// B200 layout: the iteration vectors live on the unique nodes (one value
// per GGFX class, 0.68x the element-local size at p = 7) where the
// reference keeps duplicated element-local copies.  A multiplicity-weighted
// element-local dot equals the plain unique-node dot, so the algorithm is
// unchanged.  Per iteration four kernels run back to back with no host
// round trip:
//   1. q_E = A_e w   fused element apply, w gathered from the unique nodes
//                    (box lattice indices computed, or node_class)
//   2. q = mask * assemble(q_E), <w,q>   each unique node's element copies
//                    are folded in ascending local id (box: by the element
//                    owning the node; CSR: one thread per class); the last
//                    block forms alpha
//   3. x += alpha w, r -= alpha q, rho' = <r, Dinv r>, norm(r); the last
//                    block forms beta and sets `done` at convergence
//   4. w = beta w + Dinv r
// Batches of iterations are queued ahead; every kernel returns at once
// when `done` is set, and the host reads the flag every `check_every`
// iterations.
#include <algorithm>
#include <cmath>
#include <unordered_map>
#include <vector>

#include "gf_common.cuh"
#include "k_dss.cuh"
#include "k_vec.cuh"
#include "ops_launch.cuh"

using namespace gfk;

namespace {

enum {
  S_RHO = 0,
  S_ALPHA,
  S_BETA,
  S_RNORM,
  S_RTOL,
  S_DONE,
  S_ITER,
  S_MAXIT,
  S_WQ,
  S_FLAG,   // 1: non-finite scalar (breakdown)
  S_BNORM,
  S_NTOT,   // number of element-local nodes (EUC norm)
  S_IVOL,   // 1/volume (L2, L1 norms)
  S_NORMT,  // norm type
  S_REL,    // relative stop rule
  S_RES,    // norm of the last assembled residual pass
  S_OTOL,   // stop threshold of the whole solve (S_RTOL: of the current run)
  S_INNER,  // restarted mixed solve: relative tolerance of each FP32 run
  S_ZR,     // polynomial-preconditioned solve: <r, z> of the last step
  S_FIRST,  // polynomial-preconditioned solve: 1 before its first step
  S_COUNT
};

// ---- unique-node maps ----
// rows(f) visits every unique node once, calling f(c, g) with its index c
// and (box only) lattice coordinates g; each(c, g, f) calls f(m) for the
// members m of the node in ascending local id; mult(c, g) is the count.

// Box lattice of order N-1.  rows() walks lattice rows (fixed gy, gz) by
// block, so a node's coordinates come from the launch shape; rows_sum() walks
// the flat lattice index with multiply-shift divisions by the lattice
// widths (FastDiv); the order being a compile-time constant turns every %
// and / by p into a multiply-shift.
template <int N>
struct MapBox {
  static constexpr int P = N - 1;
  int dim, ne[3], per[3], M[3];
  FastDiv fd0, fd1;  // divisions by M[0], M[1]
  static MapBox make(const BoxLattice &L) {
    MapBox m;
    m.dim = L.dim;
    m.sorted = 1;
    for (int d = 0; d < 3; d++) {
      m.ne[d] = L.ne[d];
      m.per[d] = L.per[d];
      m.M[d] = (int)L.M[d];
      if (d < L.dim && L.per[d] && L.ne[d] == 1) m.sorted = 0;
    }
    m.fd0 = FastDiv::make(m.M[0]);
    m.fd1 = FastDiv::make(m.M[1]);
    return m;
  }
  template <class F>
  __device__ __forceinline__ void rows(F f) const {
    const int nrows = M[1] * M[2];
    for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
      const int g1 = row % M[1], g2 = row / M[1];
      const int64_t base = (int64_t)row * M[0];
      for (int g0 = threadIdx.x; g0 < M[0]; g0 += blockDim.x) {
        const int g[3] = {g0, g1, g2};
        f(base + g0, g);
      }
    }
  }
  int sorted;  // 0 when some periodic direction has a single element
  // (element coordinate, local index) pairs of lattice coordinate g, dir d,
  // in ascending element coordinate
  __device__ __forceinline__ int cands(int d, int g, int (&ec)[2], int (&l)[2]) const {
    const int r = g % P, q = g / P;
    if (r != 0) {
      ec[0] = q;
      l[0] = r;
      return 1;
    }
    if (per[d]) {
      if (q == 0) {  // wraps: (0, 0) then (ne-1, P)
        ec[0] = 0;
        l[0] = 0;
        ec[1] = ne[d] - 1;
        l[1] = P;
      } else {
        ec[0] = q - 1;
        l[0] = P;
        ec[1] = q;
        l[1] = 0;
      }
      return 2;
    }
    int k = 0;
    if (q >= 1) {
      ec[k] = q - 1;
      l[k++] = P;
    }
    if (q < ne[d]) {
      ec[k] = q;
      l[k++] = 0;
    }
    return k;
  }
  // Members in ascending local id.  With every direction's candidates in
  // ascending element coordinate, the (z, y, x) nesting already yields
  // ascending element ids; only a single-element periodic direction (two
  // members in one element) needs the explicit sort.
  template <class F>
  __device__ __forceinline__ void each(int64_t, const int (&g)[3], F f) const {
    int ec[3][2], l[3][2], cnt[3] = {1, 1, 1};
    ec[2][0] = ec[2][1] = 0;
    l[2][0] = l[2][1] = 0;
    for (int d = 0; d < dim; d++) cnt[d] = cands(d, g[d], ec[d], l[d]);
    const int nn = dim > 2 ? N * N * N : N * N;
    if (sorted) {
#pragma unroll
      for (int a = 0; a < 2; a++) {
        if (a >= cnt[2]) break;
#pragma unroll
        for (int b = 0; b < 2; b++) {
          if (b >= cnt[1]) break;
#pragma unroll
          for (int i = 0; i < 2; i++) {
            if (i >= cnt[0]) break;
            const int e = ec[0][i] + ne[0] * (ec[1][b] + ne[1] * ec[2][a]);
            f((int64_t)(e * nn + (l[0][i] + N * (l[1][b] + N * l[2][a]))));
          }
        }
      }
      return;
    }
    int m[8];
    int k = 0;
    for (int a = 0; a < cnt[2]; a++)
      for (int b = 0; b < cnt[1]; b++)
        for (int i = 0; i < cnt[0]; i++) {
          const int e = ec[0][i] + ne[0] * (ec[1][b] + ne[1] * ec[2][a]);
          m[k++] = e * nn + (l[0][i] + N * (l[1][b] + N * l[2][a]));
        }
    for (int i = 1; i < k; i++) {
      const int v = m[i];
      int j = i - 1;
      while (j >= 0 && m[j] > v) {
        m[j + 1] = m[j];
        j--;
      }
      m[j + 1] = v;
    }
    for (int i = 0; i < k; i++) f((int64_t)m[i]);
  }
  // f(c, s) for every lattice point c, s = sum of its element copies in
  // ascending local id (added in TS).  One thread per lattice point in
  // lattice order (grid-stride over the flat index): the point's
  // coordinates from two multiply-shift divisions, its copies from scalar
  // offsets (lattice_offsets), added in the (z, y, x) nesting, which is
  // ascending element id when no periodic direction has a single element
  // (otherwise the explicit sort of each()).  Lattice and element-local
  // sizes are below 2^31 (checked when the problem is created).
  template <typename TS, typename TV, class F>
  __device__ __forceinline__ void rows_sum(const TV *__restrict__ inE, F f) const {
    if (!sorted) {
      rows([&](int64_t c, const int(&g)[3]) {
        TS s = TS(0);
        each(c, g, [&](int64_t m) { s = __fadd_rn_t(s, (TS)inE[m]); });
        f(c, s);
      });
      return;
    }
    constexpr int NN = N * N;
    const bool d3 = dim > 2;
    const int nn = d3 ? NN * N : NN;
    const int sy = ne[0] * nn, sz = ne[0] * ne[1] * nn;
    const int nL = M[0] * M[1] * (d3 ? M[2] : 1);
    const int stride = gridDim.x * blockDim.x;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nL;
         c = (c < nL - stride) ? c + stride : nL) {
      const int row = fd0.div(c), g0 = c - row * M[0];
      const int g2 = fd1.div(row), g1 = row - g2 * M[1];
      int ox0, ox1, oy0, oy1, oz0 = 0, oz1 = 0;
      const int nx = lattice_offsets<P>(g0, ne[0], per[0], nn, 1, ox0, ox1);
      const int ny = lattice_offsets<P>(g1, ne[1], per[1], sy, N, oy0, oy1);
      const int nz = d3 ? lattice_offsets<P>(g2, ne[2], per[2], sz, NN, oz0, oz1) : 1;
      TS s = TS(0);
#pragma unroll
      for (int az = 0; az < 2; az++) {
        if (az >= nz) break;
        const int oz = az ? oz1 : oz0;
#pragma unroll
        for (int ay = 0; ay < 2; ay++) {
          if (ay >= ny) break;
          const int o = oz + (ay ? oy1 : oy0);
          s = __fadd_rn_t(s, (TS)inE[o + ox0]);
          if (nx > 1) s = __fadd_rn_t(s, (TS)inE[o + ox1]);
        }
      }
      f((int64_t)c, s);
    }
  }
  __device__ __forceinline__ double mult(int64_t, const int (&g)[3]) const {
    int m = 1;
    for (int d = 0; d < dim; d++) {
      int ec[2], l[2];
      m *= cands(d, g[d], ec, l);
    }
    return (double)m;
  }
  __device__ __forceinline__ int64_t lof(int64_t i) const {  // E index -> lattice index
    constexpr int NN = N * N;
    const int64_t nn = dim > 2 ? (int64_t)NN * N : NN;
    const int64_t e = i / nn;
    const int a = (int)(i - e * nn);
    const int c0 = (int)(e % ne[0]);
    const int64_t r = e / ne[0];
    const int c1 = (int)(r % ne[1]), c2 = dim > 2 ? (int)(r / ne[1]) : 0;
    auto g1 = [&](int d, int ec, int l) {
      int gi = ec * P + l;
      return (per[d] && gi == M[d]) ? 0 : gi;
    };
    int64_t idx = g1(0, c0, a % N) + (int64_t)M[0] * g1(1, c1, (a / N) % N);
    if (dim > 2) idx += (int64_t)M[0] * M[1] * g1(2, c2, a / NN);
    return idx;
  }
};

struct MapCsr {
  const int32_t *ptr, *mem, *ncls;
  int64_t nL;
  template <class F>
  __device__ __forceinline__ void rows(F f) const {
    const int g[3] = {0, 0, 0};
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nL;
         c += (int64_t)gridDim.x * blockDim.x)
      f(c, g);
  }
  template <class F>
  __device__ __forceinline__ void each(int64_t c, const int (&)[3], F f) const {
    for (int32_t k = ptr[c]; k < ptr[c + 1]; k++) f((int64_t)mem[k]);
  }
  __device__ __forceinline__ double mult(int64_t c, const int (&)[3]) const {
    return (double)(ptr[c + 1] - ptr[c]);
  }
  template <typename TS, typename TV, class F>
  __device__ __forceinline__ void rows_sum(const TV *__restrict__ inE, F f) const {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nL;
         c += (int64_t)gridDim.x * blockDim.x) {
      TS s = TS(0);
      for (int32_t k = ptr[c]; k < ptr[c + 1]; k++) s = __fadd_rn_t(s, (TS)inE[mem[k]]);
      f(c, s);
    }
  }
  __device__ __forceinline__ int64_t lof(int64_t i) const { return ncls[i]; }
};

struct Weights {
  const uint8_t *maskL;  // 1 keep, 0 Dirichlet; null: no mask
  const double *massL;   // L2/L1 norms
  const uint8_t *multL;  // multiplicity (EUC norm)
};

__device__ __forceinline__ double norm_term_L(int normtype, double r, const Weights &wt,
                                              int64_t c) {
  if (normtype == GF_NORM_INF) return fabs(r);
  if (normtype == GF_NORM_EUC) return (double)wt.multL[c] * (r * r);
  if (normtype == GF_NORM_L2) return wt.massL[c] * (r * r);
  return wt.massL[c] * fabs(r);
}

__device__ __forceinline__ double finish_norm(int normtype, double v, const double *scal) {
  if (normtype == GF_NORM_INF) return v;
  if (normtype == GF_NORM_EUC) return sqrt(v / scal[S_NTOT]);
  if (normtype == GF_NORM_L2) return sqrt(v * scal[S_IVOL]);
  return v * scal[S_IVOL];
}

template <bool MAX>
__device__ __forceinline__ double acc(double a, double t) {
  return MAX ? fmax(a, t) : a + t;
}

#define GRID_STRIDE(i, n)                                                        \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);     \
       i += (int64_t)gridDim.x * blockDim.x)

// ---- E <-> L conversions ----
// out_L[c] = sum of the element copies (ascending local id), FP64
template <class MAP, typename TI>
__global__ void k_assemble(int64_t nL, MAP map, const TI *__restrict__ inE, double *__restrict__ outL) {
  map.template rows_sum<double>(inE, [&](int64_t c, double s) { outL[c] = s; });
}

// x_L[c] = x_E[smallest member]  (x_E is duplicate-consistent)
template <class MAP>
__global__ void k_pick(int64_t nL, MAP map, const double *__restrict__ xE, double *__restrict__ xL) {
  map.rows([&](int64_t c, const int(&g)[3]) {
    bool first = true;
    double v = 0.0;
    map.each(c, g, [&](int64_t m) {
      if (first) v = xE[m];
      first = false;
    });
    xL[c] = v;
  });
}

// x_E = mask_E * x_L[class] + xb_E   (solve_impl (2) epilogue)
template <class MAP>
__global__ void k_scatter(int64_t nE, MAP map, const double *__restrict__ xL,
                          const double *__restrict__ maskE, const double *__restrict__ xbE,
                          double *__restrict__ xE) {
  GRID_STRIDE(i, nE) {
    double v = xL[map.lof(i)];
    if (maskE) v *= maskE[i];
    if (xbE) v += xbE[i];
    xE[i] = v;
  }
}

// x_E = mask_E * x_E + xb_E   (solve_impl (2) prologue)
__global__ void k_lift(int64_t nE, const double *__restrict__ maskE, const double *__restrict__ xbE,
                       double *__restrict__ xE) {
  GRID_STRIDE(i, nE) {
    double v = xE[i];
    if (maskE) v *= maskE[i];
    if (xbE) v += xbE[i];
    xE[i] = v;
  }
}

// norm of the element-local b (the reference measures b as given)
__global__ void __launch_bounds__(RED_THREADS)
    k_norm_E(int64_t n, int normtype, const double *__restrict__ b, const double *__restrict__ mass,
             double *scal, double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  double rn = 0.0;
  GRID_STRIDE(i, n) {
    double t;
    if (normtype == GF_NORM_INF) t = fabs(b[i]);
    else if (normtype == GF_NORM_EUC) t = b[i] * b[i];
    else if (normtype == GF_NORM_L2) t = mass[i] * (b[i] * b[i]);
    else t = mass[i] * fabs(b[i]);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  }
  rn = normtype == GF_NORM_INF ? block_reduce<true>(rn, sh) : block_reduce<false>(rn, sh);
  double pv[1] = {rn};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    double t = normtype == GF_NORM_INF ? fold_partials<true>(partials, gridDim.x, sh)
                                       : fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      scal[S_BNORM] = finish_norm(normtype, t, scal);
      *counter = 0;
    }
  }
}

// Residual pass: r = mask * (b_L - assemble(q_E)) in FP64; also writes the
// solve-precision copy r_T and rho = <r_T, Dinv r_T>.
//   mode 0 (start): w_T = Dinv r_T and a fresh CG state: rtol from the
//     reference rule on norm(b), rnorm = 10 rtol, iter = 0.
//   mode 1 (restart of the mixed solve after a correction): a fresh CG
//     state on the new residual; the iteration count is kept; `done` = 2
//     when the true residual meets the solve's threshold, else the next
//     FP32 run stops at max(inner * norm(r), threshold).
//   mode 2 (reliable update of the mixed solve): the search direction w_T
//     and the iteration count are kept; rnorm becomes the true residual
//     norm and `done` is set only if that meets rtol (or maxit is spent).
template <typename T, class MAP>
__global__ void __launch_bounds__(RED_THREADS)
    k_resid(int64_t nL, MAP map, Weights wt, const double *__restrict__ bL,
            const double *__restrict__ qE, double *__restrict__ rL, T *__restrict__ rT,
            T *__restrict__ wT, const float *__restrict__ dinv, int mode, double tol, double *scal,
            double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  const int normtype = (int)scal[S_NORMT];
  double rho = 0.0, rn = 0.0;
  map.template rows_sum<double>(qE, [&](int64_t c, double s) {
    double r = bL[c] - s;
    if (wt.maskL && !wt.maskL[c]) r = 0.0;
    rL[c] = r;
    const T rt = (T)r;
    const T zt = dinv ? (T)dinv[c] * rt : rt;
    if (rT != (T *)rL) rT[c] = rt;
    if (mode != 2) wT[c] = zt;
    rho += (double)rt * (double)zt;
    const double t = norm_term_L(normtype, r, wt, c);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  });
  rho = block_reduce<false>(rho, sh);
  rn = normtype == GF_NORM_INF ? block_reduce<true>(rn, sh) : block_reduce<false>(rn, sh);
  double pv[2] = {rho, rn};
  if (publish_partials<2>(pv, partials, counter, gridDim.x)) {
    double rho_t = fold_partials<false>(partials, gridDim.x, sh);
    double rn_t = normtype == GF_NORM_INF ? fold_partials<true>(partials + gridDim.x, gridDim.x, sh)
                                          : fold_partials<false>(partials + gridDim.x, gridDim.x, sh);
    if (threadIdx.x == 0) {
      const double rnorm = finish_norm(normtype, rn_t, scal);
      scal[S_RES] = rnorm;
      scal[S_RHO] = rho_t;
      if (mode == 2) {
        scal[S_RNORM] = rnorm;
        const bool bad = !isfinite(rnorm) || !isfinite(rho_t);
        if (bad) scal[S_FLAG] = 1.0;
        scal[S_DONE] =
            (rnorm <= scal[S_RTOL] || scal[S_ITER] >= scal[S_MAXIT] || bad) ? 2.0 : 0.0;
      } else if (mode == 1) {
        const double otol = scal[S_OTOL];
        scal[S_RNORM] = rnorm;
        const bool bad = !isfinite(rnorm) || !isfinite(rho_t);
        if (bad) scal[S_FLAG] = 1.0;
        scal[S_DONE] = (rnorm <= otol || scal[S_ITER] >= scal[S_MAXIT] || bad) ? 2.0 : 0.0;
        scal[S_RTOL] = fmax(scal[S_INNER] * rnorm, otol);
      } else {
        const double bnorm = scal[S_BNORM];
        const double rtol = (scal[S_REL] != 0.0 || bnorm >= 1.0) ? tol * bnorm : tol;
        scal[S_OTOL] = rtol;
        scal[S_RTOL] = scal[S_INNER] > 0.0 ? fmax(scal[S_INNER] * rnorm, rtol) : rtol;
        scal[S_RNORM] = 10.0 * scal[S_RTOL];
        scal[S_ITER] = 0.0;
        // A non-finite right-hand side or initial residual stops the solve
        // before its first iteration and is reported as GF_ERR_NONFINITE
        // (the reference's loop test rnorm > rtol is false for NaN, so it
        // would return GCGERR_NONE without iterating).
        const bool bad = !isfinite(bnorm) || !isfinite(rnorm) || !isfinite(rho_t);
        scal[S_FLAG] = bad ? 1.0 : 0.0;
        scal[S_DONE] = (scal[S_MAXIT] <= 0.0 || !(10.0 * rtol > rtol) || bad) ? 1.0 : 0.0;
      }
      *counter = 0;
    }
  }
}

// 2. q_L = mask * assemble(q_E); <w,q>; alpha
template <typename T, class MAP>
__global__ void __launch_bounds__(RED_THREADS)
    k_asm_dot(int64_t nL, MAP map, Weights wt, const T *__restrict__ qE, const T *__restrict__ w,
              T *__restrict__ qL, double *scal, double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  double dot = 0.0;
  map.template rows_sum<T>(qE, [&](int64_t c, T s) {
    if (wt.maskL && !wt.maskL[c]) s = T(0);
    qL[c] = s;
    dot += (double)w[c] * (double)s;
  });
  dot = block_reduce<false>(dot, sh);
  double pv[1] = {dot};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    double wq = fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      const double alpha = scal[S_RHO] / wq;
      scal[S_WQ] = wq;
      scal[S_ALPHA] = alpha;
      if (!isfinite(alpha)) {
        scal[S_FLAG] = 1.0;
        scal[S_DONE] = 1.0;
      }
      *counter = 0;
    }
  }
}

// grid-wide finish of the x/r update: rho' and norm(r) from the block
// partials; beta; the residual history; the stop test
__device__ __forceinline__ void update_finish(double rho, double rn, int normtype,
                                              double *__restrict__ hist, double *__restrict__ ab,
                                              int nab, double *scal, double *partials,
                                              unsigned int *counter, double *sh) {
  rho = block_reduce<false>(rho, sh);
  rn = normtype == GF_NORM_INF ? block_reduce<true>(rn, sh) : block_reduce<false>(rn, sh);
  double pv[2] = {rho, rn};
  if (publish_partials<2>(pv, partials, counter, gridDim.x)) {
    double rho_t = fold_partials<false>(partials, gridDim.x, sh);
    double rn_t = normtype == GF_NORM_INF ? fold_partials<true>(partials + gridDim.x, gridDim.x, sh)
                                          : fold_partials<false>(partials + gridDim.x, gridDim.x, sh);
    if (threadIdx.x == 0) {
      const double beta = rho_t / scal[S_RHO];
      const double rnorm = finish_norm(normtype, rn_t, scal);
      const int it = (int)scal[S_ITER];
      scal[S_RHO] = rho_t;
      scal[S_BETA] = beta;
      scal[S_RNORM] = rnorm;
      if (hist) hist[it] = rnorm;
      if (ab && it < nab) {  // Lanczos coefficients of the preconditioned operator
        ab[2 * it] = scal[S_ALPHA];
        ab[2 * it + 1] = beta;
      }
      scal[S_ITER] = (double)(it + 1);
      const bool bad = !isfinite(rnorm) || !isfinite(beta);
      if (bad) scal[S_FLAG] = 1.0;
      if (rnorm <= scal[S_RTOL] || it + 1 >= (int)scal[S_MAXIT] || bad) scal[S_DONE] = 2.0;
      *counter = 0;
    }
  }
}

// 3. x += alpha w; r -= alpha q; rho' = <r, Dinv r>; norm(r); beta; stop test
template <typename T, class MAP>
__global__ void __launch_bounds__(RED_THREADS)
    k_update(int64_t nL, MAP map, Weights wt, T *__restrict__ x, const T *__restrict__ w,
             T *__restrict__ r, const T *__restrict__ q, const float *__restrict__ dinv,
             double *__restrict__ hist, double *__restrict__ ab, int nab, double *scal,
             double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  const int normtype = (int)scal[S_NORMT];
  const T alpha = (T)scal[S_ALPHA];
  double rho = 0.0, rn = 0.0;
  // plain streaming over the unique nodes (no lattice information needed)
  GRID_STRIDE(c, nL) {
    x[c] = x[c] + alpha * w[c];
    const T rc = r[c] + (-alpha) * q[c];
    r[c] = rc;
    const T zc = dinv ? (T)dinv[c] * rc : rc;
    rho += (double)rc * (double)zc;
    const double t = norm_term_L(normtype, (double)rc, wt, c);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  }
  update_finish(rho, rn, normtype, hist, ab, nab, scal, partials, counter, sh);
}

// k_update of the multigrid-preconditioned CG (FP64, no Jacobi weight),
// which also takes the first smoothing term of the next V-cycle on the new
// residual (k_mg_start's work: bm = (TM) r, xm = c0 Dinv bm in the
// multigrid's type) while r is in registers.  Points written after
// convergence are never read.
template <typename TM>
__global__ void __launch_bounds__(RED_THREADS)
    k_update_mg(int64_t nL, Weights wt, double *__restrict__ x, const double *__restrict__ w,
                double *__restrict__ r, const double *__restrict__ q,
                const TM *__restrict__ dinvm, TM c0, TM *__restrict__ bm,
                TM *__restrict__ xm, double *__restrict__ hist, double *scal,
                double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  const int normtype = (int)scal[S_NORMT];
  const double alpha = scal[S_ALPHA];
  double rho = 0.0, rn = 0.0;
  GRID_STRIDE(c, nL) {
    x[c] = x[c] + alpha * w[c];
    const double rc = r[c] + (-alpha) * q[c];
    r[c] = rc;
    rho += rc * rc;
    const TM bc = (TM)rc;
    bm[c] = bc;
    xm[c] = c0 * (dinvm[c] * bc);
    const double t = norm_term_L(normtype, rc, wt, c);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  }
  update_finish(rho, rn, normtype, hist, nullptr, 0, scal, partials, counter, sh);
}

// 4. w = beta w + Dinv r
template <typename T>
__global__ void k_wupdate(int64_t nL, T *__restrict__ w, const T *__restrict__ r,
                          const float *__restrict__ dinv, const double *scal) {
  if (scal[S_DONE] != 0.0) return;
  const T beta = (T)scal[S_BETA];
  GRID_STRIDE(c, nL) {
    const T rc = r[c];
    const T zc = dinv ? (T)dinv[c] * rc : rc;
    w[c] = beta * w[c] + T(1) * zc;
  }
}

// x_L += (double) d_L
__global__ void k_add_correction(int64_t nL, const float *__restrict__ d, double *__restrict__ x) {
  GRID_STRIDE(c, nL) { x[c] += (double)d[c]; }
}

// ---- FP32 Chebyshev polynomial preconditioner z = P(r) ----
// The Chebyshev iteration for D^-1 A z = D^-1 r on the eigenvalue interval
// [a, b] (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed.,
// Algorithm 12.1), run for a fixed number of steps from z = 0:
//   res_0 = r, d_0 = D^-1 res_0 / theta, z_1 = d_0,
//   res_j = res_{j-1} - A d_{j-1},  d_j = c1_j d_{j-1} + c2_j D^-1 res_j,
//   z_{j+1} = z_j + d_j,
// theta = (a+b)/2.  With fixed coefficients z is a fixed polynomial in
// D^-1 A applied to D^-1 r: symmetric, and positive definite when b bounds
// the spectrum.  The pass that produces the final z also reduces
// <r, z> and <z, q> for the flexible CG step (fcg_finish).
__device__ __forceinline__ void fcg_finish(double rz, double zq, double *scal, double *partials,
                                           unsigned int *counter, double *sh) {
  double pv[2] = {rz, zq};
  if (publish_partials<2>(pv, partials, counter, gridDim.x)) {
    const double rz_t = fold_partials<false>(partials, gridDim.x, sh);
    const double zq_t = fold_partials<false>(partials + gridDim.x, gridDim.x, sh);
    if (threadIdx.x == 0) {
      // Polak-Ribiere beta = <z, r - r_old> / <z_old, r_old>, with
      // r - r_old = -alpha q: robust to a preconditioner that is not
      // exactly linear (FP32 rounding)
      const double beta = scal[S_FIRST] != 0.0 ? 0.0 : -scal[S_ALPHA] * zq_t / scal[S_ZR];
      scal[S_BETA] = beta;
      scal[S_ZR] = rz_t;
      scal[S_RHO] = rz_t;
      scal[S_FIRST] = 0.0;
      if (!isfinite(beta) || !isfinite(rz_t) || !(rz_t > 0.0)) {
        scal[S_FLAG] = 1.0;
        scal[S_DONE] = 2.0;
      }
      *counter = 0;
    }
  }
}

// Fletcher-Reeves form for the multigrid preconditioner (a fixed symmetric
// operator up to FP32 rounding): beta = <r, z> / <r_old, z_old>.
__device__ __forceinline__ void fcg_finish_fr(double rz, double *scal, double *partials,
                                              unsigned int *counter, double *sh) {
  double pv[1] = {rz};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    const double rz_t = fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      const double beta = scal[S_FIRST] != 0.0 ? 0.0 : rz_t / scal[S_ZR];
      scal[S_BETA] = beta;
      scal[S_ZR] = rz_t;
      scal[S_RHO] = rz_t;
      scal[S_FIRST] = 0.0;
      if (!isfinite(beta) || !isfinite(rz_t) || !(rz_t > 0.0)) {
        scal[S_FLAG] = 1.0;
        scal[S_DONE] = 2.0;
      }
      *counter = 0;
    }
  }
}

// res = (float) r, d = z = dinv res / theta  (last: also the FCG scalars)
__global__ void __launch_bounds__(RED_THREADS)
    k_cheb_init(int64_t nL, const double *__restrict__ r, const float *__restrict__ dinv, float c0,
                float *__restrict__ res, float *__restrict__ d, float *__restrict__ z, int last,
                const double *__restrict__ q, double *scal, double *partials,
                unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  double rz = 0.0, zq = 0.0;
  GRID_STRIDE(c, nL) {
    const double r64 = r[c];
    const float rc = (float)r64;
    const float dc = c0 * (dinv[c] * rc);
    z[c] = dc;
    if (last) {
      rz += r64 * (double)dc;
      zq += (double)dc * q[c];
    } else {
      res[c] = rc;
      d[c] = dc;
    }
  }
  if (!last) return;
  rz = block_reduce<false>(rz, sh);
  zq = block_reduce<false>(zq, sh);
  fcg_finish(rz, zq, scal, partials, counter, sh);
}

// res -= mask assemble(qE) (= A d), d = c1 d + c2 dinv res, z += d
template <class MAP>
__global__ void __launch_bounds__(RED_THREADS)
    k_cheb_step(int64_t nL, MAP map, Weights wt, const float *__restrict__ qE,
                const float *__restrict__ dinv, float c1, float c2, float *__restrict__ res,
                float *__restrict__ d, float *__restrict__ z, int last,
                const double *__restrict__ r, const double *__restrict__ q, double *scal,
                double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  double rz = 0.0, zq = 0.0;
  map.template rows_sum<float>(qE, [&](int64_t c, float s) {
    if (wt.maskL && !wt.maskL[c]) s = 0.0f;
    const float rc = res[c] - s;
    const float dc = c1 * d[c] + c2 * (dinv[c] * rc);
    const float zc = z[c] + dc;
    z[c] = zc;
    if (last) {
      rz += r[c] * (double)zc;
      zq += (double)zc * q[c];
    } else {
      res[c] = rc;
      d[c] = dc;
    }
  });
  if (!last) return;
  rz = block_reduce<false>(rz, sh);
  zq = block_reduce<false>(zq, sh);
  fcg_finish(rz, zq, scal, partials, counter, sh);
}

// w = z + beta w  (FP64 search direction, FP32 or FP64 preconditioned
// residual)
template <typename TZ>
__global__ void k_fcg_w(int64_t nL, double *__restrict__ w, const TZ *__restrict__ z,
                        const double *scal) {
  if (scal[S_DONE] != 0.0) return;
  const double beta = scal[S_BETA];
  GRID_STRIDE(c, nL) { w[c] = fma(beta, w[c], (double)z[c]); }
}

// local diagonal of p L + q M at every element-local node
// gmet (deformed / embedded elements): packed G_ij with W and Jac; the
// diagonal is then sum_i sum_m D(m,l_i)^2 G_ii(line node m) plus, for
// i != j, D(l_i,l_i) D(l_j,l_j) G_ij at the node itself.
__global__ void k_helm_diag(int64_t n, int dim, int nb, Basis<double, GF_MAXN> B,
                            const double *__restrict__ egeom, const double *__restrict__ ngeom,
                            const double *__restrict__ gmet, double p, double q, int use_mass,
                            double *__restrict__ diag) {
  const int nn = dim == 2 ? nb * nb : nb * nb * nb;
  GRID_STRIDE(i, n) {
    const int64_t e = i / nn;
    const int a = (int)(i % nn);
    const int li[3] = {a % nb, (a / nb) % nb, a / (nb * nb)};
    const int stride[3] = {1, nb, nb * nb};
    double s = 0.0;
    for (int d = 0; d < dim; d++) {
      for (int m = 0; m < nb; m++) {
        const double Dm = B.D[m + li[d] * nb];
        const int64_t gb = i + (int64_t)(m - li[d]) * stride[d];
        if (gmet) {
          s += Dm * Dm * gmet[(int64_t)gpack(d, d, dim) * n + gb];
          continue;
        }
        const int b = (int)(gb % nn);
        const int bi = b % nb, bj = (b / nb) % nb, bk = b / (nb * nb);
        double X, J;
        if (egeom) {
          X = egeom[e * (dim + 1) + d];
          J = egeom[e * (dim + 1) + dim];
        } else {
          X = ngeom[(int64_t)d * n + gb];
          J = ngeom[(int64_t)dim * n + gb];
        }
        const double w = dim == 2 ? B.W[bj] * B.W[bi] : B.W[bk] * B.W[bj] * B.W[bi];
        s += Dm * Dm * (X * X) * (w * J);
      }
    }
    if (gmet)
      for (int a1 = 0; a1 < dim; a1++)
        for (int a2 = 0; a2 < dim; a2++)
          if (a1 != a2)
            s += B.D[li[a1] + li[a1] * nb] * B.D[li[a2] + li[a2] * nb] *
                 gmet[(int64_t)gpack(a1, a2, dim) * n + i];
    s *= p;
    if (use_mass) {
      const double J = egeom ? egeom[e * (dim + 1) + dim] : ngeom[(int64_t)dim * n + i];
      const double w = dim == 2 ? B.W[li[1]] * B.W[li[0]] : B.W[li[2]] * B.W[li[1]] * B.W[li[0]];
      s += q * (w * J);
    }
    diag[i] = s;
  }
}

__global__ void k_invert(int64_t n, const double *__restrict__ d, double *__restrict__ o64,
                         float *__restrict__ o32) {
  GRID_STRIDE(i, n) {
    const double v = 1.0 / d[i];
    o64[i] = v;
    o32[i] = (float)v;
  }
}

// ---- multigrid preconditioner kernels (FP32 or FP64, lattice L-vectors) ----
// Transfers between the lattices of two levels are tensor products of 1-d
// operators, P = P_z (x) P_y (x) P_x: a fine lattice point takes the
// coarse element's GLL interpolant at its position, and the restriction
// is P^T.  Each is applied one direction at a time.

// 1-d transfer between the lattices of two levels along one direction.
// Each coarse element spans R = ratio * pf fine lattice intervals; the
// fine point at offset r = 0..R in coarse element ec takes
// sum_a J[r][a] x_c(ec pc + a) (J[0] and J[R] are unit rows: shared
// vertices coincide).  The restriction is the transpose, gathered per
// coarse point.  Periodic directions wrap (Mf = nec R, Mc = nec pc).
// The multigrid runs in TM = float (the FP32 V-cycle) or double (the FP64
// V-cycle); the transfer weights are stored in TM.
constexpr int MG_XR = 2 * GF_MAXN + 1;
template <typename TM>
struct Xfer1D {
  int R, pc, nec, per, Mf, Mc;
  TM J[MG_XR * GF_MAXN];  // J[r * (pc + 1) + a]
};

__device__ __forceinline__ float mg_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double mg_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float mg_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mg_add(double a, double b) { return __dadd_rn(a, b); }

// out = T in along direction d (transpose: T^T); in and out are lattices
// of extents ei and eo that differ only in direction d.
// mode 0: out = s; 1: out += s; 2: out = mask ? s : 0 (mask of the output)
template <typename TM>
__global__ void k_xfer1d(int64_t nout, int d, int eo0, int eo1, int ei0, int ei1,
                         const __grid_constant__ Xfer1D<TM> T, int transpose,
                         const TM *__restrict__ in, TM *__restrict__ out,
                         const uint8_t *__restrict__ mask, int mode, const double *stop) {
  if (stop && *stop != 0.0) return;
  const int R = T.R, pc = T.pc, nc = T.pc + 1, nec = T.nec;
  // the weights in shared memory: along x the threads of a warp read
  // different rows, which the constant (parameter) bank would serialise
  __shared__ TM J[MG_XR * GF_MAXN];
  for (int i = threadIdx.x; i < (R + 1) * nc; i += blockDim.x) J[i] = T.J[i];
  __syncthreads();
  // lattice sizes are below 2^31 (32-bit index arithmetic)
  const int n32 = (int)nout;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n32; o += gridDim.x * blockDim.x) {
    const unsigned uo = (unsigned)o, ue0 = (unsigned)eo0, ue1 = (unsigned)eo1;
    const unsigned rr = uo / ue0;
    const int g0 = (int)(uo - rr * ue0);
    const unsigned q1 = rr / ue1;
    const int g1 = (int)(rr - q1 * ue1), g2 = (int)q1;
    int base, stride, gd;
    if (d == 0) {
      gd = g0;
      base = ei0 * (g1 + ei1 * g2);
      stride = 1;
    } else if (d == 1) {
      gd = g1;
      base = g0 + ei0 * ei1 * g2;
      stride = ei0;
    } else {
      gd = g2;
      base = g0 + ei0 * g1;
      stride = ei0 * ei1;
    }
    TM s = 0;
    if (!transpose) {  // fine point gd from coarse element ec
      const int ec = min(gd / R, nec - 1), r = gd - ec * R;
      for (int a = 0; a < nc; a++) {
        int c = ec * pc + a;
        if (c >= T.Mc) c -= T.Mc;
        s = mg_fma(J[r * nc + a], in[base + c * stride], s);
      }
    } else {  // coarse point gd = ec pc + a
      const int ec = gd / pc, a = gd - ec * pc;
      if (a != 0) {
        for (int r = 1; r < R; r++)
          s = mg_fma(J[r * nc + a], in[base + (ec * R + r) * stride], s);
      } else {
        s = in[base + (ec * R) * stride];  // the coinciding vertex
        const bool left = ec > 0 || T.per, right = ec < nec;
        if (left) {
          const int el = ec > 0 ? ec - 1 : nec - 1;
          for (int r = 1; r < R; r++)
            s = mg_fma(J[r * nc + pc], in[base + (el * R + r) * stride], s);
        }
        if (right)
          for (int r = 1; r < R; r++)
            s = mg_fma(J[r * nc], in[base + (ec * R + r) * stride], s);
      }
    }
    if (mode == 2 && mask && !mask[o]) s = 0;
    if (mode == 1) out[o] += s;
    else out[o] = s;
  }
}

// ---- transfers between p-levels (same elements), one element per
// thread-block slot: with P = J (x) J (x) J element by element (J the
// NF x NC interpolation of Xfer1D with ratio 1), no 1-d sweeps and no
// intermediate lattices.  3-d box lattices.  The lattice coordinate of
// local index l in element coordinate c along a direction is c P + l,
// wrapped to 0 at M when the direction is periodic.

// The element-wise transfers are sum-factorised one line per thread: each
// stage contracts one direction, a thread taking a whole line of the
// previous stage from shared memory (rows padded to an odd stride, so the
// lines of a warp fall in distinct banks) and the 1-d weights J(r, a) as
// compile-time operands of the kernel parameter.  Every output is the
// same fma chain from 0 in ascending index as a staged loop would form.
template <int K>
struct PadOdd {
  static constexpr int value = (K % 2) ? K : K + 1;
};

// prolongation x_f += P x_c: gather the coarse element, contract along x,
// y, z, add into the fine lattice points the element owns (local index < P,
// or P on a non-periodic upper face), so each point is written once.
template <int NF, typename TM>
__global__ void __launch_bounds__(NF *NF *((256 / (NF * NF)) < 1 ? 1 : 256 / (NF * NF)))
    k_pxfer_prolong(BoxLattice Lf, BoxLattice Lc, const __grid_constant__ Xfer1D<TM> T,
                    const TM *__restrict__ xc, TM *__restrict__ xf, const double *stop) {
  constexpr int NC = NF / 2 + 1, PF = NF - 1, NT = NF * NF;
  constexpr int EPB = (256 / NT) < 1 ? 1 : 256 / NT;
  constexpr int CP = PadOdd<NC>::value;
  // s0[c][b][a] (rows of CP), s1[(c NF + i0) CP + b], s2[(j NF + i0) CP + c]
  constexpr int S0 = NC * NC * CP, S1 = NC * NF * CP, S2 = NF * NF * CP;
  __shared__ TM sm[EPB][S0 + S1 + S2];
  if (stop && *stop != 0.0) return;
  const int t = threadIdx.x, slot = threadIdx.y;
  const int ne0 = Lf.ne[0], ne1 = Lf.ne[1], ne2 = Lf.ne[2];
  const int nel = ne0 * ne1 * ne2;
  const int e = blockIdx.x * EPB + slot;
  const bool active = e < nel;
  const int r = e / ne0, c0 = e - r * ne0, c2 = r / ne1, c1 = r - c2 * ne1;
  TM *s0 = sm[slot], *s1 = s0 + S0, *s2 = s1 + S1;
  if (active && t < NC * NC) {  // the coarse element, one z-line (a, b) per thread
    const int a = t % NC, b = t / NC, Pc = Lc.p;
    const int M0 = (int)Lc.M[0], M1 = (int)Lc.M[1], M2 = (int)Lc.M[2];
    int g0 = c0 * Pc + a, g1 = c1 * Pc + b;
    if (Lc.per[0] && g0 == M0) g0 = 0;
    if (Lc.per[1] && g1 == M1) g1 = 0;
    const TM *row = xc + g0 + M0 * g1;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      int g2 = c2 * Pc + c;
      if (Lc.per[2] && g2 == M2) g2 = 0;
      s0[(c * NC + b) * CP + a] = row[(int64_t)M0 * M1 * g2];
    }
  }
  __syncthreads();
  if (active && t < NC * NC) {  // x: line (b, c) -> s1[c][i0][b]
    const int b = t % NC, c = t / NC;
    TM in[NC];
#pragma unroll
    for (int a = 0; a < NC; a++) in[a] = s0[(c * NC + b) * CP + a];
#pragma unroll
    for (int i0 = 0; i0 < NF; i0++) {
      TM v = 0;
#pragma unroll
      for (int a = 0; a < NC; a++) v = mg_fma(T.J[i0 * NC + a], in[a], v);
      s1[(c * NF + i0) * CP + b] = v;
    }
  }
  __syncthreads();
  if (active && t < NC * NF) {  // y: line (i0, c) -> s2[j][i0][c]
    const int i0 = t % NF, c = t / NF;
    TM in[NC];
#pragma unroll
    for (int b = 0; b < NC; b++) in[b] = s1[(c * NF + i0) * CP + b];
#pragma unroll
    for (int j = 0; j < NF; j++) {
      TM v = 0;
#pragma unroll
      for (int b = 0; b < NC; b++) v = mg_fma(T.J[j * NC + b], in[b], v);
      s2[(j * NF + i0) * CP + c] = v;
    }
  }
  __syncthreads();
  if (!active) return;
  const int i0 = t % NF, j = t / NF;  // z: line (i0, j)
  if (i0 == PF && (Lf.per[0] || c0 != ne0 - 1)) return;
  if (j == PF && (Lf.per[1] || c1 != ne1 - 1)) return;
  TM in[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) in[c] = s2[(j * NF + i0) * CP + c];
  const int M0 = (int)Lf.M[0], M1 = (int)Lf.M[1], M2 = (int)Lf.M[2];
  int g0 = c0 * PF + i0, g1 = c1 * PF + j;
  if (Lf.per[0] && g0 == M0) g0 = 0;
  if (Lf.per[1] && g1 == M1) g1 = 0;
  TM *row = xf + g0 + M0 * g1;
  // the line's current values first (all loads in flight together), then
  // x += P x_c point by point
  const bool top = !Lf.per[2] && c2 == ne2 - 1;  // owns its k = P points
  int64_t off[NF];
  TM old[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    int g2 = c2 * PF + k;
    if (Lf.per[2] && g2 == M2) g2 = 0;
    off[k] = (int64_t)M0 * M1 * g2;
    old[k] = (k < PF || top) ? row[off[k]] : TM(0);
  }
#pragma unroll
  for (int k = 0; k < NF; k++) {
    if (k == PF && !top) continue;
    TM v = 0;
#pragma unroll
    for (int c = 0; c < NC; c++) v = mg_fma(T.J[k * NC + c], in[c], v);
    row[off[k]] = old[k] + v;
  }
}

// restriction into the coarse E-vector: q_c(e) = (J^T (x) J^T (x) J^T)
// (w r_f)(e), w = 1/(number of elements sharing the fine point), so that
// folding q_c's copies over the coarse lattice gives P^T r_f.
template <int NF, typename TM>
__global__ void __launch_bounds__(NF *NF *((256 / (NF * NF)) < 1 ? 1 : 256 / (NF * NF)))
    k_pxfer_restrict(BoxLattice Lf, const __grid_constant__ Xfer1D<TM> T,
                     const TM *__restrict__ rf, TM *__restrict__ qc, const double *stop) {
  constexpr int NC = NF / 2 + 1, PF = NF - 1, NT = NF * NF;
  constexpr int EPB = (256 / NT) < 1 ? 1 : 256 / NT;
  constexpr int FP = PadOdd<NF>::value;
  // s0[k][j][i0] (rows of FP), s1[(k NC + a) FP + j], s2[(b NC + a) FP + k]
  constexpr int S0 = NF * NF * FP, S1 = NF * NC * FP, S2 = NC * NC * FP;
  __shared__ TM sm[EPB][S0 + S1 + S2];
  if (stop && *stop != 0.0) return;
  const int t = threadIdx.x, slot = threadIdx.y;
  const int ne[3] = {Lf.ne[0], Lf.ne[1], Lf.ne[2]};
  const int nel = ne[0] * ne[1] * ne[2];
  const int e = blockIdx.x * EPB + slot;
  const bool active = e < nel;
  const int r = e / ne[0], q = r / ne[1];
  const int cc[3] = {e - r * ne[0], r - q * ne[1], q};
  TM *s0 = sm[slot], *s1 = s0 + S0, *s2 = s1 + S1;
  if (active) {
    // the element's fine points, one z-line (l0, l1) per thread, each
    // weighted by 1/2 per direction in which the point is shared (an exact
    // power of two)
    const int l0 = t % NF, l1 = t / NF;
    const int M0 = (int)Lf.M[0], M1 = (int)Lf.M[1], M2 = (int)Lf.M[2];
    auto shared = [&](int l, int d) {
      return (l == 0 && (Lf.per[d] || cc[d] > 0)) || (l == PF && (Lf.per[d] || cc[d] < ne[d] - 1));
    };
    TM wxy = 1;
    if (shared(l0, 0)) wxy *= TM(0.5);
    if (shared(l1, 1)) wxy *= TM(0.5);
    int g0 = cc[0] * PF + l0, g1 = cc[1] * PF + l1;
    if (Lf.per[0] && g0 == M0) g0 = 0;
    if (Lf.per[1] && g1 == M1) g1 = 0;
    const TM *row = rf + g0 + M0 * g1;
#pragma unroll
    for (int l2 = 0; l2 < NF; l2++) {
      TM w = wxy;
      if (shared(l2, 2)) w *= TM(0.5);
      int g2 = cc[2] * PF + l2;
      if (Lf.per[2] && g2 == M2) g2 = 0;
      s0[(l2 * NF + l1) * FP + l0] = w * row[(int64_t)M0 * M1 * g2];
    }
  }
  __syncthreads();
  if (active) {  // x: line (j, k) -> s1[k][a][j]
    const int j = t % NF, k = t / NF;
    TM in[NF];
#pragma unroll
    for (int i0 = 0; i0 < NF; i0++) in[i0] = s0[(k * NF + j) * FP + i0];
#pragma unroll
    for (int a = 0; a < NC; a++) {
      TM v = 0;
#pragma unroll
      for (int i0 = 0; i0 < NF; i0++) v = mg_fma(T.J[i0 * NC + a], in[i0], v);
      s1[(k * NC + a) * FP + j] = v;
    }
  }
  __syncthreads();
  if (active && t < NF * NC) {  // y: line (a, k) -> s2[b][a][k]
    const int a = t % NC, k = t / NC;
    TM in[NF];
#pragma unroll
    for (int j = 0; j < NF; j++) in[j] = s1[(k * NC + a) * FP + j];
#pragma unroll
    for (int b = 0; b < NC; b++) {
      TM v = 0;
#pragma unroll
      for (int j = 0; j < NF; j++) v = mg_fma(T.J[j * NC + b], in[j], v);
      s2[(b * NC + a) * FP + k] = v;
    }
  }
  __syncthreads();
  if (!active || t >= NC * NC) return;
  const int a = t % NC, b = t / NC;  // z: line (a, b) -> q[c][b][a]
  TM in[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) in[k] = s2[(b * NC + a) * FP + k];
#pragma unroll
  for (int c = 0; c < NC; c++) {
    TM v = 0;
#pragma unroll
    for (int k = 0; k < NF; k++) v = mg_fma(T.J[k * NC + c], in[k], v);
    qc[(int64_t)e * (NC * NC * NC) + (c * NC + b) * NC + a] = v;
  }
}

// Chebyshev smoothing of A x = b from x = 0 (the recurrence of k_cheb_*),
// first term: x = c0 Dinv b.  With r64 the level's b is first taken from
// the FP64 outer residual.
template <typename TM>
__global__ void k_mg_start(int64_t nL, const double *__restrict__ r64, TM *__restrict__ b,
                           const TM *__restrict__ dinv, TM c0, TM *__restrict__ x,
                           const double *stop) {
  if (stop && *stop != 0.0) return;
  GRID_STRIDE(c, nL) {
    const TM bc = r64 ? (TM)r64[c] : b[c];
    if (r64) b[c] = bc;
    x[c] = c0 * (dinv[c] * bc);
  }
}

// Passes that fold the element-local qE = A x into the lattice (s = mask *
// sum of copies) and advance the smoother state:
//   MG_STEP   r = b - s; d = a1 dprev + a2 Dinv r; x += d, with dprev
//             DP_NONE  (none: smoothing of the residual equation from an
//                       existing x, the first post-smoothing term),
//             DP_X     (x: the step after a start from zero, where d = x),
//             DP_D     (the stored d);
//             d is stored only when a later step reads it (wd)
//   MG_RESID  res = b - s                  (the residual to restrict)
//   MG_START  qE = a coarse E-vector (the element restriction's output):
//             b = s; x = a1 Dinv b         (smoothing from zero)
//   MG_FOLDB  b = s only (a dense coarsest level)
// DOTS (last pass of the finest level): <b, x> (b = the copy of the outer
// residual in the multigrid's type) for the CG step, finished by
// fcg_finish_fr.
// Applying x rather than the step direction keeps the running residual out
// of the smoother state: a step reads b, dinv, x (and d) and writes x (and
// d); mathematically the same Chebyshev polynomial.
enum { MG_STEP = 0, MG_RESID = 1, MG_START = 3, MG_FOLDB = 4 };
enum { DP_NONE = 0, DP_X = 1, DP_D = 2 };

// One thread per lattice point, in lattice order (grid-stride over the
// flat index): the state vectors stream fully coalesced, and a warp's
// copies of one element row are one 32-byte sector of qE.  The point's
// coordinates come from two multiply-shift divisions, its copies from
// scalar offsets (no local arrays), its state loads are issued before the
// gather (one memory round trip per point), and the copies are added in the
// (z, y, x) nesting of MapBox::rows_sum (ascending element id unless a
// periodic direction has a single element).  Lattice and element-local
// sizes are below 2^31 (checked when the problem is created).
// (Measured on B200 against this form: element-ordered walks, lattice rows
// mapped to power-of-two thread groups, several points per thread, z-column
// walks and a lattice-row layout of qE were all slower.)
template <int N, int MODE, bool DOTS, typename TM>
__global__ void __launch_bounds__(RED_THREADS)
    k_mg_pass_lat(MapBox<N> map, Weights wt,
                  const TM *__restrict__ qE, TM *__restrict__ b,
                  const TM *__restrict__ dinv, TM c1, TM c2, TM *__restrict__ res,
                  TM *__restrict__ d, TM *__restrict__ x, int dsrc, int wd, double *scal,
                  double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  constexpr int P = N - 1, NN = N * N;
  double rz = 0.0;
  const bool d3 = map.dim > 2;
  const int nn = d3 ? NN * N : NN;
  const int ne0 = map.ne[0], ne1 = map.ne[1];
  const int M0 = map.M[0], M1 = map.M[1];
  const int nL = M0 * M1 * (d3 ? map.M[2] : 1);
  const int sy = ne0 * nn, sz = ne0 * ne1 * nn;
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nL;
       c = (c < nL - stride) ? c + stride : nL) {
    const bool keep = !wt.maskL || wt.maskL[c];
    TM bc = 0, xo = 0, dv = 0, dpv = 0;
    if (MODE == MG_STEP || MODE == MG_RESID) bc = b[c];
    if (MODE == MG_STEP || MODE == MG_START) dv = dinv[c];
    if (MODE == MG_STEP) {
      xo = x[c];
      if (dsrc == DP_D) dpv = d[c];
    }
    const int row = map.fd0.div(c), g0 = c - row * M0;
    const int g2 = map.fd1.div(row), g1 = row - g2 * M1;
    int ox0, ox1, oy0, oy1, oz0 = 0, oz1 = 0;
    const int nx = lattice_offsets<P>(g0, ne0, map.per[0], nn, 1, ox0, ox1);
    const int ny = lattice_offsets<P>(g1, ne1, map.per[1], sy, N, oy0, oy1);
    const int nz = d3 ? lattice_offsets<P>(g2, map.ne[2], map.per[2], sz, NN, oz0, oz1) : 1;
    TM s = 0;
#pragma unroll
    for (int az = 0; az < 2; az++) {
      if (az >= nz) break;
      const int oz = az ? oz1 : oz0;
#pragma unroll
      for (int ay = 0; ay < 2; ay++) {
        if (ay >= ny) break;
        const int o = oz + (ay ? oy1 : oy0);
        s = mg_add(s, qE[o + ox0]);
        if (nx > 1) s = mg_add(s, qE[o + ox1]);
      }
    }
    if (!keep) s = 0;
    if (MODE == MG_FOLDB) {
      b[c] = s;
      continue;
    }
    if (MODE == MG_START) {
      b[c] = s;
      x[c] = c1 * (dv * s);
      continue;
    }
    const TM rc = bc - s;
    if (MODE == MG_RESID) {
      res[c] = rc;
      continue;
    }
    const TM dp = dsrc == DP_X ? xo : dpv;
    const TM dc = c1 * dp + c2 * (dv * rc);
    const TM xc = xo + dc;
    x[c] = xc;
    if (wd) d[c] = dc;
    if (DOTS) rz += (double)bc * (double)xc;
  }
  if (!DOTS) return;
  rz = block_reduce<false>(rz, sh);
  fcg_finish_fr(rz, scal, partials, counter, sh);
}

// condition of the solve loop's WHILE graph node: continue while the CG
// state is not done
__global__ void k_while_more(cudaGraphConditionalHandle h, const double *scal) {
  cudaGraphSetConditional(h, scal[S_DONE] == 0.0 ? 1u : 0u);
}

// deterministic pseudo-random vector in [-1, 1) (zero where masked): the
// start of the eigenvalue estimates
__global__ void k_fill_hash(int64_t n, const uint8_t *__restrict__ mask, double *__restrict__ v) {
  GRID_STRIDE(i, n) {
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
    v[i] = (mask && !mask[i]) ? 0.0 : 2.0 * u - 1.0;
  }
}

// coarsest-level solve x[free_i] = sum_j Ainv(i, j) b[free_j]: one block
// per row (the masked points of x stay 0)
template <typename TM>
__global__ void __launch_bounds__(128)
    k_dense_solve(int64_t nfree, const TM *__restrict__ ainv, const int32_t *__restrict__ idx,
                  const TM *__restrict__ b, TM *__restrict__ x, const double *stop) {
  if (stop && *stop != 0.0) return;
  __shared__ TM sh[4];
  for (int64_t i = blockIdx.x; i < nfree; i += gridDim.x) {
    const TM *row = ainv + i * nfree;
    TM s = 0;
    for (int64_t j = threadIdx.x; j < nfree; j += blockDim.x) s = mg_fma(row[j], b[idx[j]], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) x[idx[i]] = (sh[0] + sh[1]) + (sh[2] + sh[3]);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------
// Largest eigenvalue of the Lanczos tridiagonal built from n PCG steps
// (alpha_j, beta_j = rho_{j+1}/rho_j): T_jj = 1/alpha_j + beta_{j-1}/alpha_{j-1},
// T_j,j+1 = sqrt(beta_j)/alpha_j.  Its eigenvalues are Ritz values of the
// preconditioned operator, the largest converging fast from below.
// Bisection on the Sturm count; returns 0 when the coefficients are unusable.
double lanczos_max(const double *ab, int n) {
  std::vector<double> dg(n), off(n > 1 ? n - 1 : 1, 0.0);
  for (int j = 0; j < n; j++) {
    const double a = ab[2 * j], b = ab[2 * j + 1];
    if (!(a > 0.0) || !std::isfinite(a) || !(b >= 0.0) || !std::isfinite(b)) return 0.0;
    dg[j] = 1.0 / a + (j > 0 ? ab[2 * j - 1] / ab[2 * (j - 1)] : 0.0);
    if (j < n - 1) off[j] = std::sqrt(b) / a;
  }
  double lo = 0.0, hi = 0.0;
  for (int j = 0; j < n; j++) {
    const double r = (j > 0 ? std::fabs(off[j - 1]) : 0.0) + (j < n - 1 ? std::fabs(off[j]) : 0.0);
    hi = std::max(hi, dg[j] + r);
  }
  auto below = [&](double x) {  // eigenvalues < x
    int cnt = 0;
    double qv = 1.0;
    for (int j = 0; j < n; j++) {
      qv = dg[j] - x - (j > 0 ? off[j - 1] * off[j - 1] / qv : 0.0);
      if (qv == 0.0) qv = -1e-300;
      if (qv < 0.0) cnt++;
    }
    return cnt;
  };
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= n) hi = mid;
    else lo = mid;
  }
  return hi;
}

template <class MAP>
struct Solver;
// multigrid preconditioner (defined after Solver): set-up or reuse of the
// hierarchy, and the FP64 flexible CG that applies it
template <class MAP>
int mg_prepare(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass);
template <class MAP>
int solve_mg(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass,
             const double *bL, double *xL, double *rL, double *qE, double *hist, int *total,
             double *rn);

template <class MAP>
struct Solver {
  gf_problem *prob;
  gf_context *ctx;
  cudaStream_t st;
  MAP map;
  Weights wt;
  int64_t nE, nL;
  unsigned gE, gL, gRed;
  double *ab = nullptr;  // alpha, beta of the first nab iterations (Lanczos)
  int nab = 0;

  // Grid of a grid-stride reduction kernel: the blocks that are resident at
  // once (occupancy x SMs, cached per kernel), so every block runs in the
  // first wave; capped by gRed (work and partial-sum slots).
  template <class K>
  unsigned rgrid(K kern) {
    static std::unordered_map<const void *, int> occ;
    auto it = occ.find((const void *)kern);
    int nb = 0;
    if (it == occ.end()) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, RED_THREADS, 0) != cudaSuccess)
        nb = 1;
      occ[(const void *)kern] = nb;
    } else {
      nb = it->second;
    }
    return std::max(1u, std::min(gRed, (unsigned)(std::max(nb, 1) * ctx->sm_count)));
  }

  Solver(gf_problem *p, MAP m, bool masked)
      : prob(p), ctx(p->ctx), st(p->ctx->stream), map(m), nE(p->nlocal), nL(p->nclass) {
    wt.maskL = masked ? p->maskL8 : nullptr;
    wt.massL = p->massL;
    wt.multL = p->multL8;
    gE = grid_for(nE, 256, ctx->sm_count * 8);
    gL = grid_for(nL, 256, ctx->sm_count * 8);
    gRed = grid_for(nL, RED_THREADS, std::min(p->npartials, ctx->sm_count * 8));
  }

  void set_scalars(const gf_cg_traits &tr, int maxit, bool relative) {
    double *h = prob->scal_h;
    for (int i = 0; i < S_COUNT; i++) h[i] = 0.0;
    h[S_MAXIT] = (double)maxit;
    h[S_NTOT] = (double)nE;
    h[S_NORMT] = (double)tr.normtype;
    h[S_IVOL] = 1.0 / prob->volume;
    h[S_REL] = relative ? 1.0 : 0.0;
    h[S_INNER] = (tr.precision == GF_CG_MIXED && tr.inner_tol > 0.0) ? tr.inner_tol : 0.0;
  }

  // Jacobi inverse diagonal on unique nodes (FP64 and FP32), slots 8/9/10
  int jacobi(double p, double q, int use_mass, double **d64, float **d32) {
    double *dE = (double *)gf_work(prob, 8, sizeof(double) * nE);
    double *dL = (double *)gf_work(prob, 9, sizeof(double) * nL);
    float *fL = (float *)gf_work(prob, 10, sizeof(float) * nL);
    double *iL = (double *)gf_work(prob, 7, sizeof(double) * nL);
    if (!dE || !dL || !fL || !iL) return GF_ERR_NOMEM;
    Basis<double, GF_MAXN> B;
    for (int i = 0; i < prob->n * prob->n; i++) B.D[i] = prob->D[i];
    for (int i = 0; i < prob->n; i++) B.W[i] = prob->W[i];
    prob->launches += 3;
    k_helm_diag<<<gE, 256, 0, st>>>(nE, prob->dim, prob->n, B, prob->egeom_d, prob->ngeom_d,
                                    prob->gmet_d, p, q, use_mass, dE);
    k_assemble<MAP, double><<<gL, 256, 0, st>>>(nL, map, dE, dL);
    k_invert<<<gL, 256, 0, st>>>(nL, dL, iL, fL);
    *d64 = iL;
    *d32 = fL;
    return GF_OK;
  }

  // enqueue k CG iterations in precision T (each returns at once once the
  // device `done` flag is set)
  int mixed_apply = 0;  // FP64 arithmetic in the FP32 applies

  template <typename T>
  void enqueue(int k, double p, double q, int use_mass, T *x, T *r, T *w, T *qL, T *qE,
               const float *dinv, double *hist) {
    double *scal = prob->scal_d;
    for (int i = 0; i < k; i++) {
      if (std::is_same<T, float>::value && mixed_apply && prob->dim == 3)
        launch_helm_L_f32io(prob, p, q, use_mass, (const float *)w, (float *)qE, st, scal + S_DONE);
      else
        launch_helm_L<T>(prob, (T)p, (T)q, use_mass, w, qE, st, scal + S_DONE);
      k_asm_dot<T, MAP><<<rgrid(k_asm_dot<T, MAP>), RED_THREADS, 0, st>>>(nL, map, wt, qE, w, qL, scal, prob->partials,
                                                      prob->counter);
      k_update<T, MAP><<<rgrid(k_update<T, MAP>), RED_THREADS, 0, st>>>(nL, map, wt, x, w, r, qL, dinv, hist, ab,
                                                     nab, scal, prob->partials, prob->counter);
      k_wupdate<T><<<gL, 256, 0, st>>>(nL, w, r, dinv, scal);
      prob->launches += 3;
    }
  }

  // Polynomial-preconditioned FP64 CG: per iteration the FP64 apply,
  // assembly with <w,q>, x/r update and stop test, then z = P(r) in FP32
  // (poly_degree FP32 applies) and w = z + beta w.
  struct Poly {
    int m = 0;            // FP32 applies per preconditioner application
    float c0 = 0.0f;      // 1/theta
    std::vector<float> c1, c2;  // step coefficients, index 1..m
    double *w = nullptr, *qL = nullptr;
    float *res = nullptr, *d = nullptr, *z = nullptr, *qE32 = nullptr;
    const float *dinv = nullptr;
  };

  void precondition(const Poly &P, double p, double q, int use_mass, const double *rL) {
    double *scal = prob->scal_d;
    prob->launches += 1 + P.m;  // the applies count themselves
    k_cheb_init<<<rgrid(k_cheb_init), RED_THREADS, 0, st>>>(nL, rL, P.dinv, P.c0, P.res, P.d, P.z, P.m == 0,
                                              P.qL, scal, prob->partials, prob->counter);
    for (int j = 1; j <= P.m; j++) {
      launch_helm_L<float>(prob, (float)p, (float)q, use_mass, P.d, P.qE32, st, scal + S_DONE);
      k_cheb_step<MAP><<<rgrid(k_cheb_step<MAP>), RED_THREADS, 0, st>>>(nL, map, wt, P.qE32, P.dinv, P.c1[j], P.c2[j],
                                                     P.res, P.d, P.z, j == P.m, rL, P.qL, scal,
                                                     prob->partials, prob->counter);
    }
  }

  void enqueue_poly(int k, const Poly &P, double p, double q, int use_mass, double *x, double *r,
                    double *qE, double *hist) {
    double *scal = prob->scal_d;
    for (int i = 0; i < k; i++) {
      launch_helm_L<double>(prob, p, q, use_mass, P.w, qE, st, scal + S_DONE);
      k_asm_dot<double, MAP><<<rgrid(k_asm_dot<double, MAP>), RED_THREADS, 0, st>>>(nL, map, wt, qE, P.w, P.qL, scal,
                                                           prob->partials, prob->counter);
      k_update<double, MAP><<<rgrid(k_update<double, MAP>), RED_THREADS, 0, st>>>(nL, map, wt, x, P.w, r, P.qL, nullptr,
                                                          hist, nullptr, 0, scal, prob->partials,
                                                          prob->counter);
      precondition(P, p, q, use_mass, r);
      k_fcg_w<<<gL, 256, 0, st>>>(nL, P.w, P.z, scal);
      prob->launches += 3;
    }
  }

  // FP64 flexible CG with the FP32 Chebyshev preconditioner.  The first
  // LANCZOS iterations are plain Jacobi PCG; their alpha/beta give the
  // largest eigenvalue of D^-1 A (Lanczos Ritz value, times a safety
  // factor), which fixes the polynomial's interval [b/ratio, b].  The
  // direction is then restarted with w = P(r) and CG continues with the
  // polynomial preconditioner.  Iterations count FP64 outer steps.
  static constexpr int LANCZOS = 12;
  int solve_poly(const gf_cg_traits &tr, double p, double q, int use_mass, const double *bL,
                 double *xL, double *rL, double *qE, const double *d64, const float *d32,
                 double *hist, int *total, double *rn) {
    Poly P;
    P.m = std::max(0, tr.poly_degree);
    P.dinv = d32;
    P.w = (double *)gf_work(prob, 4, sizeof(double) * nL);
    P.qL = (double *)gf_work(prob, 5, sizeof(double) * nL);
    P.res = (float *)gf_work(prob, 11, sizeof(float) * nL);
    P.d = (float *)gf_work(prob, 12, sizeof(float) * nL);
    P.z = (float *)gf_work(prob, 13, sizeof(float) * nL);
    P.qE32 = (float *)gf_work(prob, 15, sizeof(float) * nE);
    double *abd = (double *)gf_work(prob, 17, sizeof(double) * 2 * LANCZOS);
    if (!P.w || !P.qL || !P.res || !P.d || !P.z || !P.qE32 || !abd)
      return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
    int rc = residual<double>(p, q, use_mass, bL, xL, qE, rL, rL, P.w, d32, 0, tr.tol);
    if (rc) return gf_fail(ctx, rc, "residual failed");
    const int n0 = std::min(tr.maxit, LANCZOS);
    ab = abd;
    nab = n0;
    rc = iterate<double>(tr, n0, p, q, use_mass, xL, rL, P.w, P.qL, qE, d32, hist, total);
    ab = nullptr;
    nab = 0;
    if (rc) return rc;
    const double *h = prob->scal_h;
    if (h[S_DONE] == 0.0 && *total < tr.maxit) {
      double abh[2 * LANCZOS];
      GF_CUDA(ctx, cudaMemcpy(abh, abd, sizeof(double) * 2 * *total, cudaMemcpyDeviceToHost));
      const double lmax = lanczos_max(abh, *total);
      if (!(lmax > 0.0)) return gf_fail(ctx, GF_ERR_NONFINITE, "eigenvalue estimate failed");
      const double ratio = tr.poly_ratio > 1.0 ? tr.poly_ratio : std::max(4.0, 2.0 * P.m * P.m);
      const double b = 1.1 * lmax, a = b / ratio;
      const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
      P.c0 = (float)(1.0 / theta);
      P.c1.assign(P.m + 1, 0.0f);
      P.c2.assign(P.m + 1, 0.0f);
      double rho = 1.0 / sigma;
      for (int j = 1; j <= P.m; j++) {
        const double rn1 = 1.0 / (2.0 * sigma - rho);
        P.c1[j] = (float)(rn1 * rho);
        P.c2[j] = (float)(2.0 * rn1 / delta);
        rho = rn1;
      }
      // restart the direction: w = P(r)
      prob->scal_h[S_FIRST] = 1.0;
      GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_d + S_FIRST, prob->scal_h + S_FIRST, sizeof(double),
                                   cudaMemcpyHostToDevice, st));
      precondition(P, p, q, use_mass, rL);
      prob->launches++;
      k_fcg_w<<<gL, 256, 0, st>>>(nL, P.w, P.z, prob->scal_d);
      rc = batches(tr, tr.maxit - *total, total, [&](int k) {
        enqueue_poly(k, P, p, q, use_mass, xL, rL, qE, hist);
      });
      if (rc) return rc;
    }
    *rn = prob->scal_h[S_RNORM];
    return (*total >= tr.maxit && *rn > prob->scal_h[S_RTOL]) ? GF_CG_NOCONVERGE : GF_OK;
  }

  // PCG iterations in precision T on unique-node vectors; the state
  // (rho, rtol, done) was set up by k_resid.  Returns iterations done.
  template <typename T>
  int iterate(const gf_cg_traits &tr, int maxit, double p, double q, int use_mass, T *x, T *r, T *w,
              T *qL, T *qE, const float *dinv, double *hist, int *iters) {
    return batches(tr, maxit, iters, [&](int k) {
      enqueue<T>(k, p, q, use_mass, x, r, w, qL, qE, dinv, hist);
    });
  }

  // Queues iterations in batches of check_every (enq(k) queues k of them)
  // and reads the device `done` flag one batch behind, so the GPU never
  // waits for the host; stops at `done` or after maxit iterations.
  template <class ENQ>
  int batches(const gf_cg_traits &tr, int maxit, int *iters, ENQ enq) {
    double *scal = prob->scal_d;
    const int every = tr.check_every > 0 ? tr.check_every : 16;
    int issued = 0, pending = -1;
    bool stop = false;
    double *hbuf = prob->scal_h + 32;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    // the state may already be converged (maxit 0 or tol 0)
    while (!stop) {
      const int k = std::min(every, maxit - issued);
      enq(k);
      issued += k;
      GF_CHECK_LAUNCH(ctx);
      const int slot = (pending + 1) & 1;
      GF_CUDA(ctx, cudaMemcpyAsync(hbuf + 2 * slot, scal + S_DONE, sizeof(double) * 2,
                                   cudaMemcpyDeviceToHost, st));
      cudaEventRecord(ev[slot], st);
      if (pending >= 0) {
        cudaEventSynchronize(ev[pending]);
        if (hbuf[2 * pending] != 0.0) stop = true;
      }
      if (issued >= maxit) {
        cudaEventSynchronize(ev[slot]);
        stop = true;
      }
      pending = slot;
    }
    cudaStreamSynchronize(st);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h, scal, sizeof(double) * S_COUNT,
                                 cudaMemcpyDeviceToHost, st));
    GF_CUDA(ctx, cudaStreamSynchronize(st));
    *iters = (int)prob->scal_h[S_ITER];
    if (prob->scal_h[S_FLAG] != 0.0)
      return gf_fail(ctx, GF_ERR_NONFINITE, "CG breakdown: non-finite scalar at iteration %d",
                     *iters);
    return GF_OK;
  }

  // FP64 residual pass for x_L: r_L = mask (b_L - A x); writes solve-
  // precision copies rT, wT = Dinv rT and sets up the CG state.
  template <typename T>
  int residual(double p, double q, int use_mass, const double *bL, const double *xL, double *qE,
               double *rL, T *rT, T *wT, const float *dinv, int mode, double tol) {
    int rc = launch_helm_L<double>(prob, p, q, use_mass, xL, qE, st);
    if (rc) return rc;
    prob->launches++;
    k_resid<T, MAP><<<rgrid(k_resid<T, MAP>), RED_THREADS, 0, st>>>(nL, map, wt, bL, qE, rL, rT, wT, dinv, mode, tol,
                                                  prob->scal_d, prob->partials, prob->counter);
    GF_CHECK_LAUNCH(ctx);
    return GF_OK;
  }

  double read_scalar(int slot) {
    cudaMemcpyAsync(prob->scal_h + slot, prob->scal_d + slot, sizeof(double),
                    cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return prob->scal_h[slot];
  }

  int solve(const gf_cg_traits &tr, double p, double q, int use_mass, const double *bE,
            const double *xbE, double *xE, int *iters_out, double *rn_out, double *hist) {
    const bool bbv = xbE != nullptr;
    const double *maskE = bbv ? prob->mask_d : nullptr;
    double *bL = (double *)gf_work(prob, 0, sizeof(double) * nL);
    double *xL = (double *)gf_work(prob, 1, sizeof(double) * nL);
    double *rL = (double *)gf_work(prob, 2, sizeof(double) * nL);
    double *qE = (double *)gf_work(prob, 3, sizeof(double) * nE);
    if (!bL || !xL || !rL || !qE) return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
    double *d64 = nullptr;
    float *d32 = nullptr;
    const bool pmg = tr.precond == GF_PRECOND_PMG || tr.precond == GF_PRECOND_PMG64;
    if (pmg) {
      // the hierarchy's set-up runs its own short solves on this problem's
      // scalar block and work slots, so it comes before the solve's state
      int rc = mg_prepare(*this, tr, p, q, use_mass);
      if (rc) return rc;
    }
    if (tr.precond != GF_PRECOND_NONE && !pmg) {
      int rc = jacobi(p, q, use_mass, &d64, &d32);
      if (rc) return gf_fail(ctx, rc, "Jacobi set-up failed");
    }
    set_scalars(tr, tr.maxit, tr.relative != 0);
    GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_d, prob->scal_h, sizeof(double) * S_COUNT,
                                 cudaMemcpyHostToDevice, st));
    // prologue: x = mask x + xb; b_L = assemble(b); x_L = x; norm(b)
    prob->launches += 4;
    if (bbv) k_lift<<<gE, 256, 0, st>>>(nE, maskE, xbE, xE);
    k_assemble<MAP, double><<<gL, 256, 0, st>>>(nL, map, bE, bL);
    k_pick<MAP><<<gL, 256, 0, st>>>(nL, map, xE, xL);
    k_norm_E<<<grid_for(nE, RED_THREADS, prob->npartials), RED_THREADS, 0, st>>>(
        nE, tr.normtype, bE, prob->mass_d, prob->scal_d, prob->partials, prob->counter);
    int rc = GF_OK, total = 0;
    double rn = 0.0;
    if (tr.precond == GF_PRECOND_CHEBYSHEV) {
      rc = solve_poly(tr, p, q, use_mass, bL, xL, rL, qE, d64, d32, hist, &total, &rn);
      if (rc < 0) return rc;
    } else if (pmg) {
      rc = solve_mg(*this, tr, p, q, use_mass, bL, xL, rL, qE, hist, &total, &rn);
      if (rc < 0) return rc;
    } else if (tr.precision == GF_CG_FP64) {
      double *w = (double *)gf_work(prob, 4, sizeof(double) * nL);
      double *qL = (double *)gf_work(prob, 5, sizeof(double) * nL);
      if (!w || !qL) return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
      rc = residual<double>(p, q, use_mass, bL, xL, qE, rL, rL, w, d32, 0, tr.tol);
      if (rc) return gf_fail(ctx, rc, "residual failed");
      rc = iterate<double>(tr, tr.maxit, p, q, use_mass, xL, rL, w, qL, qE, d32, hist, &total);
      if (rc) return rc;
      rn = prob->scal_h[S_RNORM];
      rc = (total >= tr.maxit && rn > tr.tol) ? GF_CG_NOCONVERGE : GF_OK;
    } else {
      // mixed: FP64 residual -> FP32 PCG correction -> FP64 update
      float *r32 = (float *)gf_work(prob, 11, sizeof(float) * nL);
      float *w32 = (float *)gf_work(prob, 12, sizeof(float) * nL);
      float *x32 = (float *)gf_work(prob, 13, sizeof(float) * nL);
      float *q32 = (float *)gf_work(prob, 14, sizeof(float) * nL);
      float *qE32 = (float *)gf_work(prob, 15, sizeof(float) * nE);
      if (!r32 || !w32 || !x32 || !q32 || !qE32)
        return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
      // Reliable updates (Sleijpen & van der Vorst 1996): one FP32 PCG run
      // on the correction y; every `check_every` iterations y is folded
      // into the FP64 x and the FP32 residual is replaced by the true FP64
      // residual b - A x, keeping the search direction, so the Krylov space
      // is never restarted.  The solve stops only on the true residual.
      const int every = tr.check_every > 0 ? tr.check_every : 32;
      mixed_apply = tr.mixed_apply;
      int r2 = residual<float>(p, q, use_mass, bL, xL, qE, rL, r32, w32, d32, 0, tr.tol);
      if (r2) return gf_fail(ctx, r2, "residual failed");
      GF_CUDA(ctx, cudaMemsetAsync(x32, 0, sizeof(float) * nL, st));
      rc = GF_CG_NOCONVERGE;
      // Restarted refinement (inner_tol > 0): each FP32 PCG run solves
      // A y = r from y = 0 to inner_tol * norm(r); x += y in FP64 and the
      // next run starts on the true FP64 residual.
      for (int refine = 0; tr.inner_tol > 0.0; refine++) {
        int its = 0;
        const int left = std::max(1, tr.maxit - total);
        if ((r2 = iterate<float>(tr, left, p, q, use_mass, x32, r32, w32, q32, qE32, d32, nullptr,
                                 &its)))
          return r2;
        prob->launches += 1;
        k_add_correction<<<gL, 256, 0, st>>>(nL, x32, xL);
        GF_CUDA(ctx, cudaMemsetAsync(x32, 0, sizeof(float) * nL, st));
        r2 = residual<float>(p, q, use_mass, bL, xL, qE, rL, r32, w32, d32, 1, tr.tol);
        if (r2) return gf_fail(ctx, r2, "residual failed");
        GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h, prob->scal_d, sizeof(double) * S_COUNT,
                                     cudaMemcpyDeviceToHost, st));
        GF_CUDA(ctx, cudaStreamSynchronize(st));
        const double *h = prob->scal_h;
        total = (int)h[S_ITER];
        rn = h[S_RES];
        if (h[S_FLAG] != 0.0)
          return gf_fail(ctx, GF_ERR_NONFINITE, "CG breakdown at iteration %d", total);
        if (rn <= h[S_OTOL]) {
          rc = GF_OK;
          break;
        }
        if (total >= tr.maxit || (tr.max_refine > 0 && refine + 1 >= tr.max_refine)) break;
      }
      for (; !(tr.inner_tol > 0.0);) {
        enqueue<float>(every, p, q, use_mass, x32, r32, w32, q32, qE32, d32, nullptr);
        prob->launches += 1;
        k_add_correction<<<gL, 256, 0, st>>>(nL, x32, xL);
        GF_CUDA(ctx, cudaMemsetAsync(x32, 0, sizeof(float) * nL, st));
        r2 = residual<float>(p, q, use_mass, bL, xL, qE, rL, r32, w32, d32, 2, tr.tol);
        if (r2) return gf_fail(ctx, r2, "residual failed");
        GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h, prob->scal_d, sizeof(double) * S_COUNT,
                                     cudaMemcpyDeviceToHost, st));
        GF_CUDA(ctx, cudaStreamSynchronize(st));
        const double *h = prob->scal_h;
        total = (int)h[S_ITER];
        rn = h[S_RES];
        if (h[S_FLAG] != 0.0)
          return gf_fail(ctx, GF_ERR_NONFINITE, "CG breakdown at iteration %d", total);
        if (rn <= h[S_RTOL]) {
          rc = GF_OK;
          break;
        }
        if (total >= tr.maxit) break;
      }
    }
    // epilogue: x_E = mask x_L + xb
    prob->launches++;
    k_scatter<MAP><<<gE, 256, 0, st>>>(nE, map, xL, maskE, bbv ? xbE : nullptr, xE);
    GF_CHECK_LAUNCH(ctx);
    *iters_out = total;
    *rn_out = rn;
    return rc;
  }
};

// ---------------------------------------------------------------------
// p/h multigrid preconditioner for structured affine boxes.
//
// Levels: the problem's own order p, then ceil(p/2), ... down to 1 on the
// same elements, then the p = 1 box with the element counts halved while
// they stay even and >= 2.  Each coarser level is the same SEM Helmholtz
// operator rediscretised (GLL quadrature of its order, element geometry
// merged under h-coarsening), held as a light gf_problem: basis, K1,
// element geometry and box lattice, no gather-scatter arrays.  One V-cycle
// in FP32 (or FP64, GF_PRECOND_PMG64) on the lattice (unique-node) vectors:
//   x = S b;  r = b - A x;  x_c = V(R r);  x += P x_c;  x += S (b - A x)
// S = Chebyshev-Jacobi polynomial of degree m on [lmax/ratio, 1.1 lmax]
// (the same polynomial before and after, so the cycle is symmetric), R =
// P^T with the coarse mask, and on the coarsest level a higher-degree
// Chebyshev solve.  2m + 2 applies of each level's operator per cycle.

// h-coarsening stops at a level with at most MG_DENSE_SMALL free lattice
// points; a coarsest level with at most MG_DENSE_MAX is solved exactly
// with a dense inverse (one kernel), a larger one with a Chebyshev solve.
constexpr int64_t MG_DENSE_SMALL = 512, MG_DENSE_MAX = 729;

// TM: the type the level's vectors, smoother coefficients, transfers and
// applies use (float: the FP32 V-cycle; double: the FP64 one).
template <typename TM>
struct MGLevelBase {
  gf_problem *prob = nullptr;
  bool owned = false;
  int dim = 3;
  int64_t nL = 0, nE = 0;
  int M[3] = {1, 1, 1};
  TM *dinv = nullptr, *b = nullptr, *x = nullptr, *res = nullptr, *d = nullptr, *qE = nullptr;
  const uint8_t *maskL = nullptr;  // lattice Dirichlet mask (null: none)
  int m = 0;  // smoothing degree (the coarsest level: its solve degree)
  TM c0 = 0;
  std::vector<TM> c1, c2;
  double lmax = 0.0;
  // coarsest level: x = Ainv b on the free lattice points (dense inverse)
  int64_t nfree = 0;
  const TM *ainv = nullptr;
  const int32_t *free_idx = nullptr;
  // transfer to the next coarser level
  Xfer1D<TM> X[3];
  TM *t1 = nullptr, *t2 = nullptr;
  std::vector<void *> mem;
  TM *alloc_f(int64_t n) {
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(TM) * std::max<int64_t>(n, 1)) != cudaSuccess) return nullptr;
    mem.push_back(p);
    return (TM *)p;
  }
  template <typename V>
  V *upload(const std::vector<V> &h) {
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(V) * std::max<size_t>(h.size(), 1)) != cudaSuccess) return nullptr;
    mem.push_back(p);
    cudaMemcpy(p, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice);
    return (V *)p;
  }
  virtual ~MGLevelBase() {
    for (void *p : mem) cudaFree(p);
    if (owned && prob) gf_problem_destroy(prob);
  }
  virtual int apply(const TM *in, double p, double q, int use_mass, const double *stop,
                    cudaStream_t st) = 0;
  virtual void pass(int mode, bool dots, TM a1, TM a2, int dsrc, int wd,
                    gf_problem *outer, cudaStream_t st) = 0;
  virtual int jacobi(double p, double q, int use_mass) = 0;
  virtual int estimate(double p, double q, int use_mass, int64_t nfree) = 0;
  // element-wise transfers to the next coarser level when it has the same
  // elements (p-coarsening, 3-d): restriction into C.qE, prolongation into x
  bool ptransfer = false;
  virtual void restrict_elem(MGLevelBase &C, gf_problem *outer, cudaStream_t st) = 0;
  virtual void prolong_elem(const MGLevelBase &C, gf_problem *outer, cudaStream_t st) = 0;
};

template <int N, typename TM>
struct MGLevel : MGLevelBase<TM> {
  using B = MGLevelBase<TM>;
  using B::prob, B::owned, B::dim, B::nL, B::nE, B::M, B::dinv, B::b, B::x, B::res, B::d, B::qE,
      B::maskL, B::X, B::lmax;
  Solver<MapBox<N>> S;
  const float *dinv32 = nullptr;  // FP32 Jacobi weights of the eigenvalue estimate
  MGLevel(gf_problem *lp, bool own, bool masked) : S(lp, MapBox<N>::make(lp->box), masked) {
    prob = lp;
    owned = own;
    dim = lp->dim;
    nL = lp->nclass;
    nE = lp->nlocal;
    for (int k = 0; k < 3; k++) M[k] = (int)lp->box.M[k];
    maskL = S.wt.maskL;
  }
  int apply(const TM *in, double p, double q, int use_mass, const double *stop,
            cudaStream_t st) override {
    return launch_helm_L<TM>(prob, (TM)p, (TM)q, use_mass, in, qE, st, stop);
  }
  template <int MODE, bool DOTS>
  void run_pass(TM a1, TM a2, int dsrc, int wd, gf_problem *outer, cudaStream_t st) {
    auto kern = k_mg_pass_lat<N, MODE, DOTS, TM>;
    kern<<<S.rgrid(kern), RED_THREADS, 0, st>>>(S.map, S.wt, qE, b, dinv, a1, a2, res, d, x, dsrc,
                                                 wd, outer->scal_d, outer->partials,
                                                 outer->counter);
  }
  void pass(int mode, bool dots, TM a1, TM a2, int dsrc, int wd, gf_problem *outer,
            cudaStream_t st) override {
    outer->launches++;
    if (mode == MG_RESID) run_pass<MG_RESID, false>(a1, a2, dsrc, wd, outer, st);
    else if (mode == MG_START) run_pass<MG_START, false>(a1, a2, dsrc, wd, outer, st);
    else if (mode == MG_FOLDB) run_pass<MG_FOLDB, false>(a1, a2, dsrc, wd, outer, st);
    else if (dots) run_pass<MG_STEP, true>(a1, a2, dsrc, wd, outer, st);
    else run_pass<MG_STEP, false>(a1, a2, dsrc, wd, outer, st);
  }
  void restrict_elem(B &C, gf_problem *outer, cudaStream_t st) override {
    constexpr int NT = N * N, EPB = (256 / NT) < 1 ? 1 : 256 / NT;
    const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
    outer->launches++;
    k_pxfer_restrict<N, TM><<<grid, dim3(NT, EPB), 0, st>>>(prob->box, X[0], res, C.qE,
                                                            outer->scal_d + S_DONE);
  }
  void prolong_elem(const B &C, gf_problem *outer, cudaStream_t st) override {
    constexpr int NT = N * N, EPB = (256 / NT) < 1 ? 1 : 256 / NT;
    const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
    outer->launches++;
    k_pxfer_prolong<N, TM><<<grid, dim3(NT, EPB), 0, st>>>(prob->box, C.prob->box, X[0], C.x, x,
                                                           outer->scal_d + S_DONE);
  }
  int jacobi(double p, double q, int use_mass) override {
    double *d64 = nullptr;
    float *d32 = nullptr;
    int rc = S.jacobi(p, q, use_mass, &d64, &d32);
    if (rc) return rc;
    dinv32 = d32;
    const void *src = std::is_same<TM, float>::value ? (const void *)d32 : (const void *)d64;
    return cudaMemcpyAsync(dinv, src, sizeof(TM) * nL, cudaMemcpyDeviceToDevice, S.st) ==
                   cudaSuccess
               ? GF_OK
               : GF_ERR_CUDA;
  }
  // Largest eigenvalue of Dinv A: Lanczos Ritz value from min(12, nfree)
  // FP32 PCG steps on a pseudo-random right-hand side (whatever the
  // multigrid's type: the estimate only places the smoothing interval).
  // Runs on the level problem's own scalar block and work slots (set-up
  // only), right after jacobi().
  int estimate(double p, double q, int use_mass, int64_t nfree) override {
    const int K = (int)std::min<int64_t>(12, std::max<int64_t>(nfree, 1));
    gf_cg_traits tr{};
    tr.maxit = K;
    tr.normtype = GF_NORM_INF;
    tr.tol = 1e-300;
    tr.check_every = K;
    tr.precision = GF_CG_FP64;
    S.set_scalars(tr, K, false);
    gf_problem *lp = prob;
    cudaMemcpyAsync(lp->scal_d, lp->scal_h, sizeof(double) * S_COUNT, cudaMemcpyHostToDevice, S.st);
    double *bL = (double *)gf_work(lp, 0, sizeof(double) * nL);
    double *xL = (double *)gf_work(lp, 1, sizeof(double) * nL);
    double *rL = (double *)gf_work(lp, 2, sizeof(double) * nL);
    double *qE64 = (double *)gf_work(lp, 3, sizeof(double) * nE);
    float *r32 = (float *)gf_work(lp, 11, sizeof(float) * nL);
    float *w32 = (float *)gf_work(lp, 12, sizeof(float) * nL);
    float *x32 = (float *)gf_work(lp, 13, sizeof(float) * nL);
    float *q32 = (float *)gf_work(lp, 14, sizeof(float) * nL);
    float *qE32 = (float *)gf_work(lp, 15, sizeof(float) * nE);
    double *abd = (double *)gf_work(lp, 17, sizeof(double) * 2 * K);
    if (!bL || !xL || !rL || !qE64 || !r32 || !w32 || !x32 || !q32 || !qE32 || !abd)
      return GF_ERR_NOMEM;
    k_fill_hash<<<S.gL, 256, 0, S.st>>>(nL, S.wt.maskL, bL);
    cudaMemsetAsync(xL, 0, sizeof(double) * nL, S.st);
    cudaMemsetAsync(x32, 0, sizeof(float) * nL, S.st);
    if (!dinv32) return GF_ERR_ARG;
    int rc =
        S.template residual<float>(p, q, use_mass, bL, xL, qE64, rL, r32, w32, dinv32, 0, 1e-300);
    if (rc) return rc;
    int its = 0;
    S.ab = abd;
    S.nab = K;
    rc = S.template iterate<float>(tr, K, p, q, use_mass, x32, r32, w32, q32, qE32, dinv32,
                                   nullptr, &its);
    S.ab = nullptr;
    S.nab = 0;
    if (rc) return rc;
    std::vector<double> ab(2 * (size_t)std::max(its, 1));
    if (its > 0 && cudaMemcpy(ab.data(), abd, sizeof(double) * 2 * its, cudaMemcpyDeviceToHost) !=
                       cudaSuccess)
      return GF_ERR_CUDA;
    lmax = its > 0 ? lanczos_max(ab.data(), its) : 0.0;
    return lmax > 0.0 ? GF_OK : GF_ERR_NONFINITE;
  }
};

template <int N>
struct MakeLevel {
  template <typename TM>
  static int run(gf_problem *lp, bool own, bool masked, MGLevelBase<TM> **out) {
    *out = new MGLevel<N, TM>(lp, own, masked);
    return GF_OK;
  }
};

constexpr int MG_NKEY = 7;  // p, q, use_mass, masked, degree, ratio, type

template <typename TM>
struct MGHier {
  std::vector<MGLevelBase<TM> *> lv;
  double key[MG_NKEY] = {0, 0, 0, 0, 0, 0, 0};
  // CUDA graph of the whole iteration loop: a WHILE conditional node whose
  // body is one CG iteration followed by k_while_more (captured on the
  // first solve with these vectors, replayed by later solves)
  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // buffers the recorded loop reads, and the FP32 apply variant it launches
  const void *gkey[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  uint64_t glaunches = 0;  // launches per iteration
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~MGHier() {
    drop_graph();
    if (cs) cudaStreamDestroy(cs);
    for (auto *l : lv) delete l;
  }
};

// the problem's hierarchy is an MGHier<TM> exactly when its mg_free is mg_free<TM>
template <typename TM>
void mg_free(void *h) {
  delete (MGHier<TM> *)h;
}

// A coarser level as a light problem: what the affine K1 apply, the
// Jacobi diagonal and the lattice assembly read.
int mg_light_problem(gf_context *ctx, int dim, const int (&ne)[3], const int (&per)[3], int p,
                     const std::vector<double> &eg, bool masked, gf_problem **out) {
  const int n = p + 1;
  gf_problem *lp = new gf_problem();
  lp->ctx = ctx;
  ctx->nprob++;
  lp->dim = dim;
  lp->n = n;
  lp->geom = GF_GEOM_AFFINE;
  lp->volume = 1.0;
  int64_t nel = 1, nn = 1;
  for (int k = 0; k < dim; k++) {
    nel *= ne[k];
    nn *= n;
  }
  lp->ne = nel;
  lp->nlocal = nel * nn;
  std::vector<double> xi(n);
  gf_gll_basis(p, xi.data(), lp->W, lp->D);
  gfk::gf_k1_matrix(n, lp->D, lp->W, lp->K1);
  BoxLattice L{};
  L.dim = dim;
  L.p = p;
  for (int k = 0; k < 3; k++) {
    L.ne[k] = k < dim ? ne[k] : 1;
    L.per[k] = k < dim ? per[k] : 0;
    L.M[k] = k < dim ? (int64_t)L.ne[k] * p + (L.per[k] ? 0 : 1) : 1;
  }
  lp->box = L;
  lp->has_box = true;
  lp->nclass = L.size();
  auto up = [](const void *h, size_t bytes) -> void * {
    void *d = nullptr;
    if (cudaMalloc(&d, std::max<size_t>(bytes, 1)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
    return d;
  };
  std::vector<float> egf(eg.begin(), eg.end());
  lp->egeom_d = (double *)up(eg.data(), sizeof(double) * eg.size());
  lp->egeom_f = (float *)up(egf.data(), sizeof(float) * egf.size());
  if (masked) {  // Dirichlet on the non-periodic box faces
    std::vector<uint8_t> mk((size_t)lp->nclass, 1);
    for (int64_t c = 0; c < lp->nclass; c++) {
      int64_t r = c;
      for (int k = 0; k < dim; k++) {
        const int64_t g = r % L.M[k];
        r /= L.M[k];
        if (!L.per[k] && (g == 0 || g == L.M[k] - 1)) mk[c] = 0;
      }
    }
    lp->maskL8 = (uint8_t *)up(mk.data(), mk.size());
  }
  lp->npartials = 2048;
  cudaMalloc(&lp->partials, sizeof(double) * 4 * lp->npartials);
  cudaMalloc(&lp->counter, sizeof(unsigned int) * 8);
  cudaMemset(lp->counter, 0, sizeof(unsigned int) * 8);
  cudaMalloc(&lp->scal_d, sizeof(double) * 64);
  cudaMemset(lp->scal_d, 0, sizeof(double) * 64);
  cudaMallocHost(&lp->scal_h, sizeof(double) * 64);
  if (!lp->egeom_d || !lp->egeom_f || (masked && !lp->maskL8) || !lp->partials || !lp->counter ||
      !lp->scal_d || !lp->scal_h) {
    gf_problem_destroy(lp);
    return GF_ERR_NOMEM;
  }
  *out = lp;
  return GF_OK;
}

// 1-d transfer from (nec elements, order pc) to (nef, pf), nef a multiple
// of nec: the fine point at offset r in a coarse element takes the coarse
// element's GLL Lagrange interpolant at its position (element-local
// coordinates; the fine GLL nodes of uniform children).
template <typename TM>
Xfer1D<TM> build_xfer(int nef, int pf, int nec, int pc, bool per) {
  Xfer1D<TM> T{};
  const int ratio = nef / nec;
  T.R = ratio * pf;
  T.pc = pc;
  T.nec = nec;
  T.per = per ? 1 : 0;
  T.Mf = nef * pf + (per ? 0 : 1);
  T.Mc = nec * pc + (per ? 0 : 1);
  std::vector<double> xf(pf + 1), xc(pc + 1);
  gf_gll_basis(pf, xf.data(), nullptr, nullptr);
  gf_gll_basis(pc, xc.data(), nullptr, nullptr);
  for (int r = 0; r <= T.R; r++) {
    const int cf = std::min(r / pf, ratio - 1), i = r - cf * pf;
    const double xi = 2.0 * (cf + 0.5 * (xf[i] + 1.0)) / ratio - 1.0;
    for (int a = 0; a <= pc; a++) {
      double w = 1.0;
      for (int bb = 0; bb <= pc; bb++)
        if (bb != a) w *= (xi - xc[bb]) / (xc[a] - xc[bb]);
      if (std::fabs(w) < 1e-13) w = 0.0;
      T.J[r * (pc + 1) + a] = (TM)w;
    }
  }
  return T;
}

// The fine mask must be the box-face Dirichlet mask for the coarse levels'
// masks to be its restriction: count the lattice points where it differs.
__global__ void k_boxmask_mismatch(int64_t nL, BoxLattice L, const uint8_t *__restrict__ mask,
                                   unsigned int *count) {
  GRID_STRIDE(c, nL) {
    int64_t r = c;
    uint8_t want = 1;
    for (int k = 0; k < L.dim; k++) {
      const int64_t g = r % L.M[k];
      r /= L.M[k];
      if (!L.per[k] && (g == 0 || g == L.M[k] - 1)) want = 0;
    }
    if ((mask[c] != 0) != (want != 0)) atomicAdd(count, 1u);
  }
}

// The assembled operator of an affine box level on its free lattice points,
// inverted in FP64: element matrices
//   A_e(a, b) = p sum_d X_d^2 J K1(a_d, b_d) prod_{k != d} W(a_k) delta(a_k, b_k)
//             + q J prod_k W(a_k) delta(a, b)       (K1 = D^T W D, lumped mass)
// summed into the lattice, Cholesky-factored and inverted.  Returns false
// when the matrix is not positive definite (the level then keeps its
// Chebyshev solve).
template <typename TM>
bool mg_dense_inverse(const gf_problem *lp, const std::vector<double> &eg, double p, double q,
                      int use_mass, const uint8_t *maskL_host, std::vector<TM> &ainv,
                      std::vector<int32_t> &free_idx) {
  const BoxLattice &L = lp->box;
  const int dim = lp->dim, n = lp->n;
  const int64_t nL = lp->nclass;
  std::vector<int64_t> pos(nL, -1);
  free_idx.clear();
  for (int64_t c = 0; c < nL; c++)
    if (!maskL_host || maskL_host[c]) {
      pos[c] = (int64_t)free_idx.size();
      free_idx.push_back((int32_t)c);
    }
  const int64_t nf = (int64_t)free_idx.size();
  if (nf == 0) return false;
  std::vector<double> A((size_t)nf * nf, 0.0);
  const int nn = dim == 3 ? n * n * n : n * n;
  std::vector<int64_t> gidx(nn);
  for (int64_t e = 0; e < lp->ne; e++) {
    int ec[3];
    L.elem_coords(e, ec);
    for (int a = 0; a < nn; a++) {
      const int la[3] = {a % n, (a / n) % n, dim == 3 ? a / (n * n) : 0};
      int64_t g = L.g1(0, ec[0], la[0]) + L.M[0] * L.g1(1, ec[1], la[1]);
      if (dim == 3) g += L.M[0] * L.M[1] * L.g1(2, ec[2], la[2]);
      gidx[a] = g;
    }
    const double *geo = &eg[(size_t)e * (dim + 1)];
    const double J = geo[dim];
    for (int a = 0; a < nn; a++) {
      const int64_t ia = pos[gidx[a]];
      if (ia < 0) continue;
      const int la[3] = {a % n, (a / n) % n, dim == 3 ? a / (n * n) : 0};
      for (int b = 0; b < nn; b++) {
        const int64_t ib = pos[gidx[b]];
        if (ib < 0) continue;
        const int lb[3] = {b % n, (b / n) % n, dim == 3 ? b / (n * n) : 0};
        double v = 0.0;
        for (int d = 0; d < dim; d++) {
          bool same = true;
          double w = 1.0;
          for (int k = 0; k < dim; k++)
            if (k != d) {
              if (la[k] != lb[k]) same = false;
              w *= lp->W[la[k]];
            }
          if (same) v += geo[d] * geo[d] * J * lp->K1[la[d] + lb[d] * n] * w;
        }
        v *= p;
        if (use_mass && a == b) {
          double w = J;
          for (int k = 0; k < dim; k++) w *= lp->W[la[k]];
          v += q * w;
        }
        A[(size_t)ia * nf + ib] += v;
      }
    }
  }
  // Cholesky A = L L^T (lower, in place)
  for (int64_t j = 0; j < nf; j++) {
    double dj = A[(size_t)j * nf + j];
    for (int64_t k = 0; k < j; k++) dj -= A[(size_t)j * nf + k] * A[(size_t)j * nf + k];
    if (!(dj > 0.0)) return false;
    dj = std::sqrt(dj);
    A[(size_t)j * nf + j] = dj;
    for (int64_t i = j + 1; i < nf; i++) {
      double v = A[(size_t)i * nf + j];
      for (int64_t k = 0; k < j; k++) v -= A[(size_t)i * nf + k] * A[(size_t)j * nf + k];
      A[(size_t)i * nf + j] = v / dj;
    }
  }
  // inverse column by column: L y = e_c, L^T z = y
  ainv.assign((size_t)nf * nf, TM(0));
  std::vector<double> y(nf);
  for (int64_t c = 0; c < nf; c++) {
    for (int64_t i = 0; i < nf; i++) {
      double v = i == c ? 1.0 : 0.0;
      for (int64_t k = c; k < i; k++) v -= A[(size_t)i * nf + k] * y[k];
      y[i] = i < c ? 0.0 : v / A[(size_t)i * nf + i];
    }
    for (int64_t i = nf - 1; i >= 0; i--) {
      double v = y[i];
      for (int64_t k = i + 1; k < nf; k++) v -= A[(size_t)k * nf + i] * y[k];
      y[i] = v / A[(size_t)i * nf + i];
    }
    for (int64_t i = 0; i < nf; i++) ainv[(size_t)i * nf + c] = (TM)y[i];
  }
  return true;
}

template <typename TM>
void mg_coefficients(MGLevelBase<TM> &L, int m, double ratio) {
  const double bb = 1.1 * L.lmax, a = bb / ratio;
  const double theta = 0.5 * (bb + a), delta = 0.5 * (bb - a), sigma = theta / delta;
  L.m = m;
  L.c0 = (TM)(1.0 / theta);
  L.c1.assign(m + 1, TM(0));
  L.c2.assign(m + 1, TM(0));
  double rho = 1.0 / sigma;
  for (int j = 1; j <= m; j++) {
    const double rn1 = 1.0 / (2.0 * sigma - rho);
    L.c1[j] = (TM)(rn1 * rho);
    L.c2[j] = (TM)(2.0 * rn1 / delta);
    rho = rn1;
  }
}

template <class MAP>
struct IsBox : std::false_type {};
template <int N>
struct IsBox<MapBox<N>> : std::true_type {};

template <class MAP, typename TM>
int mg_prepare_t(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass) {
  gf_problem *prob = S.prob;
  gf_context *ctx = S.ctx;
  if constexpr (!IsBox<MAP>::value) {
    return gf_fail(ctx, GF_ERR_UNSUPPORTED, "PMG needs a structured box (box_ne)");
  } else {
    GF_REQUIRE(ctx, prob->geom == GF_GEOM_AFFINE && prob->egeom_d,
               "PMG needs affine elements (GF_GEOM_AFFINE)");
    const bool masked = S.wt.maskL != nullptr;
    const int m = std::max(0, tr.poly_degree);
    const double ratio = tr.poly_ratio > 1.0 ? tr.poly_ratio : 8.0;
    const double key[MG_NKEY] = {p,          q,     (double)use_mass, masked ? 1.0 : 0.0,
                                 (double)m, ratio, (double)sizeof(TM)};
    if (prob->mg) {
      if (prob->mg_free == mg_free<TM>) {
        MGHier<TM> *H = (MGHier<TM> *)prob->mg;
        if (std::equal(key, key + MG_NKEY, H->key)) return GF_OK;
      }
      prob->mg_free(prob->mg);
      prob->mg = nullptr;
    }
    const int dim = prob->dim;
    const BoxLattice &B = prob->box;
    cudaStream_t st = S.st;
    if (masked) {
      unsigned int *cnt = (unsigned int *)gf_work(prob, 18, sizeof(unsigned int));
      if (!cnt) return gf_fail(ctx, GF_ERR_NOMEM, "PMG set-up allocation failed");
      unsigned int h = 0;
      GF_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(unsigned int), st));
      k_boxmask_mismatch<<<S.gL, 256, 0, st>>>(S.nL, B, prob->maskL8, cnt);
      GF_CUDA(ctx, cudaMemcpyAsync(&h, cnt, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
      GF_CUDA(ctx, cudaStreamSynchronize(st));
      GF_REQUIRE(ctx, h == 0, "PMG needs the box-face Dirichlet mask (%u points differ)", h);
    }
    std::vector<double> eg((size_t)prob->ne * (dim + 1));
    GF_CUDA(ctx, cudaMemcpy(eg.data(), prob->egeom_d, sizeof(double) * eg.size(),
                            cudaMemcpyDeviceToHost));
    // level descriptions: order, element counts, element geometry
    struct Desc {
      int p, ne[3];
      std::vector<double> eg;
    };
    std::vector<Desc> ds;
    Desc d0;
    d0.p = prob->n - 1;
    for (int k = 0; k < 3; k++) d0.ne[k] = B.ne[k];
    d0.eg = eg;
    ds.push_back(d0);
    while (ds.back().p > 1) {  // p -> ceil(p/2): 7, 4, 2, 1
      Desc d = ds.back();
      d.p = (d.p + 1) / 2;
      ds.push_back(d);
    }
    // free lattice points of a level (the dense coarsest solve's size)
    auto nfree_of = [&](const Desc &d) {
      int64_t nf = 1;
      for (int k = 0; k < dim; k++) {
        const int64_t Mk = (int64_t)d.ne[k] * d.p + (B.per[k] ? 0 : 1);
        nf *= (masked && !B.per[k]) ? Mk - 2 : Mk;
      }
      return nf;
    };
    for (;;) {
      const Desc &f = ds.back();
      bool ok = nfree_of(f) > MG_DENSE_SMALL;
      for (int k = 0; k < dim; k++) ok = ok && f.ne[k] % 2 == 0 && f.ne[k] / 2 >= 2;
      if (!ok) break;
      Desc c;
      c.p = 1;
      for (int k = 0; k < 3; k++) c.ne[k] = k < dim ? f.ne[k] / 2 : 1;
      const int64_t nec = (int64_t)c.ne[0] * c.ne[1] * c.ne[2];
      c.eg.assign((size_t)nec * (dim + 1), 0.0);
      for (int64_t e = 0; e < nec; e++) {
        const int ec[3] = {(int)(e % c.ne[0]), (int)((e / c.ne[0]) % c.ne[1]),
                           (int)(e / ((int64_t)c.ne[0] * c.ne[1]))};
        double jac = 1.0;
        for (int k = 0; k < dim; k++) {
          // width along k: the two children along k (at the first child
          // position in the other directions), width = 2 / dXi/dX
          double w = 0.0;
          for (int s = 0; s < 2; s++) {
            int fc[3] = {2 * ec[0], 2 * ec[1], 2 * ec[2]};
            fc[k] += s;
            const int64_t fe = fc[0] + (int64_t)f.ne[0] * (fc[1] + (int64_t)f.ne[1] * fc[2]);
            w += 2.0 / f.eg[(size_t)fe * (dim + 1) + k];
          }
          c.eg[(size_t)e * (dim + 1) + k] = 2.0 / w;
          jac *= 0.5 * w;
        }
        c.eg[(size_t)e * (dim + 1) + dim] = jac;
      }
      ds.push_back(c);
    }
    MGHier<TM> *H = new MGHier<TM>();
    std::copy(key, key + MG_NKEY, H->key);
    auto fail = [&](int rc, const char *what) {
      delete H;
      return gf_fail(ctx, rc, "PMG set-up: %s", what);
    };
    for (size_t l = 0; l < ds.size(); l++) {
      gf_problem *lp = prob;
      if (l > 0) {
        const int per[3] = {B.per[0], B.per[1], B.per[2]};
        int rc = mg_light_problem(ctx, dim, ds[l].ne, per, ds[l].p, ds[l].eg, masked, &lp);
        if (rc) return fail(rc, "level allocation failed");
      }
      MGLevelBase<TM> *L = nullptr;
      int rc = dispatch_n<MakeLevel>(ds[l].p + 1, lp, l > 0, masked, &L);
      if (rc || !L) {
        if (l > 0) gf_problem_destroy(lp);
        return fail(GF_ERR_UNSUPPORTED, "order out of range");
      }
      H->lv.push_back(L);
      L->dinv = L->alloc_f(L->nL);
      L->b = L->alloc_f(L->nL);
      L->x = L->alloc_f(L->nL);
      L->res = L->alloc_f(L->nL);
      L->d = L->alloc_f(L->nL);
      L->qE = L->alloc_f(L->nE);
      if (!L->dinv || !L->b || !L->x || !L->res || !L->d || !L->qE)
        return fail(GF_ERR_NOMEM, "vector allocation failed");
      const bool coarsest = l + 1 == ds.size();
      const int64_t nfree = nfree_of(ds[l]);
      bool dense = false;
      if (coarsest && l > 0 && nfree <= MG_DENSE_MAX) {
        // exact coarsest solve: the dense inverse of the assembled operator
        std::vector<uint8_t> mk;
        if (masked) {
          mk.assign((size_t)L->nL, 0);
          if (cudaMemcpy(mk.data(), L->maskL, L->nL, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(GF_ERR_CUDA, "mask copy failed");
        }
        std::vector<TM> ai;
        std::vector<int32_t> fi;
        if (mg_dense_inverse(lp, ds[l].eg, p, q, use_mass, masked ? mk.data() : nullptr, ai, fi)) {
          L->ainv = L->upload(ai);
          L->free_idx = L->upload(fi);
          L->nfree = (int64_t)fi.size();
          if (!L->ainv || !L->free_idx) return fail(GF_ERR_NOMEM, "coarse inverse allocation failed");
          if (cudaMemset(L->x, 0, sizeof(TM) * L->nL) != cudaSuccess)
            return fail(GF_ERR_CUDA, "coarse vector clear failed");
          dense = true;
        }
      }
      if (!dense) {
        if ((rc = L->jacobi(p, q, use_mass))) return fail(rc, "Jacobi diagonal failed");
        if ((rc = L->estimate(p, q, use_mass, nfree)))
          return fail(rc, "eigenvalue estimate failed");
        int mc = 0;
        for (int k = 0; k < dim; k++) mc = std::max(mc, L->M[k]);
        if (coarsest) mg_coefficients(*L, std::min(64, std::max(4, 2 * mc)), 30.0);
        else mg_coefficients(*L, m, ratio);
      }
      if (l > 0) {  // transfer between levels l-1 (fine) and l
        MGLevelBase<TM> *F = H->lv[l - 1];
        for (int k = 0; k < dim; k++)
          F->X[k] = build_xfer<TM>(ds[l - 1].ne[k], ds[l - 1].p, ds[l].ne[k], ds[l].p,
                                   B.per[k] != 0);
        // same elements, coarse order as the element kernels assume
        F->ptransfer = dim == 3 && ds[l - 1].ne[0] == ds[l].ne[0] &&
                       ds[l - 1].ne[1] == ds[l].ne[1] && ds[l - 1].ne[2] == ds[l].ne[2] &&
                       ds[l].p + 1 == (ds[l - 1].p + 1) / 2 + 1;
        // sweep intermediates: restriction (c, f, f), (c, c, f); prolongation
        // (f, c, c), (f, f, c)
        const int64_t f0 = F->M[0], f1 = F->M[1], f2 = F->M[2];
        const int64_t c0 = L->M[0], c1 = L->M[1], c2 = L->M[2];
        F->t1 = F->alloc_f(std::max(c0 * f1 * f2, f0 * c1 * c2));
        F->t2 = F->alloc_f(std::max(c0 * c1 * f2, f0 * f1 * c2));
        if (!F->t1 || !F->t2) return fail(GF_ERR_NOMEM, "transfer allocation failed");
      }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(GF_ERR_CUDA, "set-up failed");
    for (size_t l = 1; l < H->lv.size(); l++) H->lv[l]->prob->launches = 0;
    prob->mg = H;
    prob->mg_free = mg_free<TM>;
    return GF_OK;
  }
}

// restriction lv[l].res -> lv[l+1].b (coarse mask), prolongation
// lv[l].x += P lv[l+1].x; one k_xfer1d sweep per direction
template <typename TM>
void mg_restrict(MGLevelBase<TM> &F, MGLevelBase<TM> &C, gf_problem *outer, cudaStream_t st) {
  const double *stop = outer->scal_d + S_DONE;
  const int dim = F.dim;
  int e[3] = {F.M[0], F.M[1], F.M[2]};
  const TM *in = F.res;
  for (int k = 0; k < dim; k++) {
    int eo[3] = {e[0], e[1], e[2]};
    eo[k] = C.M[k];
    const bool last = k == dim - 1;
    TM *out = last ? C.b : (k == 0 ? F.t1 : F.t2);
    const int64_t nout = (int64_t)eo[0] * eo[1] * eo[2];
    k_xfer1d<TM><<<grid_for(nout, 256, 148 * 16), 256, 0, st>>>(
        nout, k, eo[0], eo[1], e[0], e[1], F.X[k], 1, in, out, last ? C.maskL : nullptr,
        last ? 2 : 0, stop);
    outer->launches++;
    in = out;
    e[k] = C.M[k];
  }
}

template <typename TM>
void mg_prolong(MGLevelBase<TM> &F, MGLevelBase<TM> &C, gf_problem *outer, cudaStream_t st) {
  const double *stop = outer->scal_d + S_DONE;
  const int dim = F.dim;
  int e[3] = {C.M[0], C.M[1], C.M[2]};
  const TM *in = C.x;
  for (int k = 0; k < dim; k++) {
    int eo[3] = {e[0], e[1], e[2]};
    eo[k] = F.M[k];
    const bool last = k == dim - 1;
    TM *out = last ? F.x : (k == 0 ? F.t1 : F.t2);
    const int64_t nout = (int64_t)eo[0] * eo[1] * eo[2];
    k_xfer1d<TM><<<grid_for(nout, 256, 148 * 16), 256, 0, st>>>(nout, k, eo[0], eo[1], e[0],
                                                                e[1], F.X[k], 0, in, out, nullptr,
                                                                last ? 1 : 0, stop);
    outer->launches++;
    in = out;
    e[k] = F.M[k];
  }
}

// One V-cycle from level l: lv[l].x ~= A_l^-1 lv[l].b.  At l = 0 the input
// is the FP64 outer residual r64 and the last pass reduces <r, z> for the
// CG step.
template <typename TM>
void mg_vcycle(MGHier<TM> &H, size_t l, double p, double q, int use_mass, gf_problem *outer,
               const double *r64, bool started, cudaStream_t st) {
  MGLevelBase<TM> &L = *H.lv[l];
  const double *stop = outer->scal_d + S_DONE;
  const bool top = l == 0, last = l + 1 == H.lv.size();
  const TM zero = 0;
  // b arrives as the element restriction's coarse E-vector in L.qE
  const bool folded = l > 0 && H.lv[l - 1]->ptransfer;
  if (last && L.ainv) {  // coarsest: dense solve (never the finest level)
    if (folded) L.pass(MG_FOLDB, false, zero, zero, DP_NONE, 0, outer, st);
    k_dense_solve<TM><<<(unsigned)std::min<int64_t>(L.nfree, 148 * 8), 128, 0, st>>>(
        L.nfree, L.ainv, L.free_idx, L.b, L.x, stop);
    outer->launches++;
    return;
  }
  // x = c0 Dinv b (the top level's b and x may come from the outer update)
  if (folded) {
    L.pass(MG_START, false, L.c0, zero, DP_NONE, 0, outer, st);
  } else if (!(top && started)) {
    k_mg_start<TM><<<grid_for(L.nL, 256, 148 * 16), 256, 0, st>>>(L.nL, top ? r64 : nullptr, L.b,
                                                                   L.dinv, L.c0, L.x, stop);
    outer->launches++;
  }
  // pre-smoothing x = S b (on the coarsest level: the whole Chebyshev solve)
  for (int j = 1; j <= L.m; j++) {
    L.apply(L.x, p, q, use_mass, stop, st);
    L.pass(MG_STEP, last && top && j == L.m, L.c1[j], L.c2[j], j == 1 ? DP_X : DP_D, j < L.m,
           outer, st);
  }
  if (last) return;
  L.apply(L.x, p, q, use_mass, stop, st);  // res = b - A x
  L.pass(MG_RESID, false, zero, zero, DP_NONE, 0, outer, st);
  if (L.ptransfer) L.restrict_elem(*H.lv[l + 1], outer, st);
  else mg_restrict(L, *H.lv[l + 1], outer, st);
  mg_vcycle(H, l + 1, p, q, use_mass, outer, r64, false, st);
  if (L.ptransfer) L.prolong_elem(*H.lv[l + 1], outer, st);
  else mg_prolong(L, *H.lv[l + 1], outer, st);
  // post-smoothing x += S (b - A x): the first term from the residual
  L.apply(L.x, p, q, use_mass, stop, st);
  L.pass(MG_STEP, top && L.m == 0, zero, L.c0, DP_NONE, L.m > 0, outer, st);
  for (int j = 1; j <= L.m; j++) {
    L.apply(L.x, p, q, use_mass, stop, st);
    L.pass(MG_STEP, top && j == L.m, L.c1[j], L.c2[j], DP_D, j < L.m, outer, st);
  }
}

// FP64 CG (Fletcher-Reeves beta, fcg_finish_fr) with one V-cycle in TM
// (FP32 or FP64) as the preconditioner; per iteration the FP64 apply,
// assembly with <w,q>, the x/r update with the stop test, the V-cycle and
// w = z + beta w.
template <class MAP, typename TM>
int solve_mg_t(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass,
               const double *bL, double *xL, double *rL, double *qE, double *hist, int *total,
               double *rn) {
  gf_problem *prob = S.prob;
  gf_context *ctx = S.ctx;
  if (!prob->mg || prob->mg_free != mg_free<TM>)
    return gf_fail(ctx, GF_ERR_ARG, "PMG hierarchy missing");
  MGHier<TM> *H = (MGHier<TM> *)prob->mg;
  cudaStream_t st = S.st;
  const int64_t nL = S.nL;
  double *w = (double *)gf_work(prob, 4, sizeof(double) * nL);
  double *qL = (double *)gf_work(prob, 5, sizeof(double) * nL);
  if (!w || !qL) return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
  GF_CUDA(ctx, cudaMemsetAsync(qL, 0, sizeof(double) * nL, st));
  int rc = S.template residual<double>(p, q, use_mass, bL, xL, qE, rL, rL, w, nullptr, 0, tr.tol);
  if (rc) return gf_fail(ctx, rc, "residual failed");
  const TM *z = H->lv[0]->x;
  double *scal = prob->scal_d;
  MGLevelBase<TM> &L0 = *H->lv[0];
  auto precondition = [&](cudaStream_t ls, bool started) {
    mg_vcycle(*H, 0, p, q, use_mass, prob, rL, started, ls);
    prob->launches++;
    k_fcg_w<TM><<<S.gL, 256, 0, ls>>>(nL, w, z, scal);
  };
  auto iterations = [&](int k, cudaStream_t ls) {
    for (int i = 0; i < k; i++) {
      launch_helm_L<double>(prob, p, q, use_mass, w, qE, ls, scal + S_DONE);
      k_asm_dot<double, MAP><<<S.rgrid(k_asm_dot<double, MAP>), RED_THREADS, 0, ls>>>(
          nL, S.map, S.wt, qE, w, qL, scal, prob->partials, prob->counter);
      k_update_mg<TM><<<S.rgrid(k_update_mg<TM>), RED_THREADS, 0, ls>>>(
          nL, S.wt, xL, w, rL, qL, L0.dinv, L0.c0, L0.b, L0.x, hist, scal, prob->partials,
          prob->counter);
      prob->launches += 2;
      precondition(ls, true);
    }
  };
  auto level_launches = [&]() {
    uint64_t n = prob->launches;
    for (size_t l = 1; l < H->lv.size(); l++) n += H->lv[l]->prob->launches;
    return n;
  };
  prob->scal_h[S_FIRST] = 1.0;
  GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_d + S_FIRST, prob->scal_h + S_FIRST, sizeof(double),
                               cudaMemcpyHostToDevice, st));
  precondition(st, false);
  // The iteration loop runs on the device: a graph holding one WHILE node
  // whose body is one iteration (some 95 launches, most of them small
  // coarse-level kernels, all reading their scalars from the device) and
  // k_while_more, which ends the loop once `done` is set (convergence,
  // maxit or breakdown) -- no host round trip per iteration and no
  // iterations queued past convergence.
  const void *gk[8] = {xL, rL, w, qL, qE, bL, hist, (const void *)(intptr_t)g_fp32_apply_mode};
  if (!(H->exec && std::equal(gk, gk + 8, H->gkey))) {
    H->drop_graph();
    if (!H->cs) GF_CUDA(ctx, cudaStreamCreateWithFlags(&H->cs, cudaStreamNonBlocking));
    const uint64_t n0 = level_launches();
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
      e = cudaStreamBeginCaptureToGraph(H->cs, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeRelaxed);
    }
    if (e == cudaSuccess) {
      iterations(1, H->cs);
      k_while_more<<<1, 1, 0, H->cs>>>(h, scal);
      e = cudaStreamEndCapture(H->cs, &body);
    }
    H->graph = g;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&H->exec, g, 0);
    H->glaunches = level_launches() - n0 + 1;
    for (size_t l = 1; l < H->lv.size(); l++) H->lv[l]->prob->launches = 0;
    prob->launches = n0;
    if (e != cudaSuccess) {
      H->drop_graph();
      return gf_fail(ctx, GF_ERR_CUDA, "CG loop capture failed: %s", cudaGetErrorString(e));
    }
    std::copy(gk, gk + 8, H->gkey);
  }
  GF_CUDA(ctx, cudaGraphLaunch(H->exec, st));
  GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h, scal, sizeof(double) * S_COUNT,
                               cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  *total = (int)prob->scal_h[S_ITER];
  prob->launches += H->glaunches * (uint64_t)std::max(1, *total);
  for (size_t l = 1; l < H->lv.size(); l++) {  // the levels' applies count as this problem's
    prob->launches += H->lv[l]->prob->launches;
    H->lv[l]->prob->launches = 0;
  }
  if (prob->scal_h[S_FLAG] != 0.0)
    return gf_fail(ctx, GF_ERR_NONFINITE, "CG breakdown: non-finite scalar at iteration %d",
                   *total);
  *rn = prob->scal_h[S_RNORM];
  return (*total >= tr.maxit && *rn > prob->scal_h[S_RTOL]) ? GF_CG_NOCONVERGE : GF_OK;
}

// GF_PRECOND_PMG: FP32 V-cycle; GF_PRECOND_PMG64: FP64 V-cycle
template <class MAP>
int mg_prepare(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass) {
  return tr.precond == GF_PRECOND_PMG64 ? mg_prepare_t<MAP, double>(S, tr, p, q, use_mass)
                                        : mg_prepare_t<MAP, float>(S, tr, p, q, use_mass);
}

template <class MAP>
int solve_mg(Solver<MAP> &S, const gf_cg_traits &tr, double p, double q, int use_mass,
             const double *bL, double *xL, double *rL, double *qE, double *hist, int *total,
             double *rn) {
  return tr.precond == GF_PRECOND_PMG64
             ? solve_mg_t<MAP, double>(S, tr, p, q, use_mass, bL, xL, rL, qE, hist, total, rn)
             : solve_mg_t<MAP, float>(S, tr, p, q, use_mass, bL, xL, rL, qE, hist, total, rn);
}

template <int N>
struct BoxSolve {
  static int run(gf_problem *prob, const gf_cg_traits *tr, double p, double q, int use_mass,
                 const double *b, const double *xb, double *x, int *it, double *rn, double *hist,
                 bool masked) {
    Solver<MapBox<N>> S(prob, MapBox<N>::make(prob->box), masked);
    return S.solve(*tr, p, q, use_mass, b, xb, x, it, rn, hist);
  }
};

// One kernel of the multigrid solve's finest level, launched alone (see
// gf_pmg_launch).
template <int N>
struct PMGLaunch {
  template <typename TM>
  static int level0(gf_problem *prob, Solver<MapBox<N>> &S, double p, double q, int use_mass,
                    int which) {
    gf_context *ctx = prob->ctx;
    MGHier<TM> *H = (MGHier<TM> *)prob->mg;
    MGLevelBase<TM> &L = *H->lv[0];
    cudaStream_t st = ctx->stream;
    double *stop = prob->scal_d + S_DONE;
    if (which == GF_PMG_PREPARE) {
      // finite values in every vector the launches read, and `done` clear
      TM *const vecs[4] = {L.b, L.x, L.d, L.res};
      for (TM *v : vecs) GF_CUDA(ctx, cudaMemsetAsync(v, 0x3c, sizeof(TM) * L.nL, st));
      GF_CUDA(ctx, cudaMemsetAsync(L.qE, 0x3c, sizeof(TM) * L.nE, st));
      if (H->lv.size() > 1)  // the next level's x, read by the prolongation
        GF_CUDA(ctx, cudaMemsetAsync(H->lv[1]->x, 0x3c, sizeof(TM) * H->lv[1]->nL, st));
      double *xL = (double *)gf_work(prob, 1, sizeof(double) * S.nL);
      double *qE = (double *)gf_work(prob, 3, sizeof(double) * S.nE);
      if (!xL || !qE) return gf_fail(ctx, GF_ERR_NOMEM, "work allocation failed");
      GF_CUDA(ctx, cudaMemsetAsync(xL, 0x3c, sizeof(double) * S.nL, st));
      GF_CUDA(ctx, cudaMemsetAsync(stop, 0, sizeof(double), st));
      GF_CUDA(ctx, cudaStreamSynchronize(st));
      return GF_OK;
    }
    int rc = GF_OK;
    if (which == GF_PMG_APPLY64) {
      double *xL = (double *)gf_work(prob, 1, sizeof(double) * S.nL);
      double *qE = (double *)gf_work(prob, 3, sizeof(double) * S.nE);
      if (!xL || !qE) return gf_fail(ctx, GF_ERR_NOMEM, "work allocation failed");
      rc = launch_helm_L<double>(prob, p, q, use_mass, xL, qE, st, stop);
    } else if (which == GF_PMG_APPLY) {
      rc = L.apply(L.x, p, q, use_mass, stop, st);
    } else if (which == GF_PMG_STEP) {
      L.pass(MG_STEP, false, L.c1.size() > 1 ? L.c1[1] : TM(0), L.c0, DP_D, 1, prob, st);
    } else if (which == GF_PMG_RESID) {
      L.pass(MG_RESID, false, TM(0), TM(0), DP_NONE, 0, prob, st);
    } else {  // transfers between the finest level and the next
      if (H->lv.size() < 2) return gf_fail(ctx, GF_ERR_ARG, "the hierarchy has one level");
      MGLevelBase<TM> &C = *H->lv[1];
      if (which == GF_PMG_RESTRICT) {
        if (L.ptransfer) L.restrict_elem(C, prob, st);
        else mg_restrict(L, C, prob, st);
      } else {
        if (L.ptransfer) L.prolong_elem(C, prob, st);
        else mg_prolong(L, C, prob, st);
      }
    }
    if (rc) return gf_fail(ctx, rc, "launch failed");
    GF_CHECK_LAUNCH(ctx);
    return GF_OK;
  }
  static int run(gf_problem *prob, const gf_cg_traits *tr, double p, double q, int use_mass,
                 bool masked, int which) {
    Solver<MapBox<N>> S(prob, MapBox<N>::make(prob->box), masked);
    if (which == GF_PMG_PREPARE) {
      int rc = mg_prepare(S, *tr, p, q, use_mass);
      if (rc) return rc;
    } else if (!prob->mg) {
      return gf_fail(prob->ctx, GF_ERR_ARG, "no multigrid hierarchy: GF_PMG_PREPARE first");
    }
    return tr->precond == GF_PRECOND_PMG64 ? level0<double>(prob, S, p, q, use_mass, which)
                                           : level0<float>(prob, S, p, q, use_mass, which);
  }
};

}  // namespace

extern "C" int gf_pmg_launch(gf_problem_t prob, const gf_cg_traits *tr, double p, double q,
                             int use_mass, int masked, int which) {
  if (!prob || !tr) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, tr->precond == GF_PRECOND_PMG || tr->precond == GF_PRECOND_PMG64,
             "traits must name GF_PRECOND_PMG or GF_PRECOND_PMG64");
  GF_REQUIRE(ctx, which >= GF_PMG_PREPARE && which <= GF_PMG_PROLONG, "bad kernel selector");
  GF_REQUIRE(ctx, prob->has_box, "PMG needs a structured box (box_ne)");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  if (which != GF_PMG_PREPARE) {
    const bool ok = prob->mg && prob->mg_free == (tr->precond == GF_PRECOND_PMG64
                                                      ? mg_free<double>
                                                      : mg_free<float>);
    GF_REQUIRE(ctx, ok, "no multigrid hierarchy of this type: GF_PMG_PREPARE first");
  }
  return dispatch_n<PMGLaunch>(prob->n, prob, tr, p, q, use_mass, masked != 0, which);
}

extern "C" int gf_cg_solve(gf_problem_t prob, const gf_cg_traits *tr, double p, double q,
                           int use_mass, const double *b, const double *xb, double *x, int *iters,
                           double *final_norm, double *residuals) {
  if (!prob || !tr) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, b && x, "b and x are required");
  GF_REQUIRE(ctx, tr->maxit >= 0, "maxit must be >= 0");
  GF_REQUIRE(ctx, tr->normtype >= GF_NORM_INF && tr->normtype <= GF_NORM_L1, "bad norm type");
  GF_REQUIRE(ctx, tr->precision == GF_CG_FP64 || tr->precision == GF_CG_MIXED, "bad precision");
  GF_REQUIRE(ctx, tr->precond >= GF_PRECOND_NONE && tr->precond <= GF_PRECOND_PMG64,
             "bad preconditioner");
  GF_REQUIRE(ctx, tr->precond < GF_PRECOND_CHEBYSHEV || (tr->poly_degree >= 0 &&
                                                        tr->poly_degree <= 64),
             "poly_degree must be 0..64");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  double *hist = nullptr;
  if (residuals && tr->maxit > 0) {
    hist = (double *)gf_work(prob, 16, sizeof(double) * tr->maxit);
    if (!hist) return gf_fail(ctx, GF_ERR_NOMEM, "history allocation failed");
    cudaMemsetAsync(hist, 0, sizeof(double) * tr->maxit, ctx->stream);
  }
  int it = 0, rc;
  double rn = 0.0;
  const bool masked = xb != nullptr && prob->maskL8 != nullptr;
  if (prob->has_box) {
    rc = dispatch_n<BoxSolve>(prob->n, prob, tr, p, q, use_mass, b, xb, x, &it, &rn, hist, masked);
  } else {
    Solver<MapCsr> S(prob, MapCsr{prob->class_ptr, prob->members, prob->node_class, prob->nclass},
                     masked);
    rc = S.solve(*tr, p, q, use_mass, b, xb, x, &it, &rn, hist);
  }
  if (rc < 0) return rc;
  if (iters) *iters = it;
  if (final_norm) *final_norm = rn;
  // the history holds FP64 (outer) iterations: plain FP64 and the FP64
  // flexible CG of the polynomial and multigrid preconditioners
  if (residuals && hist && it > 0 &&
      (tr->precision == GF_CG_FP64 || tr->precond >= GF_PRECOND_CHEBYSHEV)) {
    GF_CUDA(ctx, cudaMemcpyAsync(residuals, hist, sizeof(double) * std::min(it, tr->maxit),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  }
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return rc;
}

extern "C" int gf_cg_solve_host(gf_problem_t prob, const gf_cg_traits *tr, double p, double q,
                                int use_mass, const double *b, const double *xb, double *x,
                                int *iters, double *final_norm) {
  if (!prob || !tr || !b || !x) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  const int64_t n = prob->nlocal;
  const size_t bytes = sizeof(double) * n;
  double *db = (double *)gf_work(prob, 20, bytes);
  double *dx = (double *)gf_work(prob, 21, bytes);
  double *dxb = xb ? (double *)gf_work(prob, 22, bytes) : nullptr;
  if (!db || !dx || (xb && !dxb)) return gf_fail(ctx, GF_ERR_NOMEM, "staging allocation failed");
  GF_CUDA(ctx, cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, ctx->stream));
  GF_CUDA(ctx, cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream));
  if (xb) GF_CUDA(ctx, cudaMemcpyAsync(dxb, xb, bytes, cudaMemcpyHostToDevice, ctx->stream));
  int rc = gf_cg_solve(prob, tr, p, q, use_mass, db, dxb, dx, iters, final_norm, nullptr);
  if (rc < 0) return rc;
  GF_CUDA(ctx, cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return rc;
}

// api_adjoint.cu -- adjoint (vector-Jacobian) path of the RK solver of
// api_rk.cu.  The reference has no adjoint; these entry points are new.
//
// Right-hand side (k_dudt*, api_rk.cu), per evolved component k:
//   F_k(u) = Minv ( -nu L u_k - M sum_j X_j c_j D_j u_k )
// with X_j = dXi/dX_j, L v = sum_j D_j^T (M X_j^2 D_j v) (symmetric),
// c = u (Burgers), c prescribed (advection) or no advection (heat).
// Its VJP, with mu_k = Minv lam_k pointwise:
//   ubar_m = - sum_j D_j^T [ nu M X_j^2 D_j mu_m + X_j c_j M mu_m ]
//            - [Burgers] sum_k X_m (D_m u_k) M mu_k
// (the last line is the derivative through the advecting velocity u_m).
//
// DSS Smooth replaces each member of a class by the class sum times
// 1/mult, and mult is the class size, constant over the class: the matrix
// is symmetric, so the adjoint of Smooth is Smooth itself.
//
// The RK step VJP runs the stage structure of Stepper::step (api_rk.cu)
// backwards on the stage inputs it taped.  The gradient of
// J = 1/2 sum_k ||u_k(T) - obs_k||_M^2 keeps a checkpoint every C steps,
// recomputes one segment at a time with the tape on, and runs the reverse
// sweep over the segment; the last segment is taped during the forward
// sweep, so it is not recomputed.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gf_common.cuh"
#include "k_dss.cuh"
#include "k_tensor.cuh"
#include "k_vec.cuh"
#include "ops_launch.cuh"
#include "rk_common.cuh"

using namespace gfk;

namespace {

// ---------------------------------------------------------------------
// VJP of the RHS.  One element per block; threads stride over its nodes.
// ---------------------------------------------------------------------
template <int N, int DIM, int EQN>
__global__ void __launch_bounds__(256)
    k_dudt_vjp(const __grid_constant__ Basis<double, N> B, const Geom<double> g, int64_t ne,
               double nu, const double *__restrict__ c0, const double *__restrict__ c1,
               const double *__restrict__ c2, const double *__restrict__ l0,
               const double *__restrict__ l1, const double *__restrict__ l2,
               const double *__restrict__ imass, double *__restrict__ o0, double *__restrict__ o1,
               double *__restrict__ o2) {
  constexpr int NN = N * N, NE = DIM == 3 ? NN * N : NN;
  constexpr int NC = EQN == GF_EQN_BURGERS ? DIM : 1;  // evolved components
  constexpr int NV = EQN == GF_EQN_HEAT ? 0 : DIM;     // advecting velocities
  extern __shared__ __align__(16) double sm[];
  double *sc = sm;              // NV * NE velocities
  double *smu = sc + NV * NE;   // NC * NE  mu = Minv lam
  double *ss = smu + NC * NE;   // DIM * NE flux terms
  double *smass = ss + DIM * NE;
  double *sx = smass + NE;      // DIM * NE dXi/dX
  const int64_t e = blockIdx.x;
  if (e >= ne) return;
  const int64_t base = e * NE;
  const double *cin[3] = {c0, c1, c2};
  const double *lin[3] = {l0, l1, l2};
  double *outp[3] = {o0, o1, o2};
  NodeGeom<double, DIM> eg;
  for (int k = 0; k < DIM; k++) eg.X[k] = 0.0;
  eg.J = 0.0;
  elem_geom<double, DIM>(g, e, eg);
  for (int a = threadIdx.x; a < NE; a += blockDim.x) {
    const int i = a % N, j = (a / N) % N, k = DIM == 3 ? a / NN : 0;
    NodeGeom<double, DIM> ng = eg;
    node_geom<double, DIM>(g, base + a, ng);
    const double w = DIM == 3 ? B.W[k] * B.W[j] * B.W[i] : B.W[j] * B.W[i];
    smass[a] = w * ng.J;
    for (int d = 0; d < DIM; d++) sx[d * NE + a] = ng.X[d];
    for (int v = 0; v < NV; v++) sc[v * NE + a] = cin[v][base + a];
    for (int m = 0; m < NC; m++) smu[m * NE + a] = imass[base + a] * lin[m][base + a];
  }
  __syncthreads();
  const int stride[3] = {1, N, NN};
  for (int m = 0; m < NC; m++) {
    const double *mu = smu + m * NE;
    for (int a = threadIdx.x; a < NE; a += blockDim.x) {
      const int li[3] = {a % N, (a / N) % N, DIM == 3 ? a / NN : 0};
      for (int d = 0; d < DIM; d++) {
        const int b0 = a - li[d] * stride[d];
        double dmu = 0.0;
#pragma unroll
        for (int q = 0; q < N; q++) dmu = fma(B.D[li[d] + q * N], mu[b0 + q * stride[d]], dmu);
        const double X = sx[d * NE + a];
        double s = nu * (smass[a] * ((X * X) * dmu));
        if (NV) s += X * sc[d * NE + a] * smass[a] * mu[a];
        ss[d * NE + a] = s;
      }
    }
    __syncthreads();
    for (int a = threadIdx.x; a < NE; a += blockDim.x) {
      const int li[3] = {a % N, (a / N) % N, DIM == 3 ? a / NN : 0};
      double o = 0.0;
      for (int d = 0; d < DIM; d++) {
        const int b0 = a - li[d] * stride[d];
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < N; q++) t = fma(B.D[q + li[d] * N], ss[d * NE + b0 + q * stride[d]], t);
        o -= t;
      }
      if (EQN == GF_EQN_BURGERS) {
        const int b0 = a - li[m] * stride[m];
        double r = 0.0;
        for (int k = 0; k < NC; k++) {
          double du = 0.0;
#pragma unroll
          for (int q = 0; q < N; q++)
            du = fma(B.D[li[m] + q * N], sc[k * NE + b0 + q * stride[m]], du);
          r = fma(du, smu[k * NE + a], r);
        }
        o -= sx[m * NE + a] * smass[a] * r;
      }
      outp[m][base + a] = o;
    }
    __syncthreads();
  }
}

// 3-d VJP, line-based like k_dudt3d: EPB elements per block, thread
// (a0, a1) of an element owns the x-line (j=a0, k=a1), the y-line
// (i=a0, k=a1) and the z-line (i=a0, j=a1).  Per evolved component m the
// x/y owners contract their lines (D, flux, D^T) into shared memory, the
// z-owner keeps its line in registers and sums the three.  The Burgers
// term of component m, X_m M sum_k (D_m u_k) mu_k, is formed by the owners
// of direction-m lines.
template <int N> constexpr int epb_vjp3() { return (160 / (N * N)) < 1 ? 1 : 160 / (N * N); }

// AFF: affine elements (g.egeom) known at compile time, so the per-node
// geometry path is not compiled in.
template <int N, int EPB, int EQN, bool AFF>
__global__ void __launch_bounds__(N *N *EPB)
    k_dudt_vjp3d(const __grid_constant__ Basis<double, N> B, const Geom<double> g, int64_t ne,
                 double nu, const double *__restrict__ c0, const double *__restrict__ c1,
                 const double *__restrict__ c2, const double *__restrict__ l0,
                 const double *__restrict__ l1, const double *__restrict__ l2,
                 const double *__restrict__ imass, double *__restrict__ o0,
                 double *__restrict__ o1, double *__restrict__ o2) {
  constexpr int NC = EQN == GF_EQN_BURGERS ? 3 : 1;  // evolved components
  constexpr int NV = EQN == GF_EQN_HEAT ? 0 : 3;     // advecting velocities
  constexpr int P = Pad<N>::P, PLANE = N * P, VOL = N * PLANE, NN = N * N, NNN = NN * N;
  constexpr int NF = NV + NC + 2;
  extern __shared__ __align__(16) double smv[];
  double *sc = smv + threadIdx.y * NF * VOL;  // NV velocity fields
  double *smu = sc + NV * VOL;                // NC fields mu = Minv lam
  double *sx = smu + NC * VOL, *sy = sx + VOL;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int a0 = t % N, a1 = t / N;
  const int64_t base = e * NNN;
  const double *cin[3] = {c0, c1, c2};
  const double *lin[3] = {l0, l1, l2};
  double *outp[3] = {o0, o1, o2};
  NodeGeom<double, 3> eg;
  eg.X[0] = eg.X[1] = eg.X[2] = eg.J = 0.0;
  if (active) elem_geom<double, 3>(g, e, eg);
  // geometry and mass at local node (i, j, k)
  auto geo = [&](int i, int j, int k, NodeGeom<double, 3> &ng) {
    ng = eg;
    if (!AFF && active) node_geom<double, 3>(g, base + k * NN + j * N + i, ng);
    return B.W[k] * B.W[j] * B.W[i] * ng.J;
  };
#pragma unroll 1
  for (int k = 0; k < N; k++) {
    const int64_t node = base + k * NN + a1 * N + a0;
    const int si = k * PLANE + a1 * P + a0;
    for (int v = 0; v < NV; v++) sc[v * VOL + si] = active ? cin[v][node] : 0.0;
    const double im = active ? imass[node] : 0.0;
    for (int m = 0; m < NC; m++) smu[m * VOL + si] = active ? im * lin[m][node] : 0.0;
  }
  __syncthreads();
#pragma unroll 1
  for (int m = 0; m < NC; m++) {
    const double *mu = smu + m * VOL;
    // the direction-dd line starting at shared offset base_s (node stride
    // `stride`, local index ijk[slot] running along it): D, flux, D^T, plus
    // the Burgers term when dd == m; written to dst (x/y) or kept in res
    auto line = [&](int dd, int base_s, int stride, int (&ijk)[3], int slot, double *dst,
                    double (&res)[N]) {
      double a[N], d[N], s[N];
#pragma unroll
      for (int q = 0; q < N; q++) a[q] = mu[base_s + q * stride];
      line_D<double, N>(B.D, a, d);
      double bt[N];
#pragma unroll
      for (int q = 0; q < N; q++) bt[q] = 0.0;
      if (EQN == GF_EQN_BURGERS && dd == m) {
        // sum_k (D_dd u_k) mu_k along the line
#pragma unroll 1
        for (int kk = 0; kk < 3; kk++) {
          double uu[N], du[N];
#pragma unroll
          for (int q = 0; q < N; q++) uu[q] = sc[kk * VOL + base_s + q * stride];
          line_D<double, N>(B.D, uu, du);
#pragma unroll
          for (int q = 0; q < N; q++) bt[q] = fma(du[q], smu[kk * VOL + base_s + q * stride], bt[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < N; q++) {
        ijk[slot] = q;
        NodeGeom<double, 3> ng;
        const double M = geo(ijk[0], ijk[1], ijk[2], ng);
        const double X = ng.X[dd];
        double sv = nu * (M * ((X * X) * d[q]));
        if (NV) sv += X * sc[dd * VOL + base_s + q * stride] * M * a[q];
        s[q] = sv;
        bt[q] *= X * M;
      }
      line_DT<double, N>(B.D, s, res);
#pragma unroll
      for (int q = 0; q < N; q++) res[q] += bt[q];
      if (dst) {
#pragma unroll
        for (int q = 0; q < N; q++) dst[base_s + q * stride] = res[q];
      }
    };
    {
      int ijk[3] = {0, a0, a1}, slot = 0;  // x-line (j=a0, k=a1)
      double r[N];
      line(0, a1 * PLANE + a0 * P, 1, ijk, slot, sx, r);
    }
    {
      int ijk[3] = {a0, 0, a1}, slot = 1;  // y-line (i=a0, k=a1)
      double r[N];
      line(1, a1 * PLANE + a0, P, ijk, slot, sy, r);
    }
    double rz[N];
    {
      int ijk[3] = {a0, a1, 0}, slot = 2;  // z-line (i=a0, j=a1), registers
      line(2, a1 * P + a0, PLANE, ijk, slot, nullptr, rz);
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int k = 0; k < N; k++) {
        const int si = k * PLANE + a1 * P + a0;
        outp[m][base + k * NN + a1 * N + a0] = -((sx[si] + sy[si]) + rz[k]);
      }
    }
    __syncthreads();
  }
}

template <int N, int DIM, int EQN>
int launch_vjp_n(gf_problem *prob, double nu, const double *const *c, const double *const *lam,
                 double *const *out, cudaStream_t st) {
  const Basis<double, N> B = make_basis<double, N>(prob);
  const Geom<double> g = geom_of<double>(prob);
  if (DIM == 3) {
    constexpr int EPB = epb_vjp3<N>();
    constexpr int NF = (EQN == GF_EQN_HEAT ? 0 : 3) + (EQN == GF_EQN_BURGERS ? 3 : 1) + 2;
    const size_t smem = sizeof(double) * NF * N * N * Pad<N>::P * EPB;
    auto kern = g.egeom ? k_dudt_vjp3d<N, EPB, EQN, true> : k_dudt_vjp3d<N, EPB, EQN, false>;
    set_smem(kern, smem);
    prob->launches++;
    kern<<<(unsigned)((prob->ne + EPB - 1) / EPB), dim3(N * N, EPB), smem, st>>>(
        B, g, prob->ne, nu, c[0], c[1], c[2], lam[0], lam[1], lam[2], prob->imass_d, out[0],
        out[1], out[2]);
    return cudaPeekAtLastError() == cudaSuccess ? GF_OK : GF_ERR_CUDA;
  }
  constexpr int NE = DIM == 3 ? N * N * N : N * N;
  constexpr int NC = EQN == GF_EQN_BURGERS ? DIM : 1;
  constexpr int NV = EQN == GF_EQN_HEAT ? 0 : DIM;
  const size_t smem = sizeof(double) * NE * (NV + NC + 2 * DIM + 1);
  auto kern = k_dudt_vjp<N, DIM, EQN>;
  set_smem(kern, smem);
  const int threads = NE < 256 ? ((NE + 31) / 32) * 32 : 256;
  prob->launches++;
  kern<<<(unsigned)prob->ne, threads, smem, st>>>(B, g, prob->ne, nu, c[0], c[1], c[2], lam[0],
                                                 lam[1], lam[2], prob->imass_d, out[0], out[1],
                                                 out[2]);
  return cudaPeekAtLastError() == cudaSuccess ? GF_OK : GF_ERR_CUDA;
}

template <int N>
struct VjpLaunch {
  static int run(gf_problem *prob, int eqn, double nu, const double *const *c,
                 const double *const *lam, double *const *out, cudaStream_t st) {
    if (prob->dim == 3) {
      if (eqn == GF_EQN_BURGERS) return launch_vjp_n<N, 3, GF_EQN_BURGERS>(prob, nu, c, lam, out, st);
      if (eqn == GF_EQN_ADVECT) return launch_vjp_n<N, 3, GF_EQN_ADVECT>(prob, nu, c, lam, out, st);
      return launch_vjp_n<N, 3, GF_EQN_HEAT>(prob, nu, c, lam, out, st);
    }
    if (eqn == GF_EQN_BURGERS) return launch_vjp_n<N, 2, GF_EQN_BURGERS>(prob, nu, c, lam, out, st);
    if (eqn == GF_EQN_ADVECT) return launch_vjp_n<N, 2, GF_EQN_ADVECT>(prob, nu, c, lam, out, st);
    return launch_vjp_n<N, 2, GF_EQN_HEAT>(prob, nu, c, lam, out, st);
  }
};

// ubar = F'(u)^T lam for every evolved component
int vjp(gf_problem *prob, int eqn, double nu, int nstate, const double *const *u,
        const double *const *c, const double *const *lam, double *const *ubar) {
  cudaStream_t st = prob->ctx->stream;
  const double *cc[3] = {nullptr, nullptr, nullptr};
  const double *ll[3] = {nullptr, nullptr, nullptr};
  double *oo[3] = {nullptr, nullptr, nullptr};
  if (eqn == GF_EQN_HEAT) {
    for (int k = 0; k < nstate; k++) {
      ll[0] = lam[k];
      oo[0] = ubar[k];
      int rc = dispatch_n<VjpLaunch>(prob->n, prob, eqn, nu, (const double *const *)cc,
                                     (const double *const *)ll, (double *const *)oo, st);
      if (rc) return rc;
    }
    return GF_OK;
  }
  for (int d = 0; d < prob->dim; d++) cc[d] = eqn == GF_EQN_BURGERS ? u[d] : c[d];
  for (int k = 0; k < nstate; k++) {
    ll[k] = lam[k];
    oo[k] = ubar[k];
  }
  return dispatch_n<VjpLaunch>(prob->n, prob, eqn, nu, (const double *const *)cc,
                               (const double *const *)ll, (double *const *)oo, st);
}

#define GSTRIDE(i, n)                                                        \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
       i += (int64_t)gridDim.x * blockDim.x)

// Butcher reverse, start: acc = lw; lamK_m = cm * lw
__global__ void k_adj_start(int64_t n, const double *__restrict__ lw, double *__restrict__ acc,
                            double *K0, double *K1, double *K2, double *K3, double c0, double c1,
                            double c2, double c3) {
  GSTRIDE(i, n) {
    const double v = lw[i];
    acc[i] = v;
    K0[i] = c0 * v;
    if (K1) K1[i] = c1 * v;
    if (K2) K2[i] = c2 * v;
    if (K3) K3[i] = c3 * v;
  }
}
// Butcher reverse, stage m: acc += l; lamK_j += b_j l (j < m)
__global__ void k_adj_fan(int64_t n, const double *__restrict__ l, double *__restrict__ acc,
                          double *K0, double *K1, double *K2, double b0, double b1, double b2) {
  GSTRIDE(i, n) {
    const double v = l[i];
    acc[i] += v;
    if (K0) K0[i] += b0 * v;
    if (K1) K1[i] += b1 * v;
    if (K2) K2[i] += b2 * v;
  }
}
// SSP reverse, substep m: Sm += a lv + ad f; Sy += b lv; Sy2 += b2 lv
__global__ void k_adj_ssp(int64_t n, const double *__restrict__ lv, const double *__restrict__ f,
                          double a, double ad, double *Sm, double b, double *Sy, double b2,
                          double *Sy2) {
  GSTRIDE(i, n) {
    const double v = lv[i];
    Sm[i] += a * v + ad * f[i];
    if (Sy) Sy[i] += b * v;
    if (Sy2) Sy2[i] += b2 * v;
  }
}
// out = mass (u - obs); adds 1/2 sum mass (u - obs)^2 into *J
__global__ void __launch_bounds__(RED_THREADS)
    k_misfit(int64_t n, const double *__restrict__ mass, const double *__restrict__ u,
             const double *__restrict__ obs, double *__restrict__ out, double *partials,
             unsigned int *counter, double *J) {
  __shared__ double sh[32];
  double s = 0.0;
  GSTRIDE(i, n) {
    const double d = u[i] - obs[i];
    out[i] = mass[i] * d;
    s += mass[i] * d * d;
  }
  s = block_reduce<false>(s, sh);
  double pv[1] = {s};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    const double t = fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      *J += 0.5 * t;
      *counter = 0;
    }
  }
}

// Reverse sweep of one step over its taped stage inputs.
struct Reverse {
  gf_problem *prob;
  gfrk::Stepper<double> &S;
  cudaStream_t st;
  int64_t n;
  int nstate, ns;
  unsigned g;
  double *lamK[4][3] = {{nullptr}};  // Butcher: cotangents of K_m; SSP: of stage inputs
  double *acc[3] = {nullptr}, *tmp[3] = {nullptr};
  bool ok = true;

  Reverse(gf_problem *p, gfrk::Stepper<double> &s, int slot)
      : prob(p), S(s), st(p->ctx->stream), n(p->nlocal), nstate(s.nstate), ns(s.stages()) {
    g = grid_for(n, 256, p->ctx->sm_count * 8);
    for (int k = 0; k < nstate; k++) {
      acc[k] = (double *)gf_work(p, slot++, sizeof(double) * n);
      tmp[k] = (double *)gf_work(p, slot++, sizeof(double) * n);
      ok = ok && acc[k] && tmp[k];
      for (int m = 0; m < ns; m++) {
        lamK[m][k] = (double *)gf_work(p, slot++, sizeof(double) * n);
        ok = ok && lamK[m][k];
      }
    }
  }
  static int slots(int nstate) { return nstate * 6; }
  // Smooth (its own transpose) on every state component: one lattice pass
  // on box problems (the stepper's multi-component kernel), CSR otherwise
  void smooth_n(double *const *v) { S.smooth_n(v); }

  // lam <- (d step/d uin)^T lam; tape[3*m + k] = input of stage m
  int run(double *const *tape, double *const *lam, double dt) {
    if (S.scheme <= 4) return butcher(tape, lam, dt);
    return ssp(tape, lam, dt);
  }

  // uout = S(uin + sum_m c_m h K_m), K_m = S F(u^m),
  // u^m = uin + sum_{j<m} beta_mj h K_j (m < ns-1), u^{ns-1} = S(same).
  int butcher(double *const *tape, double *const *lam, double h) {
    double alpha[4], beta[4][4], cc[4];
    gfrk::butcher(S.scheme, alpha, beta, cc);
    smooth_n(lam);
    for (int k = 0; k < nstate; k++) {
      prob->launches++;
      k_adj_start<<<g, 256, 0, st>>>(n, lam[k], acc[k], lamK[0][k], ns > 1 ? lamK[1][k] : nullptr,
                                     ns > 2 ? lamK[2][k] : nullptr, ns > 3 ? lamK[3][k] : nullptr,
                                     cc[0] * h, cc[1] * h, cc[2] * h, cc[3] * h);
    }
    for (int m = ns - 1; m >= 0; m--) {
      double *mu[3] = {lamK[m][0], lamK[m][1], lamK[m][2]};
      smooth_n(mu);
      const double *um[3] = {tape[3 * m], tape[3 * m + 1], tape[3 * m + 2]};
      int rc = vjp(prob, S.eqn, (double)S.nu, nstate, um, S.c, (const double *const *)mu, tmp);
      if (rc) return rc;
      if (m == ns - 1) smooth_n(tmp);
      for (int k = 0; k < nstate; k++) {
        prob->launches++;
        k_adj_fan<<<g, 256, 0, st>>>(n, tmp[k], acc[k], m > 0 ? lamK[0][k] : nullptr,
                                     m > 1 ? lamK[1][k] : nullptr, m > 2 ? lamK[2][k] : nullptr,
                                     beta[m][0] * h, beta[m][1] * h, beta[m][2] * h);
      }
    }
    for (int k = 0; k < nstate; k++)
      cudaMemcpyAsync(lam[k], acc[k], sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    return GF_OK;
  }

  // Substep m of the SSP schemes (gexrk_stepper.ipp:533-780) maps its input
  // s_m to out_m = S(a (dt F(s_m) + s_m) + b y + b2 y2) with y, y2 earlier
  // stage inputs (s_0 = uin); out_m = s_{m+1}.
  void coeffs(int m, double &a, double &b, int &y, double &b2, int &y2) const {
    a = 1.0;
    b = b2 = 0.0;
    y = y2 = 0;
    switch (S.scheme) {
      case GF_SSP22:
        if (m == 1) a = b = 0.5;
        break;
      case GF_SSP33:
        if (m == 1) { a = 0.25; b = 0.75; }
        if (m == 2) { a = 2.0 / 3.0; b = 1.0 / 3.0; }
        break;
      default:  // SSP34
        if (m == 0) { a = 0.5; b = 0.5; }
        if (m == 1) { a = 0.5; b = 0.5; y = 1; }
        if (m == 2) { a = 1.0 / 6.0; b = 1.0 / 6.0; y = 2; b2 = 2.0 / 3.0; }
        if (m == 3) { a = 0.5; b = 0.5; y = 3; }
        break;
    }
  }

  int ssp(double *const *tape, double *const *lam, double dt) {
    for (int m = 0; m < ns; m++)
      for (int k = 0; k < nstate; k++)
        cudaMemsetAsync(lamK[m][k], 0, sizeof(double) * n, st);
    double *lout[3] = {lam[0], lam[1], lam[2]};  // cotangent of out_m
    for (int m = ns - 1; m >= 0; m--) {
      smooth_n(lout);
      const double *um[3] = {tape[3 * m], tape[3 * m + 1], tape[3 * m + 2]};
      int rc = vjp(prob, S.eqn, (double)S.nu, nstate, um, S.c, (const double *const *)lout, tmp);
      if (rc) return rc;
      double a, b, b2;
      int y, y2;
      coeffs(m, a, b, y, b2, y2);
      const double ad = a * dt;  // weight of the RHS term
      if (y == m) {  // y is this substep's own input
        a += b;
        b = 0.0;
      }
      for (int k = 0; k < nstate; k++) {
        prob->launches++;
        k_adj_ssp<<<g, 256, 0, st>>>(n, lout[k], tmp[k], a, ad, lamK[m][k], b,
                                     b != 0.0 ? lamK[y][k] : nullptr, b2,
                                     b2 != 0.0 ? lamK[y2][k] : nullptr);
      }
      // every contribution to the cotangent of s_m is in (later substeps
      // only feed stage inputs with smaller index)
      for (int k = 0; k < nstate; k++) lout[k] = lamK[m][k];
    }
    for (int k = 0; k < nstate; k++)
      cudaMemcpyAsync(lam[k], lamK[0][k], sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    return GF_OK;
  }
};

// tape buffers for `nsteps` steps: tape[(s*4 + m)*3 + k]
bool alloc_tape(gf_problem *prob, int nsteps, int ns, int nstate, int slot,
                std::vector<double *> &tape) {
  tape.assign((size_t)nsteps * 12, nullptr);
  for (int s = 0; s < nsteps; s++)
    for (int m = 0; m < ns; m++)
      for (int k = 0; k < nstate; k++) {
        double *p = (double *)gf_work(prob, slot++, sizeof(double) * prob->nlocal);
        if (!p) return false;
        tape[(s * 4 + m) * 3 + k] = p;
      }
  return true;
}

constexpr int SLOT_ADJ = 1000;  // gf_work slots of this file start here

}  // namespace

extern "C" int gf_dudt_vjp(gf_problem_t prob, int dtype, int eqn, double nu, int nstate,
                           const void *const *u, const void *const *c, const void *const *lam,
                           void *const *ubar) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, prob->geom <= GF_GEOM_REGULAR,
             "the adjoint path covers affine and regular (diagonal-metric) grids");
  GF_REQUIRE(ctx, dtype == GF_F64, "the adjoint path is FP64");
  GF_REQUIRE(ctx, eqn == GF_EQN_ADVECT || eqn == GF_EQN_BURGERS || eqn == GF_EQN_HEAT,
             "unknown equation %d", eqn);
  GF_REQUIRE(ctx, lam && ubar, "lam and ubar are required");
  GF_REQUIRE(ctx, eqn != GF_EQN_ADVECT || (c && nstate == 1), "advection: one component and c");
  GF_REQUIRE(ctx, eqn != GF_EQN_BURGERS || (u && nstate == prob->dim),
             "Burgers evolves dim components and needs u");
  GF_REQUIRE(ctx, eqn != GF_EQN_HEAT || (nstate >= 1 && nstate <= 3), "heat: 1..3 components");
  for (int k = 0; k < nstate; k++) GF_REQUIRE(ctx, lam[k] && ubar[k], "component %d missing", k);
  int rc = vjp(prob, eqn, nu, nstate, (const double *const *)u, (const double *const *)c,
               (const double *const *)lam, (double *const *)ubar);
  if (rc) return gf_fail(ctx, rc, "dudt VJP launch failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_rk_step_vjp(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                              const void *const *u0, const void *const *c, double dt,
                              void *const *lam) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, prob->geom <= GF_GEOM_REGULAR,
             "the adjoint path covers affine and regular (diagonal-metric) grids");
  GF_REQUIRE(ctx, dtype == GF_F64, "the adjoint path is FP64");
  int rc = gfrk::check_traits(prob, traits, u0, c);
  if (rc) return rc;
  GF_REQUIRE(ctx, lam, "lam is required");
  for (int k = 0; k < traits->nstate; k++) GF_REQUIRE(ctx, lam[k], "lam component %d missing", k);
  gfrk::Stepper<double> S(prob, traits, c);
  if (!S.alloc()) return gf_fail(ctx, GF_ERR_NOMEM, "RK work allocation failed");
  int slot = SLOT_ADJ;
  Reverse R(prob, S, slot);
  slot += Reverse::slots(S.nstate);
  std::vector<double *> tape;
  double *out[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < S.nstate; k++) out[k] = (double *)gf_work(prob, slot++, sizeof(double) * S.n);
  slot += 3;
  if (!R.ok || !out[0] || !alloc_tape(prob, 1, S.stages(), S.nstate, slot, tape))
    return gf_fail(ctx, GF_ERR_NOMEM, "adjoint work allocation failed");
  if ((rc = S.step((double *const *)u0, out, dt, tape.data())))
    return gf_fail(ctx, rc, "taped step failed");
  if ((rc = R.run(tape.data(), (double *const *)lam, dt)))
    return gf_fail(ctx, rc, "reverse sweep failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_adjoint_gradient(gf_problem_t prob, const gf_rk_traits *traits,
                                   const double *const *u0, const double *const *c,
                                   const double *const *u_obs, double dt, int nsteps,
                                   int checkpoint_every, double *J, double *const *grad) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, prob->geom <= GF_GEOM_REGULAR,
             "the adjoint path covers affine and regular (diagonal-metric) grids");
  int rc = gfrk::check_traits(prob, traits, (const void *const *)u0, (const void *const *)c);
  if (rc) return rc;
  GF_REQUIRE(ctx, u_obs && grad && nsteps >= 0 && checkpoint_every >= 1, "bad arguments");
  for (int k = 0; k < traits->nstate; k++)
    GF_REQUIRE(ctx, u_obs[k] && grad[k], "component %d missing", k);
  const int64_t n = prob->nlocal;
  const size_t bytes = sizeof(double) * n;
  cudaStream_t st = ctx->stream;
  gfrk::Stepper<double> S(prob, traits, (const void *const *)c);
  if (!S.alloc()) return gf_fail(ctx, GF_ERR_NOMEM, "RK work allocation failed");
  const int nst = S.nstate, ns = S.stages();
  const int C = std::max(1, std::min(checkpoint_every, std::max(nsteps, 1)));
  const int nseg = (nsteps + C - 1) / C;
  int slot = SLOT_ADJ;
  Reverse R(prob, S, slot);
  slot += Reverse::slots(nst);
  // checkpoints: the state at the start of every segment
  std::vector<double *> ck((size_t)std::max(nseg, 1) * 3, nullptr);
  for (int sg = 0; sg < nseg; sg++)
    for (int k = 0; k < nst; k++)
      if (!(ck[sg * 3 + k] = (double *)gf_work(prob, slot++, bytes)))
        return gf_fail(ctx, GF_ERR_NOMEM, "checkpoint allocation failed");
  double *ua[3] = {nullptr, nullptr, nullptr}, *ub[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < nst; k++) {
    ua[k] = (double *)gf_work(prob, slot++, bytes);
    ub[k] = (double *)gf_work(prob, slot++, bytes);
  }
  std::vector<double *> tape;
  if (!R.ok || !ua[0] || !ub[0] || !alloc_tape(prob, C, ns, nst, slot, tape))
    return gf_fail(ctx, GF_ERR_NOMEM, "adjoint work allocation failed");
  auto tp = [&](int j) { return tape.data() + (size_t)j * 12; };
  auto d2d = [&](double *dst, const double *src) {
    cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
  };
  // forward sweep; the last segment is taped on the way
  for (int k = 0; k < nst; k++) d2d(ua[k], u0[k]);
  const int last0 = nseg > 0 ? (nseg - 1) * C : 0;
  for (int s = 0; s < nsteps; s++) {
    if (s % C == 0)
      for (int k = 0; k < nst; k++) d2d(ck[(s / C) * 3 + k], ua[k]);
    if ((rc = S.step(ua, ub, dt, s >= last0 ? tp(s - last0) : nullptr)))
      return gf_fail(ctx, rc, "forward step failed");
    std::swap(ua, ub);
  }
  // J and its gradient with respect to u(T): lam = M (u(T) - obs)
  double *Jd = prob->scal_d + 60;
  cudaMemsetAsync(Jd, 0, sizeof(double), st);
  for (int k = 0; k < nst; k++) {
    prob->launches++;
    k_misfit<<<grid_for(n, RED_THREADS, prob->npartials), RED_THREADS, 0, st>>>(
        n, prob->mass_d, ua[k], u_obs[k], grad[k], prob->partials, prob->counter, Jd);
  }
  // reverse sweep, segment by segment
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int s0 = sg * C, s1 = std::min(nsteps, s0 + C);
    if (sg != nseg - 1) {  // recompute the segment with the tape on
      for (int k = 0; k < nst; k++) d2d(ua[k], ck[sg * 3 + k]);
      for (int s = s0; s < s1; s++) {
        if ((rc = S.step(ua, ub, dt, tp(s - s0)))) return gf_fail(ctx, rc, "recompute failed");
        std::swap(ua, ub);
      }
    }
    for (int s = s1 - 1; s >= s0; s--)
      if ((rc = R.run(tp(s - s0), grad, dt))) return gf_fail(ctx, rc, "reverse step failed");
  }
  GF_CHECK_LAUNCH(ctx);
  GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h + 60, Jd, sizeof(double), cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  if (J) *J = prob->scal_h[60];
  return GF_OK;
}

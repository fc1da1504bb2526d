// api_cg.cu -- conjugate gradient on the assembled Helmholtz operator,
// following GCG::solve_impl (solvers/gcg.ipp:239-382, the Deville-Fischer-
// Mund form) with the reference's DSS Sum, Dirichlet mask, multiplicity-
// weighted dots and norm-based stopping rule, plus a Jacobi preconditioner
// and a mixed-precision (FP32 inner solve, FP64 residual and refinement)
// variant, neither of which the reference has.
//
// Every iteration is four kernels that never wait on the host:
//   1. q = A w                         (fused element apply)
//   2. q = mask * DSS_Sum(q), <w,q>    (class gather-reduce-scatter + dot;
//      the last block forms alpha = rho / <w,q>)
//   3. x += alpha w, r -= alpha q, z = P^-1 r, rho' = <r,z>, norm(r)
//      (the last block forms beta, checks convergence, sets `done`)
//   4. w = beta w + z
// Scalars live in a device block; once `done` is set all later kernels of
// the batch return at once, so batches of iterations can be queued ahead
// and the host reads the state only every `check_every` iterations.
#include <cmath>
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
  S_NTOT,   // number of local nodes (EUC norm)
  S_IVOL,   // 1/volume (L2, L1 norms)
  S_NORMT,  // norm type
  S_REL,    // 1: rtol = tol * norm(b) always (inner solves)
  S_COUNT
};

struct CGVecs {
  const double *mask;   // may be null
  const double *imult;
  const double *dinv;   // may be null
  const double *mass;
  double *hist;         // residual history (maxit)
};

__device__ __forceinline__ double finish_norm(int normtype, double v, const double *scal) {
  if (normtype == GF_NORM_INF) return v;
  if (normtype == GF_NORM_EUC) return sqrt(v / scal[S_NTOT]);
  if (normtype == GF_NORM_L2) return sqrt(v * scal[S_IVOL]);
  return v * scal[S_IVOL];
}

// contribution of node i to the norm partial of type normtype
__device__ __forceinline__ double norm_term(int normtype, double r, const double *mass, int64_t i) {
  if (normtype == GF_NORM_INF) return fabs(r);
  if (normtype == GF_NORM_EUC) return r * r;
  if (normtype == GF_NORM_L2) return mass[i] * (r * r);
  return mass[i] * fabs(r);
}

// r = b - Ax (in place on ax -> r)
template <typename T>
__global__ void k_cg_resid(int64_t n, const T *__restrict__ b, const T *__restrict__ ax,
                           T *__restrict__ r) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v = b[i];
    v -= ax[i];
    r[i] = v;
  }
}

// x = mask*x + xb  (solve_impl (2) prologue) or x = mask*x + xb at exit
template <typename T>
__global__ void k_cg_lift(int64_t n, const double *__restrict__ mask, const T *__restrict__ xb,
                          T *__restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v = x[i];
    if (mask) v *= (T)mask[i];
    if (xb) v += xb[i];
    x[i] = v;
  }
}

// DSS Sum + mask over classes; with DOT also accumulates <w,q>_imult and
// the last block forms alpha = rho / <w,q>.
template <typename T, bool DOT>
__global__ void __launch_bounds__(RED_THREADS)
    k_cg_dss(int64_t nclass, const int32_t *__restrict__ ptr, const int32_t *__restrict__ mem,
             const double *__restrict__ mask, const double *__restrict__ imult,
             const T *__restrict__ w, T *__restrict__ q, double *scal, double *partials,
             unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  double dot = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nclass;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = ptr[c], e = ptr[c + 1];
    T s = T(0);
    for (int32_t k = b; k < e; k++) s = __fadd_rn_t(s, q[mem[k]]);
    for (int32_t k = b; k < e; k++) {
      const int32_t m = mem[k];
      T v = s;
      if (mask) v *= (T)mask[m];
      q[m] = v;
      if (DOT) dot += ((double)w[m] * (double)v) * imult[m];
    }
  }
  if (!DOT) return;
  dot = block_reduce<false>(dot, sh);
  double pv[1] = {dot};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    double wq = fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      double alpha = scal[S_RHO] / wq;
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

// z = P^-1 r; w = z; rho = <r,z>_imult; bnorm partial from b; sets rtol.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
    k_cg_start(int64_t n, const T *__restrict__ b, const T *__restrict__ r, T *__restrict__ w,
               CGVecs v, double tol, double *scal, double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  const int normtype = (int)scal[S_NORMT];
  double rho = 0.0, bn = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = r[i];
    const T zi = v.dinv ? (T)v.dinv[i] * ri : ri;
    w[i] = zi;
    rho += ((double)ri * (double)zi) * v.imult[i];
    const double t = norm_term(normtype, (double)b[i], v.mass, i);
    bn = normtype == GF_NORM_INF ? fmax(bn, t) : bn + t;
  }
  rho = block_reduce<false>(rho, sh);
  bn = normtype == GF_NORM_INF ? block_reduce<true>(bn, sh) : block_reduce<false>(bn, sh);
  double pv[2] = {rho, bn};
  if (publish_partials<2>(pv, partials, counter, gridDim.x)) {
    double rho_t = fold_partials<false>(partials, gridDim.x, sh);
    double bn_t = normtype == GF_NORM_INF ? fold_partials<true>(partials + gridDim.x, gridDim.x, sh)
                                          : fold_partials<false>(partials + gridDim.x, gridDim.x, sh);
    if (threadIdx.x == 0) {
      double bnorm = finish_norm(normtype, bn_t, scal);
      double rtol = (scal[S_REL] != 0.0 || bnorm >= 1.0) ? tol * bnorm : tol;
      scal[S_RHO] = rho_t;
      scal[S_BNORM] = bnorm;
      scal[S_RTOL] = rtol;
      scal[S_RNORM] = 10.0 * rtol;
      scal[S_ITER] = 0.0;
      scal[S_FLAG] = 0.0;
      scal[S_DONE] = (scal[S_MAXIT] <= 0.0 || !(10.0 * rtol > rtol)) ? 1.0 : 0.0;
      *counter = 0;
    }
  }
}

// x += alpha w; r -= alpha q; rho' = <r, P^-1 r>; norm(r); beta; stop test.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
    k_cg_update(int64_t n, T *__restrict__ x, const T *__restrict__ w, T *__restrict__ r,
                const T *__restrict__ q, CGVecs v, double *scal, double *partials,
                unsigned int *counter) {
  __shared__ double sh[32];
  if (scal[S_DONE] != 0.0) return;
  const int normtype = (int)scal[S_NORMT];
  const T alpha = (T)scal[S_ALPHA];
  double rho = 0.0, rn = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = x[i] + alpha * w[i];
    const T ri = r[i] + (-alpha) * q[i];
    r[i] = ri;
    const T zi = v.dinv ? (T)v.dinv[i] * ri : ri;
    rho += ((double)ri * (double)zi) * v.imult[i];
    const double t = norm_term(normtype, (double)ri, v.mass, i);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  }
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
      if (v.hist) v.hist[it] = rnorm;
      scal[S_ITER] = (double)(it + 1);
      if (!isfinite(rnorm) || !isfinite(beta)) scal[S_FLAG] = 1.0;
      if (rnorm <= scal[S_RTOL] || it + 1 >= (int)scal[S_MAXIT] || !isfinite(rnorm) ||
          !isfinite(beta))
        scal[S_DONE] = 2.0;
      *counter = 0;
    }
  }
}

// w = beta w + z, z = P^-1 r.  Skipped once the solve has stopped.
template <typename T>
__global__ void k_cg_wupdate(int64_t n, T *__restrict__ w, const T *__restrict__ r,
                             const double *__restrict__ dinv, const double *scal) {
  if (scal[S_DONE] != 0.0) return;
  const T beta = (T)scal[S_BETA];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = r[i];
    const T zi = dinv ? (T)dinv[i] * ri : ri;
    w[i] = beta * w[i] + T(1) * zi;
  }
}

// local diagonal of p L + q M at every node (before DSS Sum)
template <typename T>
__global__ void k_helm_diag(int64_t n, int dim, int nb, Basis<double, GF_MAXN> B,
                            const double *__restrict__ egeom, const double *__restrict__ ngeom,
                            double p, double q, int use_mass, T *__restrict__ diag) {
  const int nn = dim == 2 ? nb * nb : nb * nb * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i / nn;
    const int a = (int)(i % nn);
    int li[3] = {a % nb, (a / nb) % nb, a / (nb * nb)};
    int stride[3] = {1, nb, nb * nb};
    double s = 0.0;
    for (int d = 0; d < dim; d++) {
      for (int m = 0; m < nb; m++) {
        const double Dm = B.D[m + li[d] * nb];
        const int64_t gb = i + (int64_t)(m - li[d]) * stride[d];
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
    s *= p;
    if (use_mass) {
      const double J = egeom ? egeom[e * (dim + 1) + dim] : ngeom[(int64_t)dim * n + i];
      const double w = dim == 2 ? B.W[li[1]] * B.W[li[0]]
                                : B.W[li[2]] * B.W[li[1]] * B.W[li[0]];
      s += q * (w * J);
    }
    diag[i] = (T)s;
  }
}

__global__ void k_invert(int64_t n, double *__restrict__ d) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    d[i] = 1.0 / d[i];
}

// rnorm of an FP64 residual into scal[slot] (host reads it)
__global__ void __launch_bounds__(RED_THREADS)
    k_norm(int64_t n, int normtype, const double *__restrict__ r, const double *__restrict__ mass,
           double *scal, int slot, double *partials, unsigned int *counter) {
  __shared__ double sh[32];
  double rn = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double t = norm_term(normtype, r[i], mass, i);
    rn = normtype == GF_NORM_INF ? fmax(rn, t) : rn + t;
  }
  rn = normtype == GF_NORM_INF ? block_reduce<true>(rn, sh) : block_reduce<false>(rn, sh);
  double pv[1] = {rn};
  if (publish_partials<1>(pv, partials, counter, gridDim.x)) {
    double t = normtype == GF_NORM_INF ? fold_partials<true>(partials, gridDim.x, sh)
                                       : fold_partials<false>(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      scal[slot] = finish_norm(normtype, t, scal);
      *counter = 0;
    }
  }
}

struct Solver {
  gf_problem *prob;
  gf_context *ctx;
  cudaStream_t st;
  int64_t n;
  unsigned gvec, gcls;

  explicit Solver(gf_problem *p) : prob(p), ctx(p->ctx), st(p->ctx->stream), n(p->nlocal) {
    gvec = grid_for(n, RED_THREADS, std::min(p->npartials, ctx->sm_count * 4));
    gcls = grid_for(p->nclass, RED_THREADS, std::min(p->npartials, ctx->sm_count * 4));
  }

  // Jacobi inverse diagonal (assembled), FP64, cached in work slot 9
  double *jacobi(double p, double q, int use_mass) {
    double *d = (double *)gf_work(prob, 9, sizeof(double) * n);
    if (!d) return nullptr;
    Basis<double, GF_MAXN> B;
    for (int i = 0; i < prob->n * prob->n; i++) B.D[i] = prob->D[i];
    for (int i = 0; i < prob->n; i++) B.W[i] = prob->W[i];
    unsigned g = grid_for(n, 256, ctx->sm_count * 8);
    prob->launches++;
    k_helm_diag<double><<<g, 256, 0, st>>>(n, prob->dim, prob->n, B, prob->egeom_d, prob->ngeom_d,
                                           p, q, use_mass, d);
    launch_dss<double>(prob, GF_DSS_SUM, d, st);
    prob->launches++;
    k_invert<<<g, 256, 0, st>>>(n, d);
    return d;
  }

  // One CG solve in precision T on device vectors; x holds the initial
  // guess.  b: right-hand side; xb: boundary lift or null.  Returns the
  // GCGERR-style code; iterations in *iters.
  template <typename T>
  int solve(const gf_cg_traits &tr, double p, double q, int use_mass, const T *b, const T *xb,
            T *x, bool bbv, double tol, bool relative, int maxit, const double *dinv, double *hist,
            int *iters, double *rnorm_out, int slot0) {
    T *r = (T *)gf_work(prob, slot0 + 0, sizeof(T) * n);
    T *w = (T *)gf_work(prob, slot0 + 1, sizeof(T) * n);
    T *qv = (T *)gf_work(prob, slot0 + 2, sizeof(T) * n);
    if (!r || !w || !qv) return gf_fail(ctx, GF_ERR_NOMEM, "CG work allocation failed");
    double *scal = prob->scal_d;
    const double *mask = bbv ? prob->mask_d : nullptr;
    CGVecs v{mask, prob->imult_d, dinv, prob->mass_d, hist};
    // scalars
    double init[S_COUNT] = {0};
    init[S_MAXIT] = (double)maxit;
    init[S_NTOT] = (double)n;
    init[S_NORMT] = (double)tr.normtype;
    init[S_IVOL] = 1.0 / prob->volume;
    init[S_REL] = relative ? 1.0 : 0.0;
    std::copy(init, init + S_COUNT, prob->scal_h);
    GF_CUDA(ctx, cudaMemcpyAsync(scal, prob->scal_h, sizeof(double) * S_COUNT,
                                 cudaMemcpyHostToDevice, st));
    unsigned gel = grid_for(n, 256, ctx->sm_count * 8);
    if (bbv && (xb || mask)) {
      prob->launches++;
      k_cg_lift<T><<<gel, 256, 0, st>>>(n, mask, xb, x);
    }
    // r = b - A x; DSS Sum; mask
    int rc = launch_helm<T>(prob, (T)p, nullptr, (T)q, nullptr, use_mass, x, w, st);
    if (rc) return gf_fail(ctx, rc, "apply failed");
    prob->launches++;
    k_cg_resid<T><<<gel, 256, 0, st>>>(n, b, w, r);
    prob->launches++;
    k_cg_dss<T, false><<<gcls, RED_THREADS, 0, st>>>(prob->nclass, prob->class_ptr, prob->members,
                                                      mask, prob->imult_d, w, r, scal,
                                                      prob->partials, prob->counter);
    prob->launches++;
    k_cg_start<T><<<gvec, RED_THREADS, 0, st>>>(n, b, r, w, v, tol, scal, prob->partials,
                                               prob->counter);
    GF_CHECK_LAUNCH(ctx);
    const int every = tr.check_every > 0 ? tr.check_every : 16;
    int issued = 0;
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    double *hbuf = prob->scal_h + 32;  // two host slots of S_COUNT..: DONE, ITER
    int pending = -1;
    bool stop = false;
    int status = 0;
    while (!stop) {
      // enqueue a batch
      for (int k = 0; k < every && issued < maxit; k++, issued++) {
        launch_helm<T>(prob, (T)p, nullptr, (T)q, nullptr, use_mass, w, qv, st, scal + S_DONE);
        prob->launches++;
        k_cg_dss<T, true><<<gcls, RED_THREADS, 0, st>>>(prob->nclass, prob->class_ptr,
                                                         prob->members, mask, prob->imult_d, w,
                                                         qv, scal, prob->partials, prob->counter);
        prob->launches++;
        k_cg_update<T><<<gvec, RED_THREADS, 0, st>>>(n, x, w, r, qv, v, scal, prob->partials,
                                                    prob->counter);
        prob->launches++;
        k_cg_wupdate<T><<<gel, 256, 0, st>>>(n, w, r, dinv, scal);
      }
      GF_CHECK_LAUNCH(ctx);
      const int slot = (pending + 1) & 1;
      GF_CUDA(ctx, cudaMemcpyAsync(hbuf + 2 * slot, scal + S_DONE, sizeof(double) * 2,
                                   cudaMemcpyDeviceToHost, st));
      cudaEventRecord(ev[slot], st);
      // wait for the previous batch's flag while this one runs
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
    const int it = (int)prob->scal_h[S_ITER];
    const double rn = prob->scal_h[S_RNORM];
    if (iters) *iters = it;
    if (rnorm_out) *rnorm_out = rn;
    if (prob->scal_h[S_FLAG] != 0.0) status = GF_ERR_NONFINITE;
    if (bbv) {
      prob->launches++;
      k_cg_lift<T><<<gel, 256, 0, st>>>(n, prob->mask_d, xb, x);
    }
    GF_CHECK_LAUNCH(ctx);
    if (status) return gf_fail(ctx, status, "CG breakdown: non-finite scalar at iteration %d", it);
    if (it >= maxit && rn > tr.tol) return GF_CG_NOCONVERGE;
    return GF_OK;
  }
};

}  // namespace

extern "C" int gf_cg_solve(gf_problem_t prob, const gf_cg_traits *tr, double p, double q,
                           int use_mass, const double *b, const double *xb, double *x, int *iters,
                           double *final_norm, double *residuals) {
  if (!prob || !tr) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, b && x, "b and x are required");
  GF_REQUIRE(ctx, tr->maxit >= 0, "maxit must be >= 0");
  GF_REQUIRE(ctx, tr->normtype >= GF_NORM_INF && tr->normtype <= GF_NORM_L1, "bad norm type");
  GF_REQUIRE(ctx, tr->precision == GF_CG_FP64 || tr->precision == GF_CG_MIXED, "bad precision");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  Solver S(prob);
  const int64_t n = prob->nlocal;
  const bool bbv = xb != nullptr;
  double *dinv = nullptr;
  if (tr->precond == GF_PRECOND_JACOBI) {
    dinv = S.jacobi(p, q, use_mass);
    if (!dinv) return gf_fail(ctx, GF_ERR_NOMEM, "Jacobi diagonal allocation failed");
  }
  double *hist = nullptr;
  if (residuals && tr->maxit > 0) {
    hist = (double *)gf_work(prob, 11, sizeof(double) * tr->maxit);
    cudaMemsetAsync(hist, 0, sizeof(double) * tr->maxit, ctx->stream);
  }
  int rc;
  int it = 0;
  double rn = 0.0;
  if (tr->precision == GF_CG_FP64) {
    rc = S.solve<double>(*tr, p, q, use_mass, b, xb, x, bbv, tr->tol, tr->relative != 0, tr->maxit, dinv, hist,
                         &it, &rn, 0);
  } else {
    // Mixed precision: FP64 residual r = b - A x (assembled, masked),
    // FP32 PCG for the correction, FP64 update of x, repeated.
    cudaStream_t st = ctx->stream;
    double *r64 = (double *)gf_work(prob, 3, sizeof(double) * n);
    double *ax = (double *)gf_work(prob, 4, sizeof(double) * n);
    float *r32 = (float *)gf_work(prob, 5, sizeof(float) * n);
    float *d32 = (float *)gf_work(prob, 6, sizeof(float) * n);
    if (!r64 || !ax || !r32 || !d32) return gf_fail(ctx, GF_ERR_NOMEM, "work allocation failed");
    const unsigned gel = grid_for(n, 256, ctx->sm_count * 8);
    const double *mask = bbv ? prob->mask_d : nullptr;
    if (bbv) {
      prob->launches++;
      k_cg_lift<double><<<gel, 256, 0, st>>>(n, mask, xb, x);
    }
    // b norm and rtol as the reference (gcg.ipp:290-293)
    prob->scal_h[S_NORMT] = tr->normtype;
    prob->scal_h[S_NTOT] = (double)n;
    prob->scal_h[S_IVOL] = 1.0 / prob->volume;
    GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_d + S_NTOT, prob->scal_h + S_NTOT, sizeof(double) * 3,
                                 cudaMemcpyHostToDevice, st));
    prob->launches++;
    k_norm<<<S.gvec, RED_THREADS, 0, st>>>(n, tr->normtype, b, prob->mass_d, prob->scal_d, 40,
                                           prob->partials, prob->counter);
    GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h + 40, prob->scal_d + 40, sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    GF_CUDA(ctx, cudaStreamSynchronize(st));
    const double bnorm = prob->scal_h[40];
    const double rtol = (tr->relative || bnorm >= 1.0) ? tr->tol * bnorm : tr->tol;
    const int sweeps = tr->max_refine > 0 ? tr->max_refine : 20;
    const double itol = tr->inner_tol > 0 ? tr->inner_tol : 1e-5;
    rc = GF_CG_NOCONVERGE;
    int total = 0;
    for (int sweep = 0; sweep <= sweeps; sweep++) {
      // FP64 residual
      int rr = launch_helm<double>(prob, p, nullptr, q, nullptr, use_mass, x, ax, st);
      if (rr) return gf_fail(ctx, rr, "apply failed");
      prob->launches++;
      k_cg_resid<double><<<gel, 256, 0, st>>>(n, b, ax, r64);
      prob->launches++;
      k_cg_dss<double, false><<<S.gcls, RED_THREADS, 0, st>>>(
          prob->nclass, prob->class_ptr, prob->members, mask, prob->imult_d, ax, r64,
          prob->scal_d, prob->partials, prob->counter);
      prob->launches++;
      k_norm<<<S.gvec, RED_THREADS, 0, st>>>(n, tr->normtype, r64, prob->mass_d, prob->scal_d, 41,
                                             prob->partials, prob->counter);
      GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h + 41, prob->scal_d + 41, sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
      GF_CUDA(ctx, cudaStreamSynchronize(st));
      rn = prob->scal_h[41];
      if (rn <= rtol) {
        rc = GF_OK;
        break;
      }
      if (sweep == sweeps || total >= tr->maxit) break;
      // FP32 correction: A d = r, d0 = 0, to a relative drop itol
      prob->launches++;
      k_convert<float, double><<<gel, 256, 0, st>>>(n, r64, r32);
      cudaMemsetAsync(d32, 0, sizeof(float) * n, st);
      int in_it = 0;
      double in_rn = 0.0;
      // relative drop itol, but no deeper than needed to reach rtol
      const double rel = std::max(itol, 0.5 * rtol / rn);
      // the correction obeys the same Dirichlet mask (zero lift)
      int irc = S.solve<float>(*tr, p, q, use_mass, r32, nullptr, d32, bbv, rel, true,
                               tr->maxit - total, dinv, nullptr, &in_it, &in_rn, 13);
      if (irc < 0) return irc;
      total += in_it;
      // x += d
      prob->launches++;
      k_convert<double, float><<<gel, 256, 0, st>>>(n, d32, ax);
      prob->launches++;
      k_axpby<double><<<gel, 256, 0, st>>>(n, 1.0, ax, 1.0, x);
    }
    if (bbv) {
      prob->launches++;
      k_cg_lift<double><<<gel, 256, 0, st>>>(n, prob->mask_d, xb, x);
    }
    GF_CHECK_LAUNCH(ctx);
    it = total;
    if (rc == GF_CG_NOCONVERGE && rn <= tr->tol) rc = GF_OK;
  }
  if (iters) *iters = it;
  if (final_norm) *final_norm = rn;
  if (residuals && hist && tr->maxit > 0) {
    GF_CUDA(ctx, cudaMemcpyAsync(residuals, hist, sizeof(double) * std::min(it, tr->maxit),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
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

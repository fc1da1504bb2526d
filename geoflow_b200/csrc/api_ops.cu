// api_ops.cu -- operator entry points: Helmholtz, mass, derivatives,
// advection, Burgers RHS, gather-scatter, multiplicity, integral.
#include "gf_common.cuh"
#include "k_dss.cuh"
#include "k_dudt.cuh"
#include "k_tensor.cuh"
#include "k_vec.cuh"
#include "ops_launch.cuh"

using namespace gfk;

namespace gfk {
int g_fp32_apply_mode = GF_FP32_APPLY_FMA;
}

extern "C" int gf_set_fp32_apply(int mode) {
  if (mode != GF_FP32_APPLY_FMA && mode != GF_FP32_APPLY_TF32) return GF_ERR_ARG;
  const int prev = g_fp32_apply_mode;
  g_fp32_apply_mode = mode;
  return prev;
}

// ---------------------------------------------------------------------
// Helmholtz
// ---------------------------------------------------------------------
template <typename T>
int launch_helm(gf_problem *prob, T p, const T *pvec, T q, const T *qvec, int use_mass,
                const T *u, T *uo, cudaStream_t st, const double *stop) {
  return dispatch_n<HelmLaunch<T, LoadE<T>>::template F>(prob->n, prob, p, pvec, q, qvec, use_mass,
                                                         LoadE<T>{u}, uo, st, stop);
}
template int launch_helm<double>(gf_problem *, double, const double *, double, const double *, int,
                                 const double *, double *, cudaStream_t, const double *);
template int launch_helm<float>(gf_problem *, float, const float *, float, const float *, int,
                                const float *, float *, cudaStream_t, const double *);

template <typename T>
int launch_helm_L(gf_problem *prob, T p, T q, int use_mass, const T *wL, T *uo, cudaStream_t st,
                  const double *stop) {
  if (prob->has_box)
    return dispatch_n<HelmLaunch<T, LoadBox<T>>::template F>(
        prob->n, prob, p, (const T *)nullptr, q, (const T *)nullptr, use_mass,
        LoadBox<T>{wL, prob->box}, uo, st, stop);
  return dispatch_n<HelmLaunch<T, LoadCsr<T>>::template F>(
      prob->n, prob, p, (const T *)nullptr, q, (const T *)nullptr, use_mass,
      LoadCsr<T>{wL, prob->node_class}, uo, st, stop);
}
template int launch_helm_L<double>(gf_problem *, double, double, int, const double *, double *,
                                   cudaStream_t, const double *);

int launch_helm_L_f32io(gf_problem *prob, double p, double q, int use_mass, const float *wL,
                        float *uo, cudaStream_t st, const double *stop) {
  if (prob->dim != 3) return GF_ERR_UNSUPPORTED;
  if (prob->has_box)
    return dispatch_n<HelmLaunch<double, LoadBox<float>, float>::template F>(
        prob->n, prob, p, (const double *)nullptr, q, (const double *)nullptr, use_mass,
        LoadBox<float>{wL, prob->box}, uo, st, stop);
  return dispatch_n<HelmLaunch<double, LoadCsr<float>, float>::template F>(
      prob->n, prob, p, (const double *)nullptr, q, (const double *)nullptr, use_mass,
      LoadCsr<float>{wL, prob->node_class}, uo, st, stop);
}
template int launch_helm_L<float>(gf_problem *, float, float, int, const float *, float *,
                                  cudaStream_t, const double *);

extern "C" int gf_helmholtz_apply(gf_problem_t prob, int dtype, double p, const void *p_vec,
                                  double q, const void *q_vec, int use_mass, const void *u,
                                  void *uo) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && uo, "u and uo are required");
  GF_REQUIRE(ctx, dtype == GF_F64 || dtype == GF_F32, "unknown dtype %d", dtype);
  int rc;
  if (dtype == GF_F64)
    rc = launch_helm<double>(prob, p, (const double *)p_vec, q, (const double *)q_vec, use_mass,
                             (const double *)u, (double *)uo, ctx->stream);
  else
    rc = launch_helm<float>(prob, (float)p, (const float *)p_vec, (float)q, (const float *)q_vec,
                            use_mass, (const float *)u, (float *)uo, ctx->stream);
  if (rc != GF_OK) return gf_fail(ctx, rc, "helmholtz launch failed (n=%d)", prob->n);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// H is symmetric element by element (Dk^T (M Gk) Dk with M, Gk diagonal,
// plus q M), so its transpose is the same operator.
extern "C" int gf_helmholtz_apply_T(gf_problem_t prob, int dtype, double p, double q, int use_mass,
                                    const void *u, void *uo) {
  return gf_helmholtz_apply(prob, dtype, p, nullptr, q, nullptr, use_mass, u, uo);
}

// ---------------------------------------------------------------------
// mass
// ---------------------------------------------------------------------
template <typename T>
__global__ void k_mass(int64_t n, int nn, const T *__restrict__ egeom, const T *__restrict__ ngeom,
                       int dim, Basis<T, GF_MAXN> B, int nb, const T *__restrict__ imass,
                       const T *__restrict__ u, T *__restrict__ uo) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (imass) {
      uo[i] = imass[i] * u[i];
    } else {
      int64_t e = i / nn;
      int a = (int)(i % nn);
      int ii = a % nb, jj = (a / nb) % nb, kk = a / (nb * nb);
      T J = egeom ? egeom[e * (dim + 1) + dim] : ngeom[(int64_t)dim * n + i];
      T w = dim == 2 ? B.W[jj] * B.W[ii] : B.W[kk] * B.W[jj] * B.W[ii];
      uo[i] = (w * J) * u[i];
    }
  }
}

extern "C" int gf_mass_apply(gf_problem_t prob, int dtype, int inverse, const void *u, void *uo) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && uo, "u and uo are required");
  int nn = prob->dim == 2 ? prob->n * prob->n : prob->n * prob->n * prob->n;
  unsigned grid = grid_for(prob->nlocal, 256, ctx->sm_count * 8);
  if (dtype == GF_F64) {
    Basis<double, GF_MAXN> B;
    for (int i = 0; i < prob->n; i++) B.W[i] = prob->W[i];
    prob->launches++;
    k_mass<double><<<grid, 256, 0, ctx->stream>>>(prob->nlocal, nn, prob->egeom_d, prob->ngeom_d,
                                                   prob->dim, B, prob->n,
                                                   inverse ? prob->imass_d : nullptr,
                                                   (const double *)u, (double *)uo);
  } else if (dtype == GF_F32) {
    Basis<float, GF_MAXN> B;
    for (int i = 0; i < prob->n; i++) B.W[i] = (float)prob->W[i];
    prob->launches++;
    k_mass<float><<<grid, 256, 0, ctx->stream>>>(prob->nlocal, nn, prob->egeom_f, prob->ngeom_f,
                                                  prob->dim, B, prob->n,
                                                  inverse ? prob->imass_f : nullptr,
                                                  (const float *)u, (float *)uo);
  } else {
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  }
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// ---------------------------------------------------------------------
// reference derivatives
// ---------------------------------------------------------------------
template <typename T>
static int deriv_common(gf_problem *prob, const T *u, int idir, int dotrans, int phys, int accum,
                        T *du) {
  return dispatch_n<DerivLaunch<T>::template F>(prob->n, prob, u, idir, dotrans, phys, accum, du,
                                                prob->ctx->stream);
}

extern "C" int gf_grefderiv(gf_problem_t prob, int dtype, const void *u, int idir, int dotrans,
                            void *du) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && du && idir >= 1 && idir <= prob->dim, "bad arguments");
  int rc = dtype == GF_F64
               ? deriv_common<double>(prob, (const double *)u, idir, dotrans, 0, 0, (double *)du)
               : deriv_common<float>(prob, (const float *)u, idir, dotrans, 0, 0, (float *)du);
  if (rc) return gf_fail(ctx, rc, "grefderiv launch failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_deriv(gf_problem_t prob, int dtype, const void *u, int idir, void *du) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  const int nphys = prob->nxy ? prob->nxy : prob->dim;
  GF_REQUIRE(ctx, u && du && idir >= 1 && idir <= nphys, "bad arguments");
  int rc;
  if (prob->geom >= GF_GEOM_DEFORMED) {  // sum_j dXi_j/dX_idir D_j u
    rc = dtype == GF_F64
             ? dispatch_n<DefLaunch<double, LoadE<double>>::template F>(
                   prob->n, prob, (int)DEF_DERIV, 0.0, (const double *)nullptr, 0.0,
                   (const double *)nullptr, 0, LoadE<double>{(const double *)u}, 0,
                   (const double *const *)nullptr, idir, (double *)du, ctx->stream,
                   (const double *)nullptr)
             : dispatch_n<DefLaunch<float, LoadE<float>>::template F>(
                   prob->n, prob, (int)DEF_DERIV, 0.0f, (const float *)nullptr, 0.0f,
                   (const float *)nullptr, 0, LoadE<float>{(const float *)u}, 0,
                   (const float *const *)nullptr, idir, (float *)du, ctx->stream,
                   (const double *)nullptr);
  } else {
    rc = dtype == GF_F64
             ? deriv_common<double>(prob, (const double *)u, idir, 0, 1, 0, (double *)du)
             : deriv_common<float>(prob, (const float *)u, idir, 0, 1, 0, (float *)du);
  }
  if (rc) return gf_fail(ctx, rc, "deriv launch failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_grefdiv(gf_problem_t prob, int dtype, const void *const *u, int dotrans,
                          void *divu) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && divu, "bad arguments");
  for (int k = 0; k < prob->dim; k++) {
    GF_REQUIRE(ctx, u[k], "component %d missing", k);
    int rc = dtype == GF_F64 ? deriv_common<double>(prob, (const double *)u[k], k + 1, dotrans, 0,
                                                    k > 0, (double *)divu)
                             : deriv_common<float>(prob, (const float *)u[k], k + 1, dotrans, 0,
                                                   k > 0, (float *)divu);
    if (rc) return gf_fail(ctx, rc, "grefdiv launch failed");
  }
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// ---------------------------------------------------------------------
// advection and Burgers RHS
// ---------------------------------------------------------------------
// Deformed / embedded elements: one k_def launch per evolved component,
// the reference gradient shared by advection and diffusion.  f as for
// launch_dudt: ADVECT {p, c0, c1, c2}, BURGERS {u0, u1, u2}, HEAT {u}.
template <typename T>
static int launch_def_dudt(gf_problem *prob, int eqn, int mode, T nu, const T *const *f,
                           T *const *o, cudaStream_t st) {
  const int nv = prob->nxy;
  if (eqn == GF_EQN_ADVECT) {
    const T *c[3] = {f[1], f[2], f[3]};
    return dispatch_n<DefLaunch<T, LoadE<T>>::template F>(
        prob->n, prob, mode == MODE_ADVECT ? (int)DEF_ADVECT : (int)DEF_DUDT, nu, (const T *)nullptr,
        T(0), (const T *)nullptr, 0, LoadE<T>{f[0]}, nv, (const T *const *)c, 0, o[0], st,
        (const double *)nullptr);
  }
  if (eqn == GF_EQN_HEAT)
    return dispatch_n<DefLaunch<T, LoadE<T>>::template F>(
        prob->n, prob, (int)DEF_DUDT, nu, (const T *)nullptr, T(0), (const T *)nullptr, 0,
        LoadE<T>{f[0]}, 0, (const T *const *)nullptr, 0, o[0], st, (const double *)nullptr);
  for (int k = 0; k < nv; k++) {  // Burgers: the velocity is the state
    int rc = dispatch_n<DefLaunch<T, LoadE<T>>::template F>(
        prob->n, prob, (int)DEF_DUDT, nu, (const T *)nullptr, T(0), (const T *)nullptr, 0,
        LoadE<T>{f[k]}, nv, f, 0, o[k], st, (const double *)nullptr);
    if (rc) return rc;
  }
  return GF_OK;
}

template <typename T>
int launch_dudt(gf_problem *prob, int eqn, int mode, T nu, const T *const *f, T *const *o,
                cudaStream_t st, const gfk::RKEpi<T> *epi) {
  if (prob->geom >= GF_GEOM_DEFORMED) {
    if (mode == MODE_EULER) return GF_ERR_UNSUPPORTED;
    return launch_def_dudt<T>(prob, eqn, mode, nu, f, o, st);
  }
  const RKEpi<T> none{};
  return dispatch_n<DudtLaunch<T>::template F>(prob->n, prob, eqn, mode, nu, f, o, st,
                                               epi ? *epi : none);
}
template int launch_dudt<double>(gf_problem *, int, int, double, const double *const *,
                                 double *const *, cudaStream_t, const gfk::RKEpi<double> *);
template int launch_dudt<float>(gf_problem *, int, int, float, const float *const *,
                                float *const *, cudaStream_t, const gfk::RKEpi<float> *);

extern "C" int gf_advect_apply(gf_problem_t prob, int dtype, const void *p, int ncomp,
                               const void *const *c, void *po) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  const int nvel = prob->nxy ? prob->nxy : prob->dim;
  GF_REQUIRE(ctx, p && c && po && ncomp == nvel,
             "advect needs p, %d velocity components (one per physical coordinate), po", nvel);
  for (int k = 0; k < ncomp; k++) GF_REQUIRE(ctx, c[k], "velocity component %d missing", k);
  int rc;
  if (dtype == GF_F64) {
    const double *f[4] = {(const double *)p, (const double *)c[0], (const double *)c[1],
                          ncomp > 2 ? (const double *)c[2] : nullptr};
    double *o[3] = {(double *)po, nullptr, nullptr};
    rc = launch_dudt<double>(prob, GF_EQN_ADVECT, MODE_ADVECT, 1.0, f, o, ctx->stream);
  } else {
    const float *f[4] = {(const float *)p, (const float *)c[0], (const float *)c[1],
                         ncomp > 2 ? (const float *)c[2] : nullptr};
    float *o[3] = {(float *)po, nullptr, nullptr};
    rc = launch_dudt<float>(prob, GF_EQN_ADVECT, MODE_ADVECT, 1.0f, f, o, ctx->stream);
  }
  if (rc) return gf_fail(ctx, rc, "advect launch failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_dudt(gf_problem_t prob, int dtype, int eqn, double nu, int nstate,
                       const void *const *u, const void *const *c, void *const *dudt) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && dudt, "u and dudt are required");
  // velocity components: one per physical coordinate (3 on an embedded surface)
  const int nvel = prob->nxy ? prob->nxy : prob->dim;
  GF_REQUIRE(ctx, eqn == GF_EQN_ADVECT || eqn == GF_EQN_BURGERS || eqn == GF_EQN_HEAT,
             "unknown equation %d", eqn);
  if (eqn == GF_EQN_BURGERS) {
    GF_REQUIRE(ctx, nstate == nvel, "Burgers evolves one component per physical coordinate");
  } else if (eqn == GF_EQN_HEAT) {
    // heat evolves each component independently
    for (int k = 0; k < nstate; k++) {
      const void *uk[1] = {u[k]};
      void *dk[1] = {dudt[k]};
      int rc = dtype == GF_F64
                   ? launch_dudt<double>(prob, GF_EQN_HEAT, MODE_DUDT, nu,
                                         (const double *const *)uk, (double *const *)dk, ctx->stream)
                   : launch_dudt<float>(prob, GF_EQN_HEAT, MODE_DUDT, (float)nu,
                                        (const float *const *)uk, (float *const *)dk, ctx->stream);
      if (rc) return gf_fail(ctx, rc, "dudt launch failed");
    }
    GF_CHECK_LAUNCH(ctx);
    return GF_OK;
  } else {
    GF_REQUIRE(ctx, nstate == 1 && c, "pure advection evolves one component with dim velocities");
  }
  int rc;
  if (dtype == GF_F64) {
    const double *f[4] = {nullptr, nullptr, nullptr, nullptr};
    double *o[3] = {nullptr, nullptr, nullptr};
    if (eqn == GF_EQN_ADVECT) {
      f[0] = (const double *)u[0];
      for (int k = 0; k < nvel; k++) f[1 + k] = (const double *)c[k];
      o[0] = (double *)dudt[0];
    } else {
      for (int k = 0; k < nvel; k++) {
        f[k] = (const double *)u[k];
        o[k] = (double *)dudt[k];
      }
    }
    rc = launch_dudt<double>(prob, eqn, MODE_DUDT, nu, f, o, ctx->stream);
  } else {
    const float *f[4] = {nullptr, nullptr, nullptr, nullptr};
    float *o[3] = {nullptr, nullptr, nullptr};
    if (eqn == GF_EQN_ADVECT) {
      f[0] = (const float *)u[0];
      for (int k = 0; k < nvel; k++) f[1 + k] = (const float *)c[k];
      o[0] = (float *)dudt[0];
    } else {
      for (int k = 0; k < nvel; k++) {
        f[k] = (const float *)u[k];
        o[k] = (float *)dudt[k];
      }
    }
    rc = launch_dudt<float>(prob, eqn, MODE_DUDT, (float)nu, f, o, ctx->stream);
  }
  if (rc) return gf_fail(ctx, rc, "dudt launch failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// ---------------------------------------------------------------------
// gather-scatter
// ---------------------------------------------------------------------
template <typename T>
int launch_dss(gf_problem *prob, int op, T *u, cudaStream_t st) {
  unsigned grid = grid_for(prob->nclass, 256, prob->ctx->sm_count * 16);
  BoxWalk w;
  if (dss_box_walk(prob, w)) {  // lattice classes: no index arrays
    prob->launches++;
    switch (op) {
      case GF_DSS_SUM: k_dss_box<T, GF_DSS_SUM><<<grid, 256, 0, st>>>(u, w); break;
      case GF_DSS_SMOOTH: k_dss_box<T, GF_DSS_SMOOTH><<<grid, 256, 0, st>>>(u, w); break;
      case GF_DSS_MAX: k_dss_box<T, GF_DSS_MAX><<<grid, 256, 0, st>>>(u, w); break;
      case GF_DSS_MIN: k_dss_box<T, GF_DSS_MIN><<<grid, 256, 0, st>>>(u, w); break;
      default: prob->launches--; return GF_ERR_ARG;
    }
    return GF_OK;
  }
  const SplitCls sc = split_of(prob);
  grid = grid_for(sc.n + sc.nsh, 256, prob->ctx->sm_count * 16);
  prob->launches++;
  switch (op) {
    case GF_DSS_SUM: k_dss_split<T, GF_DSS_SUM><<<grid, 256, 0, st>>>(u, sc); break;
    case GF_DSS_SMOOTH: k_dss_split<T, GF_DSS_SMOOTH><<<grid, 256, 0, st>>>(u, sc); break;
    case GF_DSS_MAX: k_dss_split<T, GF_DSS_MAX><<<grid, 256, 0, st>>>(u, sc); break;
    case GF_DSS_MIN: k_dss_split<T, GF_DSS_MIN><<<grid, 256, 0, st>>>(u, sc); break;
    default: prob->launches--; return GF_ERR_ARG;
  }
  return GF_OK;
}
template int launch_dss<double>(gf_problem *, int, double *, cudaStream_t);
template int launch_dss<float>(gf_problem *, int, float *, cudaStream_t);

extern "C" int gf_dss(gf_problem_t prob, int dtype, int op, void *u) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u, "u is required");
  int rc = dtype == GF_F64 ? launch_dss<double>(prob, op, (double *)u, ctx->stream)
                           : (dtype == GF_F32 ? launch_dss<float>(prob, op, (float *)u, ctx->stream)
                                              : GF_ERR_ARG);
  if (rc) return gf_fail(ctx, rc, "bad dss op %d or dtype %d", op, dtype);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// Sum and Smooth give every member of a class the same combination with
// one weight (1 or 1/|class|), so the map is symmetric: its transpose is
// itself.
extern "C" int gf_dss_T(gf_problem_t prob, int dtype, int op, void *u) {
  if (!prob) return GF_ERR_ARG;
  GF_REQUIRE(prob->ctx, op == GF_DSS_SUM || op == GF_DSS_SMOOTH,
             "only the linear reductions Sum and Smooth have a transpose");
  return gf_dss(prob, dtype, op, u);
}

__global__ void k_mult(int64_t n, const double *__restrict__ imult, int inverse,
                       double *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = inverse ? imult[i] : 1.0 / imult[i];
}

extern "C" int gf_mult(gf_problem_t prob, int inverse, double *mult) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, mult, "mult is required");
  prob->launches++;
  k_mult<<<grid_for(prob->nlocal, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(
      prob->nlocal, prob->imult_d, inverse, mult);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_integrate(gf_problem_t prob, int dtype, const void *u, double *result) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, u && result, "u and result are required");
  unsigned grid = grid_for(prob->nlocal, RED_THREADS, prob->npartials);
  double *out = prob->scal_d + 63;
  prob->launches++;
  if (dtype == GF_F64)
    k_integrate<double><<<grid, RED_THREADS, 0, ctx->stream>>>(
        prob->nlocal, prob->mass_d, (const double *)u, prob->partials, prob->counter, out);
  else
    k_integrate<float><<<grid, RED_THREADS, 0, ctx->stream>>>(
        prob->nlocal, prob->mass_d, (const float *)u, prob->partials, prob->counter, out);
  GF_CHECK_LAUNCH(ctx);
  GF_CUDA(ctx, cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

// ---------------------------------------------------------------------
// GMTK::constrain2sphere (2) (blas/gmtk.ipp:2957-2976)
// ---------------------------------------------------------------------
extern "C" int gf_constrain2sphere(gf_problem_t prob, int dtype, void *const *v,
                                   const void *const *xyz) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, v && xyz, "v and xyz are required");
  for (int k = 0; k < 3; k++) GF_REQUIRE(ctx, v[k] && xyz[k], "component %d missing", k);
  GF_REQUIRE(ctx, dtype == GF_F64 || dtype == GF_F32, "unknown dtype %d", dtype);
  if (prob->geom != GF_GEOM_EMBEDDED) return GF_OK;  // as the reference: only on 2-d surfaces
  const unsigned g = grid_for(prob->nlocal, 256, ctx->sm_count * 8);
  prob->launches++;
  if (dtype == GF_F64)
    k_constrain2sphere<double><<<g, 256, 0, ctx->stream>>>(
        prob->nlocal, (double *)v[0], (double *)v[1], (double *)v[2], (const double *)xyz[0],
        (const double *)xyz[1], (const double *)xyz[2]);
  else
    k_constrain2sphere<float><<<g, 256, 0, ctx->stream>>>(
        prob->nlocal, (float *)v[0], (float *)v[1], (float *)v[2], (const float *)xyz[0],
        (const float *)xyz[1], (const float *)xyz[2]);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

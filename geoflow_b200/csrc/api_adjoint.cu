// api_adjoint.cu -- adjoint (vector-Jacobian) path: VJP of the Burgers
// right-hand side, of one RK step, and the checkpointed gradient of a
// final-time misfit.  The reference has no adjoint; these entry points are
// new.
#include "gf_common.cuh"
#include "rk_common.cuh"

extern "C" int gf_dudt_vjp(gf_problem_t prob, int dtype, int eqn, double nu, int nstate,
                           const void *const *u, const void *const *c, const void *const *lam,
                           void *const *ubar) {
  if (!prob) return GF_ERR_ARG;
  (void)dtype; (void)eqn; (void)nu; (void)nstate; (void)u; (void)c; (void)lam; (void)ubar;
  return gf_fail(prob->ctx, GF_ERR_UNSUPPORTED, "gf_dudt_vjp: not built yet");
}

extern "C" int gf_rk_step_vjp(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                              const void *const *u0, const void *const *c, double dt,
                              void *const *lam) {
  if (!prob) return GF_ERR_ARG;
  (void)dtype; (void)traits; (void)u0; (void)c; (void)dt; (void)lam;
  return gf_fail(prob->ctx, GF_ERR_UNSUPPORTED, "gf_rk_step_vjp: not built yet");
}

extern "C" int gf_adjoint_gradient(gf_problem_t prob, const gf_rk_traits *traits,
                                   const double *const *u0, const double *const *c,
                                   const double *const *u_obs, double dt, int nsteps,
                                   int checkpoint_every, double *J, double *const *grad) {
  if (!prob) return GF_ERR_ARG;
  (void)traits; (void)u0; (void)c; (void)u_obs; (void)dt; (void)nsteps; (void)checkpoint_every;
  (void)J; (void)grad;
  return gf_fail(prob->ctx, GF_ERR_UNSUPPORTED, "gf_adjoint_gradient: not built yet");
}

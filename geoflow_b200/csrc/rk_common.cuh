// rk_common.cuh -- the device-side RK stepper object shared by the
// forward stepper (api_rk.cu) and its adjoint (api_adjoint.cu).
#pragma once
#include "gf_common.cuh"

namespace gfrk {

void butcher(int order, double *alpha, double beta[4][4], double *c);
// the coefficient planes of the advection fast path (k_def.cuh
// adv_coef_point) of a 2-d deformed or embedded problem, velocity c[nxy]
template <typename T>
int adv_coef_launch(gf_problem *prob, const T *const *c, T *b0, T *b1, cudaStream_t st);
int check_traits(gf_problem *prob, const gf_rk_traits *tr, const void *const *u,
                 const void *const *c);

template <typename T>
struct Stepper {
  gf_problem *prob;
  cudaStream_t st;
  int64_t n;
  int eqn, nstate, scheme;
  T nu;
  const T *c[3] = {nullptr, nullptr, nullptr};
  T *uold[3] = {nullptr, nullptr, nullptr};
  T *utmp[3] = {nullptr, nullptr, nullptr};
  T *K[3][3] = {{nullptr}};
  // advection fast path (prescribed velocity, nu = 0, 2-d deformed or
  // embedded): coefficient planes b_0, b_1 of adv_element, or null
  T *advb[2] = {nullptr, nullptr};
  T *advbuf[2] = {nullptr, nullptr};  // their storage (alloc), unused until prepare_adv
  bool adv_ok() const;

  Stepper(gf_problem *p, const gf_rk_traits *tr, const void *const *cv)
      : prob(p), st(p->ctx->stream), n(p->nlocal), eqn(tr->eqn), nstate(tr->nstate),
        scheme(tr->scheme), nu((T)tr->nu) {
    if (cv)
      for (int k = 0; k < gf_nvel(p); k++) c[k] = (const T *)cv[k];
  }
  bool alloc();
  // forms the fast path's coefficients when the problem and equation allow
  // it (k_def.cuh adv_coef_point); returns false when they do not
  bool prepare_adv();
  int rhs(T *const *u, T *const *Kout);
  // x = the SSP substep update of dudt(u) before its Smooth (the RHS
  // kernel's MODE_EULER epilogue; 3-d non-deformed problems), then Smooth;
  // false when the problem takes the separate RHS and update passes
  bool rhs_euler_smooth(T *const *u, T *const *x, T dt, T *const *uin, T a, T *const *y, T b,
                        T a2, T *const *y2, T b2, int *rc);
  void smooth(T *v);
  // GMTK::constrain2sphere on the state where step_b calls it, on embedded
  // surfaces with node coordinates and a state of >= 3 components
  void constrain(T *const *u);
  // Smooth fused with the stage update before or after it
  void euler_smooth(T *x, T dt, const T *uin, T a, const T *y, T b, T a2, const T *y2, T b2);
  void smooth_accum(T *K, T ch, T *uout);
  void accum_smooth(T *uout, const T *K, T ch);
  // the same on every state component (arrays of nstate pointers; y and y2
  // may be null): one pass over the lattice on box problems
  void smooth_n(T *const *v);
  void euler_smooth_n(T *const *x, T dt, T *const *uin, T a, T *const *y, T b, T a2,
                      T *const *y2, T b2);
  void smooth_accum_n(T *const *K, T ch, T *const *uout);
  void accum_smooth_n(T *const *uout, T *const *K, T ch);
  // One step uin -> uout.  With a tape (pointers tape[3*m + k], m = 0 ..
  // stages-1), stage m's input state (the argument of its RHS call) is left
  // in tape[3*m + k] for the adjoint sweep.
  int step(T *const *uin, T *const *uout, T dt, T *const *tape = nullptr);
  int step_ssp(T *const *uin, T *const *uout, T dt);
  int stages() const { return scheme <= 4 ? scheme : (scheme == GF_SSP22 ? 2 : (scheme == GF_SSP33 ? 3 : 4)); }
};

}  // namespace gfrk

// rk_common.cuh -- the device-side RK stepper object shared by the
// forward stepper (api_rk.cu) and its adjoint (api_adjoint.cu).
#pragma once
#include "gf_common.cuh"

namespace gfrk {

void butcher(int order, double *alpha, double beta[4][4], double *c);
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

  Stepper(gf_problem *p, const gf_rk_traits *tr, const void *const *cv)
      : prob(p), st(p->ctx->stream), n(p->nlocal), eqn(tr->eqn), nstate(tr->nstate),
        scheme(tr->scheme), nu((T)tr->nu) {
    if (cv)
      for (int k = 0; k < p->dim; k++) c[k] = (const T *)cv[k];
  }
  bool alloc();
  int rhs(T *const *u, T *const *Kout);
  void smooth(T *v);
  int step(T *const *uin, T *const *uout, T dt);
};

}  // namespace gfrk

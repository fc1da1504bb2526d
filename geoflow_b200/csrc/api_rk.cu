// api_rk.cu -- explicit Runge-Kutta steps of GExRKStepper
// (pdes/gexrk_stepper.ipp) on the GBurgers right-hand side, with the DSS
// Smooth calls exactly where the reference places them:
//   Butcher step_b (1)  (gexrk_stepper.ipp:252-341), tableau of
//                       GButcherRK::computeCoeffs (gbutcherrk.ipp:69-125)
//   SSP22 / SSP33 / SSP34 (gexrk_stepper.ipp:533-780), step_euler (809-819)
// and GBurgers::step_impl (gburgers.ipp:275-333): uold = u; step(uold -> u).
//
// Per stage: one fused element kernel for the RHS (k_dudt*), one class
// kernel for Smooth, and elementwise stage combinations.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gf_common.cuh"
#include "k_dss.cuh"
#include "k_vec.cuh"
#include "ops_launch.cuh"
#include "rk_common.cuh"

using namespace gfk;

namespace gfrk {

// slot of the problem's scalar block holding the RK non-finite flag
constexpr int RK_FLAG_SLOT = 62;

void butcher(int order, double *alpha, double beta[4][4], double *c) {
  std::memset(beta, 0, sizeof(double) * 16);
  for (int i = 0; i < 4; i++) alpha[i] = c[i] = 0.0;
  if (order == 1) {
    c[0] = 1.0;
  } else if (order == 2) {
    c[0] = 0.5;
    alpha[1] = 1.0;
    c[1] = 0.5;
    beta[1][0] = 1.0;
  } else if (order == 3) {
    c[0] = 0.25;
    alpha[1] = 1.0 / 3.0;
    c[1] = 0.0;
    alpha[2] = 2.0 / 3.0;
    c[2] = 0.75;
    beta[1][0] = 1.0 / 3.0;
    beta[2][1] = 2.0 / 3.0;
  } else {
    c[0] = 1.0 / 6.0;
    alpha[1] = 0.5;
    c[1] = 1.0 / 3.0;
    alpha[2] = 0.5;
    c[2] = 1.0 / 3.0;
    alpha[3] = 1.0;
    c[3] = 1.0 / 6.0;
    beta[1][0] = 0.5;
    beta[2][1] = 0.5;
    beta[3][2] = 1.0;
  }
}

// y = uin + ((0 + b0 K0) + b1 K1 + ...)   (isum accumulation of step_b)
template <typename T>
__global__ void k_stage_sum(int64_t n, const T *__restrict__ uin, int nk, const T *__restrict__ K0,
                            const T *__restrict__ K1, const T *__restrict__ K2, T b0, T b1, T b2,
                            T *__restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = rk_stage_point(uin[i], nk, K0, K1, K2, b0, b1, b2, i);
}

// flag[0] = 1 when any of the nstate fields holds a non-finite value
// (GBurgers::step_impl asserts isfinite on the evolved state after every
// step, gburgers.ipp:325-331).  Only a bad value writes the flag.
template <typename T>
__global__ void k_nonfinite(int64_t n, int nstate, const T *__restrict__ u0,
                            const T *__restrict__ u1, const T *__restrict__ u2,
                            double *__restrict__ flag) {
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    bad |= !isfinite(u0[i]);
    if (nstate > 1) bad |= !isfinite(u1[i]);
    if (nstate > 2) bad |= !isfinite(u2[i]);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) flag[0] = 1.0;
}

template <typename T>
struct AdvLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, const T *u, const T *b0, const T *b1, T *out,
                   cudaStream_t st) {
      const Basis<T, N> B = make_basis<T, N>(prob);
      prob->launches++;
      k_adv_def<T, N, LoadE<T>><<<(unsigned)((prob->ne + 3) / 4), 128, 0, st>>>(
          B, prob->ne, LoadE<T>{u}, b0, b1, out);
      return GF_OK;
    }
  };
};

template <typename T>
struct AdvCoefLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, const T *const *c, T *b0, T *b1, cudaStream_t st) {
      const Basis<T, N> B = make_basis<T, N>(prob);
      prob->launches++;
      k_adv_coef<T, N><<<grid_for(prob->nlocal, 256, prob->ctx->sm_count * 8), 256, 0, st>>>(
          B, def_of<T>(prob), c[0], c[1], c[2], imass_of<T>(prob), b0, b1);
      return GF_OK;
    }
  };
};

template <typename T>
int adv_coef_launch(gf_problem *prob, const T *const *c, T *b0, T *b1, cudaStream_t st) {
  return dispatch_n<AdvCoefLaunch<T>::template F>(prob->n, prob, c, b0, b1, st);
}
template int adv_coef_launch<double>(gf_problem *, const double *const *, double *, double *,
                                     cudaStream_t);
template int adv_coef_launch<float>(gf_problem *, const float *const *, float *, float *,
                                    cudaStream_t);

template <typename T>
bool Stepper<T>::adv_ok() const {
  if (eqn != GF_EQN_ADVECT || nu != T(0) || prob->geom < GF_GEOM_DEFORMED || prob->dim != 2)
    return false;
  for (int k = 0; k < gf_nvel(prob); k++)
    if (!c[k]) return false;
  return true;
}

template <typename T>
bool Stepper<T>::prepare_adv() {
  advb[0] = advb[1] = nullptr;
  if (!adv_ok() || !advbuf[0] || !advbuf[1]) return false;
  const T *cc[3] = {c[0], c[1], gf_nvel(prob) > 2 ? c[2] : nullptr};
  if (adv_coef_launch<T>(prob, cc, advbuf[0], advbuf[1], st)) return false;
  advb[0] = advbuf[0];
  advb[1] = advbuf[1];
  return true;
}

template <typename T>
int Stepper<T>::rhs(T *const *u, T *const *K) {
  const T *f[4] = {nullptr, nullptr, nullptr, nullptr};
  T *o[3] = {nullptr, nullptr, nullptr};
  if (eqn == GF_EQN_ADVECT && advb[0])
    return dispatch_n<AdvLaunch<T>::template F>(prob->n, prob, (const T *)u[0],
                                                (const T *)advb[0], (const T *)advb[1], K[0], st);
  if (eqn == GF_EQN_ADVECT) {
    f[0] = u[0];
    for (int k = 0; k < gf_nvel(prob); k++) f[1 + k] = c[k];
    o[0] = K[0];
    return launch_dudt<T>(prob, eqn, 0, nu, f, o, st);
  }
  if (eqn == GF_EQN_HEAT) {
    for (int k = 0; k < nstate; k++) {
      const T *fk[4] = {u[k], nullptr, nullptr, nullptr};
      T *ok[3] = {K[k], nullptr, nullptr};
      int rc = launch_dudt<T>(prob, eqn, 0, nu, fk, ok, st);
      if (rc) return rc;
    }
    return GF_OK;
  }
  for (int k = 0; k < gf_nvel(prob); k++) {
    f[k] = u[k];
    o[k] = K[k];
  }
  return launch_dudt<T>(prob, eqn, 0, nu, f, o, st);
}

template <typename T>
bool Stepper<T>::rhs_euler_smooth(T *const *u, T *const *x, T dt, T *const *uin, T a,
                                  T *const *y, T b, T a2, T *const *y2, T b2, int *rc) {
  // FP32 only: measured on B200 (64^3 p=5 SSP-RK3 Burgers), the fused
  // epilogue takes an FP32 stage from 1.96 to 1.75 ms but an FP64 one from
  // 3.28 to 3.59 ms (the FP64 RHS kernel, at 104-109 registers and 3 blocks
  // per SM, absorbs the extra loads badly)
  if (sizeof(T) != 4 || prob->dim != 3 || prob->geom >= GF_GEOM_DEFORMED) return false;
  auto epi_for = [&](int k0, int nk) {
    RKEpi<T> e{};
    for (int j = 0; j < nk; j++) {
      e.uin[j] = uin[k0 + j];
      e.y[j] = y ? y[k0 + j] : nullptr;
      e.y2[j] = y2 ? y2[k0 + j] : nullptr;
    }
    e.dt = dt;
    e.a = a;
    e.b = b;
    e.a2 = a2;
    e.b2 = b2;
    e.uin_is_u = 1;
    for (int j = 0; j < nk; j++)
      if (uin[k0 + j] != u[k0 + j]) e.uin_is_u = 0;
    return e;
  };
  const T *f[4] = {nullptr, nullptr, nullptr, nullptr};
  T *o[3] = {nullptr, nullptr, nullptr};
  if (eqn == GF_EQN_HEAT) {
    for (int k = 0; k < nstate; k++) {
      const T *fk[4] = {u[k], nullptr, nullptr, nullptr};
      T *ok[3] = {x[k], nullptr, nullptr};
      const RKEpi<T> e = epi_for(k, 1);
      if ((*rc = launch_dudt<T>(prob, eqn, MODE_EULER, nu, fk, ok, st, &e))) return true;
    }
  } else {
    if (eqn == GF_EQN_ADVECT) {
      f[0] = u[0];
      for (int k = 0; k < gf_nvel(prob); k++) f[1 + k] = c[k];
      o[0] = x[0];
    } else {
      for (int k = 0; k < gf_nvel(prob); k++) {
        f[k] = u[k];
        o[k] = x[k];
      }
    }
    const RKEpi<T> e = epi_for(0, nstate);
    if ((*rc = launch_dudt<T>(prob, eqn, MODE_EULER, nu, f, o, st, &e))) return true;
  }
  smooth_n(x);
  *rc = GF_OK;
  return true;
}

template <typename T>
void Stepper<T>::smooth(T *v) {
  launch_dss<T>(prob, GF_DSS_SMOOTH, v, st);
}

// gather-scatter Smooth fused with the stage update around it, one
// component, CSR members (k_dss.cuh); box problems take the *_n forms below
template <typename T>
void Stepper<T>::euler_smooth(T *x, T dt, const T *uin, T a, const T *y, T b, T a2, const T *y2,
                              T b2) {
  prob->launches++;
  const SplitCls sc = split_of(prob);
  k_dss_rk_split<T, FUSE_EULER><<<grid_for(sc.n + sc.nsh, 256, prob->ctx->sm_count * 16), 256, 0,
                                  st>>>(x, sc, dt, uin, a, y, b, a2, y2, b2, nullptr, nullptr, T(0));
}

template <typename T>
void Stepper<T>::smooth_accum(T *K, T ch, T *uout) {
  prob->launches++;
  const SplitCls sc = split_of(prob);
  k_dss_rk_split<T, FUSE_ACCUM_AFTER><<<grid_for(sc.n + sc.nsh, 256, prob->ctx->sm_count * 16), 256,
                                        0, st>>>(K, sc, T(0), nullptr, T(0), nullptr, T(0), T(0),
                                                 nullptr, T(0), uout, nullptr, ch);
}

template <typename T>
void Stepper<T>::accum_smooth(T *uout, const T *K, T ch) {
  prob->launches++;
  const SplitCls sc = split_of(prob);
  k_dss_rk_split<T, FUSE_ACCUM_BEFORE><<<grid_for(sc.n + sc.nsh, 256, prob->ctx->sm_count * 16),
                                         256, 0, st>>>(uout, sc, T(0), nullptr, T(0), nullptr, T(0),
                                                       T(0), nullptr, T(0), nullptr, K, ch);
}

// Launch k_dss_rk_box_n / k_dss_smooth_box_n for nstate components; false
// when the problem takes the per-component CSR kernels.
template <typename T, int MODE>
static bool launch_rk_n(gf_problem *prob, cudaStream_t st, int nstate, const RKComps<T> &pc,
                        T dt, T a, T b, T a2, T b2, T ch, bool plain) {
  BoxWalk w;
  if (!dss_box_walk(prob, w) || nstate < 1 || nstate > 3) return false;
  const unsigned grid = grid_for(prob->nclass, 256, prob->ctx->sm_count * 16);
  prob->launches++;
  if (plain) {
    if (nstate == 1) k_dss_smooth_box_n<T, 1><<<grid, 256, 0, st>>>(pc, w);
    else if (nstate == 2) k_dss_smooth_box_n<T, 2><<<grid, 256, 0, st>>>(pc, w);
    else k_dss_smooth_box_n<T, 3><<<grid, 256, 0, st>>>(pc, w);
  } else {
    if (nstate == 1) k_dss_rk_box_n<T, MODE, 1><<<grid, 256, 0, st>>>(pc, w, dt, a, b, a2, b2, ch);
    else if (nstate == 2) k_dss_rk_box_n<T, MODE, 2><<<grid, 256, 0, st>>>(pc, w, dt, a, b, a2, b2, ch);
    else k_dss_rk_box_n<T, MODE, 3><<<grid, 256, 0, st>>>(pc, w, dt, a, b, a2, b2, ch);
  }
  return true;
}

template <typename T>
static RKComps<T> comps(int nstate, T *const *x, T *const *uin, T *const *y, T *const *y2,
                        T *const *K, T *const *acc) {
  RKComps<T> pc{};
  for (int k = 0; k < nstate && k < 3; k++) {
    pc.x[k] = x[k];
    pc.uin[k] = uin ? uin[k] : nullptr;
    pc.y[k] = y ? y[k] : nullptr;
    pc.y2[k] = y2 ? y2[k] : nullptr;
    pc.K[k] = K ? K[k] : nullptr;
    pc.acc[k] = acc ? acc[k] : nullptr;
  }
  return pc;
}

template <typename T>
void Stepper<T>::smooth_n(T *const *v) {
  if (launch_rk_n<T, FUSE_EULER>(prob, st, nstate,
                                 comps<T>(nstate, v, nullptr, nullptr, nullptr, nullptr, nullptr),
                                 T(0), T(0), T(0), T(0), T(0), T(0), true))
    return;
  for (int k = 0; k < nstate; k++) smooth(v[k]);
}

template <typename T>
void Stepper<T>::euler_smooth_n(T *const *x, T dt, T *const *uin, T a, T *const *y, T b, T a2,
                                T *const *y2, T b2) {
  if (launch_rk_n<T, FUSE_EULER>(prob, st, nstate,
                                 comps<T>(nstate, x, uin, y, y2, nullptr, nullptr), dt, a, b, a2,
                                 b2, T(0), false))
    return;
  for (int k = 0; k < nstate; k++)
    euler_smooth(x[k], dt, uin[k], a, y ? y[k] : nullptr, b, a2, y2 ? y2[k] : nullptr, b2);
}

template <typename T>
void Stepper<T>::smooth_accum_n(T *const *Kv, T ch, T *const *uout) {
  if (launch_rk_n<T, FUSE_ACCUM_AFTER>(
          prob, st, nstate, comps<T>(nstate, Kv, nullptr, nullptr, nullptr, nullptr, uout), T(0),
          T(0), T(0), T(0), T(0), ch, false))
    return;
  for (int k = 0; k < nstate; k++) smooth_accum(Kv[k], ch, uout[k]);
}

template <typename T>
void Stepper<T>::accum_smooth_n(T *const *uout, T *const *Kv, T ch) {
  if (launch_rk_n<T, FUSE_ACCUM_BEFORE>(
          prob, st, nstate, comps<T>(nstate, uout, nullptr, nullptr, nullptr, Kv, nullptr), T(0),
          T(0), T(0), T(0), T(0), ch, false))
    return;
  for (int k = 0; k < nstate; k++) accum_smooth(uout[k], Kv[k], ch);
}

template <typename T>
void Stepper<T>::constrain(T *const *u) {
  if (prob->geom != GF_GEOM_EMBEDDED || nstate < 3 || !prob->xyz_d) return;
  const T *x = sizeof(T) == 8 ? (const T *)prob->xyz_d : (const T *)prob->xyz_f;
  const unsigned g = grid_for(n, 256, prob->ctx->sm_count * 8);
  prob->launches++;
  k_constrain2sphere<T><<<g, 256, 0, st>>>(n, u[0], u[1], u[2], x, x + n, x + 2 * n);
}

template <typename T>
bool Stepper<T>::alloc() {
  const size_t bytes = sizeof(T) * n;
  int slot = 30 + (sizeof(T) == 8 ? 0 : 20);
  for (int k = 0; k < nstate; k++) {
    uold[k] = (T *)gf_work(prob, slot++, bytes);
    utmp[k] = (T *)gf_work(prob, slot++, bytes);
    for (int j = 0; j < 3; j++) K[j][k] = (T *)gf_work(prob, slot++, bytes);
    if (!uold[k] || !utmp[k] || !K[0][k] || !K[1][k] || !K[2][k]) return false;
  }
  if (adv_ok()) {
    const int s2 = sizeof(T) == 8 ? 70 : 72;
    advbuf[0] = (T *)gf_work(prob, s2, bytes);
    advbuf[1] = (T *)gf_work(prob, s2 + 1, bytes);
    if (!advbuf[0] || !advbuf[1]) return false;
  }
  return true;
}

// One step uin -> uout (uout may not alias uin).
template <typename T>
int Stepper<T>::step(T *const *uin, T *const *uout, T dt, T *const *tape) {
  const unsigned g = grid_for(n, 256, prob->ctx->sm_count * 8);
  int rc;
  if (scheme >= 1 && scheme <= 4) {
    double alpha[4], beta[4][4], cc[4];
    butcher(scheme, alpha, beta, cc);
    const int ns = scheme;
    const T h = dt;
    // stage inputs go to the tape when one is given
    auto stage_in = [&](int m) { return tape ? tape + 3 * m : (T *const *)utmp; };
    for (int k = 0; k < nstate; k++)
      cudaMemcpyAsync(uout[k], uin[k], sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
    for (int m = 0; m < ns - 1; m++) {
      T *const *um = stage_in(m);
      for (int k = 0; k < nstate; k++) {
        prob->launches++;
        k_stage_sum<T><<<g, 256, 0, st>>>(n, uin[k], m, K[0][k], K[1][k], K[2][k],
                                          (T)beta[m][0] * h, (T)beta[m][1] * h,
                                          (T)beta[m][2] * h, um[k]);
      }
      constrain(um);
      if ((rc = rhs(um, K[m]))) return rc;
      smooth_accum_n(K[m], (T)cc[m] * h, uout);
      constrain(uout);
    }
    T *const *uf = stage_in(ns - 1);
    for (int k = 0; k < nstate; k++) {
      prob->launches++;
      k_stage_sum<T><<<g, 256, 0, st>>>(n, uin[k], ns - 1, K[0][k], K[1][k], K[2][k],
                                        (T)beta[ns - 1][0] * h, (T)beta[ns - 1][1] * h,
                                        (T)beta[ns - 1][2] * h, uf[k]);
    }
    smooth_n(uf);
    constrain(uf);
    // the final stage result goes to the last K slot (K[0] in the
    // reference, whose earlier content is no longer needed)
    T *const *Kf = K[0];
    if ((rc = rhs(uf, Kf))) return rc;
    smooth_n(Kf);
    accum_smooth_n(uout, Kf, (T)cc[ns - 1] * h);
    constrain(uout);
    return GF_OK;
  }
  // SSP stage inputs are uin and the substep results left in K[0..ns-2]
  if (tape) {
    if ((rc = step_ssp(uin, uout, dt))) return rc;
    for (int k = 0; k < nstate; k++) {
      cudaMemcpyAsync(tape[k], uin[k], sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
      for (int m = 1; m < stages(); m++)
        cudaMemcpyAsync(tape[3 * m + k], K[m - 1][k], sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
    }
    return GF_OK;
  }
  return step_ssp(uin, uout, dt);
}

// One SSP substep: x = Smooth(update(dudt(u))), as the RHS call followed by
// euler_smooth_n, or in two passes (the RHS kernel writing the update,
// then the Smooth) where the RHS kernel has the fused epilogue.
template <typename T>
static int ssp_substep(Stepper<T> &S, T *const *u, T *const *x, T dt, T *const *uin, T a,
                       T *const *y, T b, T a2, T *const *y2, T b2) {
  int rc = GF_OK;
  if (S.rhs_euler_smooth(u, x, dt, uin, a, y, b, a2, y2, b2, &rc)) return rc;
  if ((rc = S.rhs(u, x))) return rc;
  S.euler_smooth_n(x, dt, uin, a, y, b, a2, y2, b2);
  return GF_OK;
}

template <typename T>
int Stepper<T>::step_ssp(T *const *uin, T *const *uout, T dt) {
  int rc;
  const T one = T(1);
  if (scheme == GF_SSP22) {
    if ((rc = ssp_substep<T>(*this, uin, K[0], dt, uin, one, nullptr, T(0), one, nullptr, T(0))))
      return rc;
    return ssp_substep<T>(*this, K[0], uout, dt, K[0], T(0.5), uin, T(0.5), one, nullptr, T(0));
  }
  if (scheme == GF_SSP33) {
    if ((rc = ssp_substep<T>(*this, uin, K[0], dt, uin, one, nullptr, T(0), one, nullptr, T(0))))
      return rc;
    if ((rc = ssp_substep<T>(*this, K[0], K[1], dt, K[0], T(0.25), uin, T(0.75), one, nullptr,
                             T(0))))
      return rc;
    return ssp_substep<T>(*this, K[1], uout, dt, K[1], T(2.0 / 3.0), uin, T(1.0 / 3.0), one,
                          nullptr, T(0));
  }
  if (scheme == GF_SSP34) {
    if ((rc = ssp_substep<T>(*this, uin, K[0], dt, uin, T(0.5), uin, T(0.5), one, nullptr, T(0))))
      return rc;
    if ((rc = ssp_substep<T>(*this, K[0], K[1], dt, K[0], T(0.5), K[0], T(0.5), one, nullptr,
                             T(0))))
      return rc;
    if ((rc = ssp_substep<T>(*this, K[1], K[2], dt, K[1], T(1.0 / 6.0), K[1], T(1.0 / 6.0), one,
                             uin, T(2.0 / 3.0))))
      return rc;
    return ssp_substep<T>(*this, K[2], uout, dt, K[2], T(0.5), K[2], T(0.5), one, nullptr, T(0));
  }
  return GF_ERR_ARG;
}

template struct Stepper<double>;
template struct Stepper<float>;

int check_traits(gf_problem *prob, const gf_rk_traits *tr, const void *const *u, const void *const *c) {
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, tr && u, "traits and u are required");
  GF_REQUIRE(ctx, tr->eqn == GF_EQN_ADVECT || tr->eqn == GF_EQN_BURGERS || tr->eqn == GF_EQN_HEAT,
             "unknown equation %d", tr->eqn);
  const int s = tr->scheme;
  GF_REQUIRE(ctx, (s >= 1 && s <= 4) || s == GF_SSP22 || s == GF_SSP33 || s == GF_SSP34,
             "unknown RK scheme %d", s);
  if (tr->eqn == GF_EQN_BURGERS)
    GF_REQUIRE(ctx, tr->nstate == gf_nvel(prob),
               "Burgers evolves one component per physical coordinate");
  else if (tr->eqn == GF_EQN_ADVECT)
    GF_REQUIRE(ctx, tr->nstate == 1 && c, "pure advection: one component and dim velocities");
  else
    GF_REQUIRE(ctx, tr->nstate >= 1 && tr->nstate <= 3, "heat: 1..3 components");
  for (int k = 0; k < tr->nstate; k++) GF_REQUIRE(ctx, u[k], "state component %d missing", k);
  if (tr->eqn == GF_EQN_ADVECT)
    for (int k = 0; k < gf_nvel(prob); k++) GF_REQUIRE(ctx, c[k], "velocity component %d missing", k);
  return GF_OK;
}

template <typename T>
int advance(gf_problem *prob, const gf_rk_traits *tr, void *const *u, const void *const *c,
            double dt, int nsteps) {
  gf_context *ctx = prob->ctx;
  Stepper<T> S(prob, tr, c);
  if (!S.alloc()) return gf_fail(ctx, GF_ERR_NOMEM, "RK work allocation failed");
  S.prepare_adv();  // advection with a prescribed velocity and nu = 0
  T *uu[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < tr->nstate; k++) uu[k] = (T *)u[k];
  for (int s = 0; s < nsteps; s++) {
    for (int k = 0; k < tr->nstate; k++)
      cudaMemcpyAsync(S.uold[k], uu[k], sizeof(T) * S.n, cudaMemcpyDeviceToDevice, S.st);
    int rc = S.step(S.uold, uu, (T)dt);
    if (rc) return gf_fail(ctx, rc, "RK step failed");
  }
  GF_CHECK_LAUNCH(ctx);
  // The reference asserts a finite state after every step; a NaN or Inf
  // stays in the state once made, so one check of the result after the
  // last step finds the same failures.  It reads the state once and waits
  // for the stream; inside a stream capture (a recorded step graph) it is
  // skipped, since the capture cannot wait.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  GF_CUDA(ctx, cudaStreamIsCapturing(S.st, &cs));
  if (nsteps > 0 && cs == cudaStreamCaptureStatusNone) {
    double *flag = prob->scal_d + RK_FLAG_SLOT;
    GF_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(double), S.st));
    prob->launches++;
    k_nonfinite<T><<<grid_for(S.n, 256, ctx->sm_count * 8), 256, 0, S.st>>>(
        S.n, tr->nstate, uu[0], uu[tr->nstate > 1 ? 1 : 0], uu[tr->nstate > 2 ? 2 : 0], flag);
    GF_CHECK_LAUNCH(ctx);
    GF_CUDA(ctx, cudaMemcpyAsync(prob->scal_h + RK_FLAG_SLOT, flag, sizeof(double),
                                 cudaMemcpyDeviceToHost, S.st));
    GF_CUDA(ctx, cudaStreamSynchronize(S.st));
    if (prob->scal_h[RK_FLAG_SLOT] != 0.0)
      return gf_fail(ctx, GF_ERR_NONFINITE, "solution not finite after %d RK steps", nsteps);
  }
  return GF_OK;
}

}  // namespace gfrk

using namespace gfrk;

extern "C" int gf_rk_advance(gf_problem_t prob, int dtype, const gf_rk_traits *tr, void *const *u,
                             const void *const *c, double t0, double dt, int nsteps) {
  if (!prob) return GF_ERR_ARG;
  (void)t0;
  int rc = check_traits(prob, tr, (const void *const *)u, c);
  if (rc) return rc;
  GF_REQUIRE(prob->ctx, nsteps >= 0, "nsteps must be >= 0");
  if (dtype == GF_F64) return advance<double>(prob, tr, u, c, dt, nsteps);
  if (dtype == GF_F32) return advance<float>(prob, tr, u, c, dt, nsteps);
  return gf_fail(prob->ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
}

// y = uin + ((0 + b0 K0) + b1 K1 + ...) on the problem's nlocal nodes: the
// stage input of step_b, as the stepper forms it (k_stage_sum); used by the
// partitioned stepper (geoflow_b200/dist.py).
extern "C" int gf_rk_stage_sum(gf_problem_t prob, int dtype, const void *uin, int nk,
                               const void *K0, const void *K1, const void *K2, double b0,
                               double b1, double b2, void *y) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, uin && y && nk >= 0 && nk <= 3, "stage sum needs uin, y and 0..3 terms");
  GF_REQUIRE(ctx, (nk < 1 || K0) && (nk < 2 || K1) && (nk < 3 || K2), "missing stage vector");
  const int64_t n = prob->nlocal;
  const unsigned g = grid_for(n, 256, ctx->sm_count * 8);
  prob->launches++;
  if (dtype == GF_F64)
    k_stage_sum<double><<<g, 256, 0, ctx->stream>>>(n, (const double *)uin, nk,
                                                    (const double *)K0, (const double *)K1,
                                                    (const double *)K2, b0, b1, b2, (double *)y);
  else if (dtype == GF_F32)
    k_stage_sum<float><<<g, 256, 0, ctx->stream>>>(n, (const float *)uin, nk, (const float *)K0,
                                                   (const float *)K1, (const float *)K2,
                                                   (float)b0, (float)b1, (float)b2, (float *)y);
  else
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_rk_advance_host(gf_problem_t prob, int dtype, const gf_rk_traits *tr,
                                  void *const *u, const void *const *c, double t0, double dt,
                                  int nsteps) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  int rc = check_traits(prob, tr, (const void *const *)u, c);
  if (rc) return rc;
  const size_t bytes = (dtype == GF_F64 ? 8 : 4) * (size_t)prob->nlocal;
  void *du[3] = {nullptr, nullptr, nullptr};
  const void *dc[3] = {nullptr, nullptr, nullptr};
  for (int k = 0; k < tr->nstate; k++) {
    du[k] = gf_work(prob, 90 + k, bytes);
    if (!du[k]) return gf_fail(ctx, GF_ERR_NOMEM, "staging allocation failed");
    GF_CUDA(ctx, cudaMemcpyAsync(du[k], u[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (tr->eqn == GF_EQN_ADVECT) {
    for (int k = 0; k < gf_nvel(prob); k++) {
      void *d = gf_work(prob, 93 + k, bytes);
      if (!d) return gf_fail(ctx, GF_ERR_NOMEM, "staging allocation failed");
      GF_CUDA(ctx, cudaMemcpyAsync(d, c[k], bytes, cudaMemcpyHostToDevice, ctx->stream));
      dc[k] = d;
    }
  }
  rc = gf_rk_advance(prob, dtype, tr, du, dc, t0, dt, nsteps);
  if (rc) return rc;
  for (int k = 0; k < tr->nstate; k++)
    GF_CUDA(ctx, cudaMemcpyAsync(u[k], du[k], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

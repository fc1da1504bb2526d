// gfgpu.hpp -- C++ host adapters over the libgfgpu C ABI (gfgpu.h).
//
// These classes keep the reference's interfaces on the hot path so that a
// GeoFLOW application can switch to the B200 kernels without touching its
// equation, stepper or solver code (reference citations relative to
// NOAA-GSL/GeoFLOW src/cdg/):
//   gfgpu::Helmholtz  ~ GHelmholtz<Types>::opVec_prod   (sem/ghelmholtz.hpp:58-60)
//   gfgpu::GGFX       ~ GGFX<T>::doOp(u, Sum/Smooth/Max/Min), get_mult/get_imult
//                                                    (comm/ggfx.hpp:87-98)
//   gfgpu::CG         ~ GCG<Types>::solve(A, b, [xb,] x) -> GCGERR code
//                                                    (solvers/gcg.hpp:32, lin_solver_base.hpp:66-97)
//   gfgpu::ExRK       ~ GExRKStepper::step on the GBurgers RHS
//                                                    (pdes/gexrk_stepper.hpp:44-66)
// Fields are device pointers (E-vector layout, exactly the GTVector layout
// of the reference).  Errors below zero throw gfgpu::Error; solver outcomes
// (GCGERR codes) are returned as in the reference.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "gfgpu.h"

namespace gfgpu {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline int check(gf_ctx_t ctx, int rc, const char *what) {
  if (rc < 0) throw Error(rc, std::string(what) + ": " + gf_ctx_last_error(ctx));
  return rc;
}

// Device + stream (one per host thread).
class Context {
 public:
  explicit Context(int device = 0, void *stream = nullptr) {
    int rc = gf_ctx_create(device, stream, &h_);
    if (rc) throw Error(rc, "gf_ctx_create failed");
  }
  ~Context() { gf_ctx_destroy(h_); }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  gf_ctx_t get() const { return h_; }
  void synchronize() { check(h_, gf_ctx_synchronize(h_), "synchronize"); }

 private:
  gf_ctx_t h_ = nullptr;
};

// Host description of a regular box grid (GGridBox), built by the library
// exactly as the reference lays it out, with its GGFX classes.
struct BoxGrid {
  int dim, p;
  std::vector<int> ne, periodic;
  std::vector<double> xi, W, D, elem_geom, mask;
  std::vector<std::vector<double>> xyz;
  std::vector<int32_t> node_class, class_ptr, members;
  int64_t nclass = 0;

  BoxGrid(int dim_, std::vector<int> ne_, int p_, std::vector<double> x0,
          std::vector<double> len, std::vector<int> per)
      : dim(dim_), p(p_), ne(ne_), periodic(per) {
    const int n = p + 1;
    xi.resize(n);
    W.resize(n);
    D.resize(n * n);
    gf_gll_basis(p, xi.data(), W.data(), D.data());
    int64_t nel = 1, nn = 1;
    for (int d = 0; d < dim; d++) {
      nel *= ne[d];
      nn *= n;
    }
    const int64_t N = nel * nn;
    xyz.assign(dim, std::vector<double>(N));
    std::vector<double *> xp;
    for (auto &v : xyz) xp.push_back(v.data());
    elem_geom.resize(nel * (dim + 1));
    mask.resize(N);
    int rc = gf_box_grid(dim, ne.data(), p, x0.data(), len.data(), periodic.data(), xp.data(),
                         elem_geom.data(), mask.data());
    if (rc) throw Error(rc, "gf_box_grid");
    node_class.resize(N);
    class_ptr.resize(N + 1);
    members.resize(N);
    nclass = gf_box_classes(dim, ne.data(), p, periodic.data(), node_class.data(),
                            class_ptr.data(), members.data());
    if (nclass < 0) throw Error((int)nclass, "gf_box_classes");
    class_ptr.resize(nclass + 1);
  }
  int64_t ndof() const { return (int64_t)members.size(); }
};

// Device-resident problem (geometry, operators, gather-scatter map).
class Problem {
 public:
  Problem(Context &ctx, const BoxGrid &g, bool dirichlet = true) : ctx_(ctx.get()) {
    gf_problem_desc d{};
    d.dim = g.dim;
    d.ne = (int64_t)g.elem_geom.size() / (g.dim + 1);
    d.n = g.p + 1;
    d.D = g.D.data();
    d.W = g.W.data();
    d.geom = GF_GEOM_AFFINE;
    d.elem_geom = g.elem_geom.data();
    d.mask = dirichlet ? g.mask.data() : nullptr;
    d.nclass = g.nclass;
    d.class_ptr = g.class_ptr.data();
    d.members = g.members.data();
    for (int k = 0; k < g.dim; k++) {
      d.box_ne[k] = g.ne[k];
      d.box_periodic[k] = g.periodic[k];
    }
    check(ctx_, gf_problem_create(ctx_, &d, &h_), "gf_problem_create");
  }
  ~Problem() { gf_problem_destroy(h_); }
  Problem(const Problem &) = delete;
  Problem &operator=(const Problem &) = delete;
  gf_problem_t get() const { return h_; }
  gf_ctx_t ctx() const { return ctx_; }

 private:
  gf_ctx_t ctx_;
  gf_problem_t h_ = nullptr;
};

// GGFX::doOp
class GGFX {
 public:
  enum Op { Sum = GF_DSS_SUM, Smooth = GF_DSS_SMOOTH, Max = GF_DSS_MAX, Min = GF_DSS_MIN };
  explicit GGFX(Problem &p) : p_(p) {}
  bool doOp(double *u, Op op) {
    check(p_.ctx(), gf_dss(p_.get(), GF_F64, op, u), "GGFX::doOp");
    return true;
  }
  bool doOp(float *u, Op op) {
    check(p_.ctx(), gf_dss(p_.get(), GF_F32, op, u), "GGFX::doOp");
    return true;
  }
  void get_mult(double *mult) { check(p_.ctx(), gf_mult(p_.get(), 0, mult), "get_mult"); }
  void get_imult(double *imult) { check(p_.ctx(), gf_mult(p_.get(), 1, imult), "get_imult"); }

 private:
  Problem &p_;
};

// GHelmholtz: H = q M + p L; the mass term is on once set_mass_scalar is called.
class Helmholtz {
 public:
  explicit Helmholtz(Problem &p) : p_(p) {}
  void set_Lap_scalar(double p) { lap_ = p; }
  void set_mass_scalar(double q) {
    q_ = q;
    use_mass_ = 1;
  }
  void opVec_prod(const double *u, double *uo) {
    check(p_.ctx(), gf_helmholtz_apply(p_.get(), GF_F64, lap_, nullptr, q_, nullptr, use_mass_, u, uo),
          "GHelmholtz::opVec_prod");
  }
  void opVec_prod(const float *u, float *uo) {
    check(p_.ctx(), gf_helmholtz_apply(p_.get(), GF_F32, lap_, nullptr, q_, nullptr, use_mass_, u, uo),
          "GHelmholtz::opVec_prod");
  }
  // The reference's three-argument form GHelmholtz::opVec_prod(in, utmp, out)
  // (sem/ghelmholtz.hpp:58-60, GLinOpBase, sem/glinop_base.hpp:32-34): the
  // library keeps its own scratch, so utmp is accepted and not touched.
  template <class Tmp>
  void opVec_prod(const double *u, Tmp & /*utmp*/, double *uo) { opVec_prod(u, uo); }
  template <class Tmp>
  void opVec_prod(const float *u, Tmp & /*utmp*/, float *uo) { opVec_prod(u, uo); }
  double lap() const { return lap_; }
  double mass_scalar() const { return q_; }
  int use_mass() const { return use_mass_; }

 private:
  Problem &p_;
  double lap_ = 1.0, q_ = 0.0;
  int use_mass_ = 0;
};

// GCG: solve(A, b, x) / solve(A, b, xb, x) returning GCGERR codes.
class CG {
 public:
  enum GCGERR { GCGERR_NONE = 0, GCGERR_NOCONVERGE, GCGERR_SOLVE, GCGERR_PRECOND, GCGERR_BADITERNUM };
  CG(const gf_cg_traits &tr, Problem &p) : tr_(tr), p_(p) {}
  int solve(Helmholtz &A, const double *b, double *x) { return run(A, b, nullptr, x); }
  int solve(Helmholtz &A, const double *b, const double *xb, double *x) { return run(A, b, xb, x); }
  // As GCG::get_iteration_count (solvers/gcg.hpp:75): iterations taken + 1.
  int get_iteration_count() const { return iters_ + 1; }
  int iterations() const { return iters_; }
  double get_resid() const { return rnorm_; }
  const std::vector<double> &get_residuals() const { return res_; }

 private:
  int run(Helmholtz &A, const double *b, const double *xb, double *x) {
    res_.assign(tr_.maxit > 0 ? tr_.maxit : 1, 0.0);
    int rc = gf_cg_solve(p_.get(), &tr_, A.lap(), A.mass_scalar(), A.use_mass(), b, xb, x, &iters_,
                         &rnorm_, res_.data());
    check(p_.ctx(), rc, "GCG::solve");
    res_.resize(iters_);
    return rc;
  }
  gf_cg_traits tr_;
  Problem &p_;
  int iters_ = 0;
  double rnorm_ = 0.0;
  std::vector<double> res_;
};

// GExRKStepper on the GBurgers right-hand side.
class ExRK {
 public:
  ExRK(Problem &p, int eqn, double nu, int nstate, int scheme) : p_(p) {
    tr_.eqn = eqn;
    tr_.nu = nu;
    tr_.nstate = nstate;
    tr_.scheme = scheme;
  }
  // u[nstate] advanced in place; c[dim] prescribed velocities (advection)
  void step(double *const *u, const double *const *c, double t, double dt, int nsteps = 1) {
    check(p_.ctx(),
          gf_rk_advance(p_.get(), GF_F64, &tr_, (void *const *)u, (const void *const *)c, t, dt,
                        nsteps),
          "GExRKStepper::step");
  }

 private:
  Problem &p_;
  gf_rk_traits tr_{};
};

}  // namespace gfgpu

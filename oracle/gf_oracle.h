/*
 * gf_oracle.h -- CPU oracle for the GeoFLOW spectral-element hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference algorithms (NOAA-GSL/GeoFLOW, src/cdg/...), used by the test
 * suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as
 * the checker.  Nothing in the product library links or calls it.
 *
 * Parity pins: GLL basis and the GMTK tensor products are checked against
 * the reference's own GLLBasis/GMTK sources compiled in oracle/_ref; the
 * grid, GGFX, Helmholtz, CG and RK restatements are pinned by the known
 * answers of the reference's own tests (cdg_gmtk, cdg_ggfx, cdg_cg,
 * cdg_mass/integrate, hackathon derivative) re-run against this oracle.
 *
 * Conventions: all matrices are column-major (GTMatrix, gtmatrix.hpp:104),
 * D[l + j*n] = dphi_j/dxi (xi_l) (gllbasis.ipp:580-606).  Fields are
 * element-major E-vectors with x fastest inside an element.
 */
#ifndef GF_ORACLE_H
#define GF_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* GGFX reduction ops (ggfx.hpp:36-76). */
enum { GFO_SUM = 0, GFO_SMOOTH = 1, GFO_MAX = 2, GFO_MIN = 3 };
/* LinSolverBase norm types (lin_solver_base.hpp:38-44). */
enum { GFO_NORM_INF = 0, GFO_NORM_EUC = 1, GFO_NORM_L2 = 2, GFO_NORM_L1 = 3 };
/* CG error codes (gcg.hpp:32). */
enum { GFO_CG_NONE = 0, GFO_CG_NOCONVERGE = 1, GFO_CG_SOLVE = 2, GFO_CG_PRECOND = 3, GFO_CG_BADITERNUM = 4 };

/* ---- GLL basis (gllbasis.ipp:411-606), long double internally ---- */
int gfo_gll(int p, double *xi, double *w, double *D);

/* ---- Fortran dmxm contract (cff_blas.F:846-943, dmxmp.F) ---- */
void gfo_dmxm(double *C, const double *A, size_t nai, const double *B,
              size_t nbi, size_t nbj);

/* ---- GMTK tensor products, per element, all Ne elements ---- */
void gfo_I2_X_D1(const double *D1, const double *u, size_t N1, size_t N2,
                 size_t Ne, double *y);
void gfo_D2_X_I1(const double *D2T, const double *u, size_t N1, size_t N2,
                 size_t Ne, double *y);
void gfo_I3_X_I2_X_D1(const double *D1, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y);
void gfo_I3_X_D2_X_I1(const double *D2T, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y);
void gfo_D3_X_I2_X_I1(const double *D3T, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y);

/* ---- Grid description (regular elements, GGridBox) ----
 * D holds dim column-major n_d x n_d matrices packed back to back, W the
 * dim weight vectors packed back to back.  dXidX holds dim per-node arrays
 * (dXidX(k,0) of ggrid.ipp reg_geom_init), Jac one per-node array. */
typedef struct {
  int dim;
  size_t Ne;
  int n[3];
  const double *D[3];
  const double *W[3];
  const double *dXidX[3];
  const double *Jac;
  const double *mass;   /* W x W (x W) x Jac, gmass.ipp:134-220 */
} gfo_grid;

size_t gfo_box_ndof(int dim, const int *ne, const int *p);
/* Build a GGridBox-equivalent element list: node coordinates (x,y[,z]),
 * dXidX, Jac, mask (0 on non-periodic boundary nodes).  periodic[d]!=0
 * marks a periodic direction.  Arrays are ndof long. */
void gfo_box_build(int dim, const int *ne, const int *p, const double *x0,
                   const double *len, const int *periodic, double *x,
                   double *y, double *z, double *dXidX0, double *dXidX1,
                   double *dXidX2, double *Jac, double *mask);
/* GMass::init2d/init3d (gmass.ipp:134-220). */
void gfo_mass(const gfo_grid *g, double *mass);
/* GGrid::integrate (ggrid.ipp:1077-1147). */
double gfo_integrate(const gfo_grid *g, const double *u);

/* ---- GGFX (ggfx.hpp) ----
 * init: classes from coordinate matching with box tolerance tol, after the
 * periodize step (ggrid_box.ipp:753-806).  Outputs node_class[N] and a CSR
 * (class_ptr[nclass+1], members[N], ascending within each class; classes
 * ordered by smallest member).  Returns nclass, or -1 on error. */
long gfo_ggfx_init(size_t N, int dim, const double *x, const double *y,
                   const double *z, double tol, int32_t *node_class,
                   int32_t *class_ptr, int32_t *members);
void gfo_ggfx_doop(double *u, size_t nclass, const int32_t *class_ptr,
                   const int32_t *members, int op);
void gfo_ggfx_doop_f(float *u, size_t nclass, const int32_t *class_ptr,
                     const int32_t *members, int op);
void gfo_ggfx_mult(size_t N, size_t nclass, const int32_t *class_ptr,
                   const int32_t *members, double *mult);

/* ---- reference-space derivatives (ggrid.ipp:1847-2265) ---- */
void gfo_grefderiv(const gfo_grid *g, const double *u, int idir, int dotrans,
                   double *du);
void gfo_grefdiv(const gfo_grid *g, const double *const *u, int dotrans,
                 double *divu);
/* GGrid::deriv (ggrid.ipp:1163-1190), regular grid. */
void gfo_deriv(const gfo_grid *g, const double *u, int idir, double *du);

/* ---- GHelmholtz::reg_prod (ghelmholtz.ipp:309-378) ----
 * p: scalar p_scalar unless p_vec != NULL; q_vec != NULL adds q M u. */
void gfo_helmholtz(const gfo_grid *g, const double *u, double p_scalar,
                   const double *p_vec, const double *q_vec, double *uo);
/* FP32 restatement of the same operator (GFLOAT instantiation). */
void gfo_helmholtz_f(int dim, size_t Ne, int n, const float *D,
                     const float *W, const float *gscale, float p_scalar,
                     const float *q_vec, const float *u, float *uo);

/* ---- GAdvect::apply (gadvect.ipp:58-100), ncomp velocity components ---- */
void gfo_advect(const gfo_grid *g, const double *p, int ncomp,
                const double *const *c, double *po);

/* ---- GBurgers::dudt_impl (gburgers.ipp:203-257) ----
 * kind 0: pure advection (nstate=1, c given), 1: nonlinear Burgers
 * (nstate=dim, c=u), 2: heat.  imass = 1/Smooth(mass). */
void gfo_dudt(const gfo_grid *g, int kind, double nu, const double *imass,
              int nstate, const double *const *u, const double *const *c,
              double *const *dudt);

/* ---- deformed (GE_DEFORMED) and 2-d embedded (GE_2DEMBEDDED) elements ----
 * X[i][k] = dXi_i/dX_k per node, i < dim, k < nxy (nxy = dim, or 3 for a
 * 2-d surface embedded in 3-d space); base->Jac, base->mass as for regular
 * grids (base->dXidX unused). */
typedef struct {
  const gfo_grid *base;
  int nxy;
  const double *X[3][3];
} gfo_defgrid;
/* GHelmholtz::def_init (ghelmholtz.ipp:416-519): G(i,j) = sum_k X[i][k]
 * X[j][k] W Jac for i,j < dim, as the 2-d branch computes it (the 3-d
 * branch accumulates each off-diagonal twice through the shared storage of
 * G(i,j) and G(j,i); the formula in its comment is followed here). */
void gfo_def_metric(const gfo_defgrid *g, double *const G[3][3]);
/* GHelmholtz::def_prod / embed_prod (ghelmholtz.ipp:109-293). */
void gfo_def_helmholtz(const gfo_defgrid *g, const double *const G[3][3], const double *u,
                       double p_scalar, const double *p_vec, const double *q_vec,
                       double *uo);
/* GGrid::deriv (ggrid.ipp:1163-1190), deformed branch: idir = 1..nxy. */
void gfo_def_deriv(const gfo_defgrid *g, const double *u, int idir, double *du);
/* GAdvect::apply (gadvect.ipp:58-100) with nxy velocity components. */
void gfo_def_advect(const gfo_defgrid *g, const double *p, const double *const *c,
                    double *po);
/* GBurgers::dudt_impl on a deformed/embedded grid: kind as gfo_dudt;
 * Burgers evolves nxy components. */
void gfo_def_dudt(const gfo_defgrid *g, const double *const G[3][3], int kind, double nu,
                  const double *imass, int nstate, const double *const *u,
                  const double *const *c, double *const *dudt);
/* GMTK::constrain2sphere (2) (gmtk.ipp:2957-2976), in place on v[0..2] of
 * N nodes at coordinates xyz[0..2]: components updated in order, each from
 * the already-updated earlier ones, r^2 taken at node 0. */
void gfo_constrain2sphere(size_t N, const double *const *xyz, double *const *v);

/* ---- GExRKStepper (gexrk_stepper.ipp) on the Burgers RHS ----
 * scheme: 1..4 Butcher step_b(1) of that order, 22/33/34 SSP schemes.
 * u[nstate] updated in place over nsteps steps of size dt. */
typedef struct {
  const gfo_grid *g;
  int kind;
  double nu;
  const double *imass;
  const double *const *c;  /* prescribed velocity for kind 0 */
  size_t nclass;
  const int32_t *class_ptr;
  const int32_t *members;
} gfo_burgers;
void gfo_rk_advance(const gfo_burgers *b, int scheme, int nstate,
                    double *const *u, double t0, double dt, int nsteps);

/* ---- GCG::solve_impl (gcg.ipp:239-382) on the Helmholtz operator ----
 * xb may be NULL (solve_impl(1)); otherwise solve_impl(2).  dinv: Jacobi
 * preconditioner (no reference counterpart) or NULL for identity.
 * residuals: optional maxit-long history. */
typedef struct {
  int maxit;
  int normtype;
  double tol;
} gfo_cg_traits;
int gfo_cg_solve(const gfo_grid *g, double p_scalar, const double *q_vec,
                 const double *mask, size_t nclass, const int32_t *class_ptr,
                 const int32_t *members, const double *dinv,
                 const gfo_cg_traits *tr, const double *b, const double *xb,
                 double *x, int *iters, double *residuals);
/* Assembled diagonal of the Helmholtz operator (DSS Sum of local diag). */
void gfo_helmholtz_diag(const gfo_grid *g, double p_scalar,
                        const double *q_vec, size_t nclass,
                        const int32_t *class_ptr, const int32_t *members,
                        double *diag);

#ifdef __cplusplus
}
#endif
#endif

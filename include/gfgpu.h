/*
 * gfgpu.h -- C ABI of libgfgpu, the B200 (sm_100a) implementation of the
 * GeoFLOW spectral-element hot path.
 *
 * Conventions
 *  - Every entry point returns int: 0 on success, a positive GCG-style code
 *    for solver outcomes (GF_CG_NOCONVERGE ...), a negative GF_ERR_* on
 *    argument or CUDA errors.  The last error message of a context is kept
 *    (sticky) and read with gf_ctx_last_error().
 *  - Field arguments are DEVICE pointers in element-local ("E-vector")
 *    layout: element-major, x fastest inside an element, exactly the
 *    GTVector layout of the reference (grid/ggrid_box.ipp:394-406).  The
 *    *_host entry points take host pointers and stage through the device.
 *  - All work is ordered on the context's CUDA stream; calls that return a
 *    scalar to the host synchronise that stream.
 *  - 1-d operators are column-major, D[l + j*n] = dphi_j/dxi(xi_l), as
 *    GLLBasis::getDerivMatrix(FALSE) (sem/gllbasis.ipp:580-606).
 *
 * Reference file citations are relative to NOAA-GSL/GeoFLOW src/cdg/.
 */
#ifndef GFGPU_H
#define GFGPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GFGPU_ABI_VERSION 1

/* ---- status codes ---- */
enum {
  GF_OK = 0,
  /* GCG::GCGERR (solvers/gcg.hpp:32), returned by gf_cg_solve */
  GF_CG_NOCONVERGE = 1,
  GF_CG_SOLVE = 2,
  GF_CG_PRECOND = 3,
  GF_CG_BADITERNUM = 4,
  /* ABI errors */
  GF_ERR_ARG = -1,
  GF_ERR_CUDA = -2,
  GF_ERR_UNSUPPORTED = -3,
  GF_ERR_NOMEM = -4,
  GF_ERR_NONFINITE = -5,
  GF_ERR_WATCHDOG = -6,
  GF_ERR_IO = -7
};

/* ---- enumerations ---- */
enum { GF_F64 = 0, GF_F32 = 1 };                       /* field dtype */
enum { GF_DSS_SUM = 0, GF_DSS_SMOOTH = 1, GF_DSS_MAX = 2, GF_DSS_MIN = 3 }; /* ggfx.hpp:36-76 */
enum { GF_NORM_INF = 0, GF_NORM_EUC = 1, GF_NORM_L2 = 2, GF_NORM_L1 = 3 }; /* lin_solver_base.hpp:38 */
/* CHEBYSHEV: FP64 flexible CG whose preconditioner is a Chebyshev
 * polynomial in D^-1 A applied in FP32 (poly_degree FP32 applies per step);
 * no reference counterpart */
/* PMG: FP64 flexible CG whose preconditioner is one FP32 multigrid V-cycle:
 * p-coarsening p -> ceil(p/2) -> ... -> 1 on the same elements, then h-coarsening
 * of the p = 1 box by 2 in every direction while the element counts stay
 * even, with Chebyshev-Jacobi smoothing of degree poly_degree on every
 * level (interval [lmax/poly_ratio, lmax], lmax from a Lanczos estimate).
 * Structured affine boxes only (box_ne set, GF_GEOM_AFFINE, mask absent or
 * the box-face Dirichlet mask); the hierarchy is kept with the problem and
 * reused while p, q and the traits stay the same.  No reference counterpart.
 * PMG64: the same V-cycle with every level's vectors, transfers, smoother
 * and coarsest solve in FP64 (what the FP32 V-cycle saves, measured). */
enum {
  GF_PRECOND_NONE = 0,
  GF_PRECOND_JACOBI = 1,
  GF_PRECOND_CHEBYSHEV = 2,
  GF_PRECOND_PMG = 3,
  GF_PRECOND_PMG64 = 4
};
enum { GF_CG_FP64 = 0, GF_CG_MIXED = 1 };            /* plain FP64 / FP32 apply + FP64 refinement */
/* see gf_problem_desc; DEFORMED = GE_DEFORMED, EMBEDDED = GE_2DEMBEDDED */
enum { GF_GEOM_AFFINE = 0, GF_GEOM_REGULAR = 1, GF_GEOM_DEFORMED = 2, GF_GEOM_EMBEDDED = 3 };
enum { GF_EQN_ADVECT = 0, GF_EQN_BURGERS = 1, GF_EQN_HEAT = 2 }; /* GBurgers traits */
/* GExRKStepper schemes: Butcher orders 1..4 (gbutcherrk.ipp:69-125) and
 * the SSP schemes (gexrk_stepper.ipp:533-780) */
enum { GF_RK1 = 1, GF_RK2 = 2, GF_RK3 = 3, GF_RK4 = 4, GF_SSP22 = 22, GF_SSP33 = 33, GF_SSP34 = 34 };

typedef struct gf_context *gf_ctx_t;
typedef struct gf_problem *gf_problem_t;

/* ---- context ---- */
/* Creates a context on CUDA device `device`; `stream` is the cudaStream_t
 * all of the context's work is ordered on (NULL: the legacy default
 * stream, ordered with every other blocking stream of the process). */
int gf_ctx_create(int device, void *stream, gf_ctx_t *out);
int gf_ctx_destroy(gf_ctx_t ctx);
/* Last error message of the context ("" if none); clears it. */
const char *gf_ctx_last_error(gf_ctx_t ctx);
int gf_ctx_synchronize(gf_ctx_t ctx);
int gf_abi_version(void);

/* ---- host-side set-up helpers (no device work) ---- */
/* GLL nodes xi[p+1], weights w[p+1] and D[(p+1)^2] in the reference's
 * long-double construction cast to double.  Replaces GLLBasis::init
 * (sem/gllbasis.ipp:411-606,715-737). */
int gf_gll_basis(int p, double *xi, double *w, double *D);

/* Regular box grid of GGridBox (grid/ggrid_box.ipp:24-105,250-463,860-980):
 * lexicographic element list, node coordinates xyz[dim][N_local], regular
 * geometry (dXidX = 2/L per element, Jac = prod L / 2^dim), mask[N_local]
 * (0 on non-periodic boundary nodes, ggrid.ipp:1458-1466).  Any output
 * pointer may be NULL.  elem_geom[ne*(dim+1)] = {dXidX_0..dim-1, Jac}. */
int gf_box_grid(int dim, const int *ne, int p, const double *x0,
                const double *len, const int *periodic, double *const *xyz,
                double *elem_geom, double *mask);

/* Equivalence classes of a regular box grid (the result of GGFX::init on
 * periodized coordinates, comm/ggfx.hpp:169-342, ggrid_box.ipp:753-840),
 * built directly from the lattice: node_class[N_local], class_ptr[nclass+1],
 * members[N_local] ascending within each class, classes ordered by smallest
 * member.  Returns nclass (>=0) or a negative error. */
int64_t gf_box_classes(int dim, const int *ne, int p, const int *periodic,
                       int32_t *node_class, int32_t *class_ptr,
                       int32_t *members);

/* Geometry-free matching of GGFX::init (comm/ggfx.hpp:169-342): classes of
 * nodes whose tolerance boxes intersect, from coordinates xyz[dim][n].
 * Same outputs as gf_box_classes. */
int64_t gf_classes_from_coords(int dim, int64_t n, const double *const *xyz,
                               double tol, int32_t *node_class,
                               int32_t *class_ptr, int32_t *members);

/* The same two constructions on the device: identical classes, numbering
 * and CSR (bit for bit), written into DEVICE arrays node_class[n],
 * class_ptr[n+1] (the first ncls+1 entries are set) and members[n];
 * returns the class count or a negative error.  xyz is a host array of dim
 * DEVICE pointers.  The coordinate matching bins nodes in cells of width
 * 4 tol (at most 2^21 - 2 cells per direction) and takes, for every node,
 * the smallest id among the nodes whose tolerance boxes meet its own: the
 * host's classes whenever matches are transitive (tolerance below half the
 * node spacing, as GGFX::init requires). */
int64_t gf_box_classes_device(gf_ctx_t ctx, int dim, const int *ne, int p, const int *periodic,
                              int32_t *node_class, int32_t *class_ptr, int32_t *members);
int64_t gf_classes_from_coords_device(gf_ctx_t ctx, int dim, int64_t n,
                                      const double *const *xyz, double tol, int32_t *node_class,
                                      int32_t *class_ptr, int32_t *members);

/* The 2-d icosahedral sphere of GGridIcos (GE_2DEMBEDDED surface):
 * the base icosahedron (grid/ggrid_icos.ipp:134-225) refined by
 * GICOS_BISECTION (2^level - 1 rows of sub-triangles per face) or
 * GICOS_LAGRANGIAN (level rows) (lagrefine, 252-320), each triangle cut
 * into 3 quadrilateral elements of order p on the sphere of `radius`
 * (do_elems2d, 378-515).  gf_icos_sizes gives the element and node
 * counts; gf_icos_grid fills the node coordinates xyz[0..2] (3 host arrays
 * of nlocal) and, when node_geom != NULL, the embedded metric as
 * gf_problem_desc.node_geom takes it for GF_GEOM_EMBEDDED: planes
 * i*3 + k = dXi_i/dX_k (i < 2, k < 3) and plane 6 = Jac, each nlocal long
 * (GElem_base::dogeom2d, sem/gelem_base.cpp:877-970).  Host only.
 * Elements come in the reference's order (one rank). */
enum { GF_ICOS_BISECTION = 0, GF_ICOS_LAGRANGIAN = 1 };
int gf_icos_sizes(int level, int p, int refine, int64_t *nelems, int64_t *nlocal);
int gf_icos_grid(int level, int p, double radius, int refine, double *const *xyz,
                 double *node_geom);

/* ---- problem (grid + operators + gather-scatter map) ---- */
typedef struct {
  int dim;                 /* 2 or 3 */
  int64_t ne;              /* number of elements */
  int n;                   /* GLL points per direction (p+1), 2..12 */
  const double *D;         /* host, n*n column-major 1-d derivative */
  const double *W;         /* host, n GLL weights */
  int geom;                /* GF_GEOM_* */
  /* GF_GEOM_AFFINE: host ne*(dim+1): dXidX_0..dim-1, Jac per element */
  const double *elem_geom;
  /* GF_GEOM_REGULAR: host (dim+1)*N_local: dXidX_0..dim-1, Jac per node
   * (GGrid::dXidX(k,0), GGrid::Jac of reg_geom_init, ggrid.ipp:707-797).
   * GF_GEOM_DEFORMED / GF_GEOM_EMBEDDED (dim 2 surface in 3-d space):
   * host (dim*nxy+1)*N_local, nxy = dim (DEFORMED) or 3 (EMBEDDED):
   * plane i*nxy+k = dXi_i/dX_k (GGrid::dXidX(i,k), def_geom_init), then Jac.
   * The Laplacian uses G_ij = sum_k dXi_i/dX_k dXi_j/dX_k W Jac
   * (GHelmholtz::def_init, ghelmholtz.ipp:416-519). */
  const double *node_geom;
  const double *mask;      /* host N_local, or NULL (all ones) */
  /* gather-scatter map (GGFX::recv_map_ as CSR) */
  int64_t nclass;
  const int32_t *class_ptr; /* host nclass+1 */
  const int32_t *members;   /* host N_local, ascending inside each class */
  /* optional: the grid is a regular box of box_ne[d] elements per direction
   * in lexicographic order (GGridBox), periodic where box_periodic[d] != 0.
   * When box_ne[0] > 0 the library checks that the CSR equals the lattice
   * classes and then indexes unique nodes by lattice point, reading no
   * index arrays in the solver. */
  int box_ne[3];
  int box_periodic[3];
  /* optional host 3*N_local node coordinates (GGrid::xNodes); used by
   * constrain2sphere in the RK stepper on EMBEDDED grids */
  const double *node_xyz;
} gf_problem_desc;

int gf_problem_create(gf_ctx_t ctx, const gf_problem_desc *desc, gf_problem_t *out);
int gf_problem_destroy(gf_problem_t prob);
int gf_problem_sizes(gf_problem_t prob, int64_t *nlocal, int64_t *nclass);
/* Number of kernels the library has launched for this problem so far
 * (instrumentation, in the spirit of the reference's tracer ranges). */
int gf_problem_stats(gf_problem_t prob, int64_t *kernel_launches);

/* ---- library options ---- */
/* The FP32 3-d apply on affine elements at p = 7 (gf_helmholtz_apply and
 * the FP32 applies inside the CG solvers): GF_FP32_APPLY_FMA contracts the
 * lines with packed FP32x2 FMAs; GF_FP32_APPLY_TF32 as 3xTF32 tensor-core
 * products (mma.sync m16n8k8: TF32 head and tail of each operand, FP32
 * accumulation; FP32-level accuracy).  Process-wide; returns the previous
 * mode, or GF_ERR_ARG for an unknown one.  No reference counterpart. */
enum { GF_FP32_APPLY_FMA = 0, GF_FP32_APPLY_TF32 = 1 };
int gf_set_fp32_apply(int mode);

/* ---- operators (device pointers) ---- */
/* GHelmholtz::opVec_prod (sem/ghelmholtz.ipp:77-93, reg_prod 309-378):
 * uo = p L u + q M u with L the weak Laplacian sum_k Dk^T (Gk M) Dk u.
 * p_vec/q_vec (device, N_local, same dtype) override the scalars when
 * non-NULL; use_mass=0 drops the mass term (set_mass_scalar never called). */
int gf_helmholtz_apply(gf_problem_t prob, int dtype, double p, const void *p_vec,
                       double q, const void *q_vec, int use_mass,
                       const void *u, void *uo);
/* Adjoint (transpose) of gf_helmholtz_apply: the operator is symmetric
 * element by element, so this applies the transposed contractions
 * explicitly; used by the adjoint path and its dot-product test. */
int gf_helmholtz_apply_T(gf_problem_t prob, int dtype, double p, double q,
                         int use_mass, const void *u, void *uo);
/* GMass::opVec_prod (sem/gmass.ipp:226-233); inverse=1 uses
 * 1/Smooth(M) (gmass.ipp:65-92). */
int gf_mass_apply(gf_problem_t prob, int dtype, int inverse, const void *u, void *uo);
/* GGrid::compute_grefderiv (ggrid.ipp:2046-2265): du = (D_idir or
 * D_idir^T when dotrans) u, idir = 1..dim. */
int gf_grefderiv(gf_problem_t prob, int dtype, const void *u, int idir, int dotrans, void *du);
/* GGrid::compute_grefdiv (ggrid.ipp:1847-1927): divu = sum_k Dk^T u_k
 * (dotrans=1) or sum_k Dk u_k (dotrans=0). */
int gf_grefdiv(gf_problem_t prob, int dtype, const void *const *u, int dotrans, void *divu);
/* GGrid::deriv (ggrid.ipp:1163-1190): physical derivative du/dx_idir. */
int gf_deriv(gf_problem_t prob, int dtype, const void *u, int idir, void *du);
/* GAdvect::apply (sem/gadvect.ipp:58-100): po = M sum_j c_j dp/dx_j. */
int gf_advect_apply(gf_problem_t prob, int dtype, const void *p, int ncomp,
                    const void *const *c, void *po);
/* GBurgers::dudt_impl (pdes/gburgers.ipp:203-257), fused per element.
 * eqn: GF_EQN_ADVECT (nstate=1, c = dim prescribed velocities),
 * GF_EQN_BURGERS (nstate=dim, c ignored), GF_EQN_HEAT. */
int gf_dudt(gf_problem_t prob, int dtype, int eqn, double nu, int nstate,
            const void *const *u, const void *const *c, void *const *dudt);
/* GGFX::doOp (comm/ggfx.hpp:346-443), bit-exact: each class reduced in
 * ascending local id order, Sum/Smooth from 0, Max/Min as std::max/min
 * folds from lowest()/max().  (A NaN produced by Sum/Smooth is the GPU's
 * canonical NaN, not the input's payload.) */
int gf_dss(gf_problem_t prob, int dtype, int op, void *u);
/* GGFX::get_mult / get_imult (comm/ggfx.hpp:453-487), double output. */
int gf_mult(gf_problem_t prob, int inverse, double *mult);
/* GGrid::integrate (ggrid.ipp:1077-1147): returns the integral in *result
 * (host).  Synchronises. */
int gf_integrate(gf_problem_t prob, int dtype, const void *u, double *result);
/* Full tensor product of per-direction n x n matrices (host, column-major
 * like D): out = (A3 (x) A2 (x) A1) u in every element, A3 ignored in 2-d.
 * GMTK::D2_X_D1 (blas/gmtk.ipp:1570-1619), D3_X_D2_X_D1 (1930-1996) and the
 * weighted forms (1639-1911, 2311-2519) with the weights folded into A_d;
 * GBoydFilter::apply_impl (sem/gboyd_filter.ipp) is A_d = the basis' filter
 * matrix F. out must not alias u. */
int gf_tensor_apply(gf_problem_t prob, int dtype, const double *A1, const double *A2,
                    const double *A3, const void *u, void *out);
/* GMTK::constrain2sphere (2) (blas/gmtk.ipp:2957-2976): v[0..2] (device,
 * N_local each) projected in place onto the sphere through the node
 * coordinates xyz[0..2] (device), with the reference's order: components
 * updated in turn, each from the already-updated earlier ones, r^2 of
 * node 0.  Does nothing unless the problem is GF_GEOM_EMBEDDED, as the
 * reference does nothing unless the grid is GE_2DEMBEDDED. */
int gf_constrain2sphere(gf_problem_t prob, int dtype, void *const *v, const void *const *xyz);

/* ---- conjugate gradient (solvers/gcg.ipp:239-429) ---- */
typedef struct {
  int maxit;        /* LinSolverBase::Traits::maxit */
  int normtype;     /* GF_NORM_* */
  double tol;       /* stop when norm(r) <= (norm(b) < 1 ? tol : tol*norm(b)) */
  int precond;      /* GF_PRECOND_* (Jacobi has no reference counterpart) */
  int precision;    /* GF_CG_FP64 or GF_CG_MIXED */
  double inner_tol; /* MIXED: > 0 restarted refinement, each FP32 PCG run
                       reduces the true residual by this factor; 0 one FP32
                       PCG run with reliable updates every check_every its */
  int max_refine;   /* MIXED, restarted: maximum refinement sweeps (0: no cap) */
  int check_every;  /* iterations between host convergence checks (>=1) */
  int relative;     /* 1: stop at norm(r) <= tol*norm(b) even when norm(b) < 1 */
  int mixed_apply;  /* MIXED, 3-d: 0 FP32 arithmetic in the FP32 solve's applies,
                       1 FP64 arithmetic on the FP32-stored vectors */
  int poly_degree;  /* CHEBYSHEV: FP32 applies per preconditioner application;
                       PMG: Chebyshev smoothing degree per level and side */
  double poly_ratio;/* CHEBYSHEV: b/a of the polynomial's interval [a, b], b from
                       a Lanczos estimate of the largest eigenvalue of D^-1 A
                       (<= 1: max(4, 2 poly_degree^2)); PMG: the same ratio of
                       the smoothing interval (<= 1: 8) */
} gf_cg_traits;

/* Solves (p L + q M) x = b on the assembled space (DSS Sum + mask), as
 * GCG::solve_impl(A,b,xb,x) when xb != NULL or solve_impl(A,b,x) when
 * xb == NULL.  b, xb, x are device FP64 E-vectors; x holds the initial
 * guess on entry.  iters/final_norm/residuals (host, maxit) may be NULL.
 * Returns 0, GF_CG_NOCONVERGE or a negative error. */
int gf_cg_solve(gf_problem_t prob, const gf_cg_traits *traits, double p, double q,
                int use_mass, const double *b, const double *xb, double *x,
                int *iters, double *final_norm, double *residuals);
/* Same with host buffers: copies b, xb, x to the device, solves, copies x
 * back.  Synchronises. */
int gf_cg_solve_host(gf_problem_t prob, const gf_cg_traits *traits, double p, double q,
                     int use_mass, const double *b, const double *xb, double *x,
                     int *iters, double *final_norm);

/* Launches ONE kernel that the multigrid-preconditioned solve (precond
 * GF_PRECOND_PMG or GF_PRECOND_PMG64) runs on its finest level, outside
 * the solve's graph, so that a caller can time it with events on the
 * context's stream: GF_PMG_PREPARE builds (or reuses) the hierarchy of
 * these traits and operator (masked = 1: the Dirichlet-masked form, the
 * solve with xb) and fills the level's vectors with finite values;
 * GF_PMG_APPLY64 the outer FP64 lattice -> element apply; GF_PMG_APPLY the
 * V-cycle's lattice -> element apply (FP32 or FP64); GF_PMG_STEP a
 * smoother step pass (fold, residual, x and d update); GF_PMG_RESID the
 * residual pass; GF_PMG_RESTRICT / GF_PMG_PROLONG the transfers between the
 * finest level and the next.  Overwrites the hierarchy's vectors and the problem's CG
 * work vectors.  Not a reference interface (measurement only). */
enum {
  GF_PMG_PREPARE = 0,
  GF_PMG_APPLY64 = 1,
  GF_PMG_APPLY = 2,
  GF_PMG_STEP = 3,
  GF_PMG_RESID = 4,
  GF_PMG_RESTRICT = 5,
  GF_PMG_PROLONG = 6
};
int gf_pmg_launch(gf_problem_t prob, const gf_cg_traits *traits, double p, double q, int use_mass,
                  int masked, int which);

/* ---- explicit RK (pdes/gexrk_stepper.ipp) on the GBurgers RHS ---- */
typedef struct {
  int eqn;        /* GF_EQN_* */
  double nu;      /* dissipation (GBurgers traits nu) */
  int nstate;     /* evolved components: 1 for ADVECT/HEAT, dim for BURGERS */
  int scheme;     /* GF_RK1..4, GF_SSP22/33/34 */
} gf_rk_traits;
/* Advances u[nstate] (device, dtype) in place by nsteps steps of size dt,
 * with the DSS Smooth calls where GExRKStepper::step_b / step_ssp* place
 * them.  c[dim] are prescribed velocities for GF_EQN_ADVECT (else NULL).
 * Returns GF_ERR_NONFINITE when the state holds a NaN or Inf after the last
 * step (GBurgers::step_impl asserts a finite state, gburgers.ipp:325-331);
 * that check waits for the stream, and is skipped while the stream is
 * being captured into a graph. */
int gf_rk_advance(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                  void *const *u, const void *const *c, double t0, double dt, int nsteps);
/* Host-buffer variant: copies u and c in, advances, copies u out. */
int gf_rk_advance_host(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                       void *const *u, const void *const *c, double t0, double dt, int nsteps);

/* ---- building blocks of the element-partitioned (multi-GPU) path ----
 * (geoflow_b200/dist.py; no single reference counterpart: GGFX::doOp's
 * send/recv exchange, comm/ggfx.hpp:346-443, and GExRKStepper's stage
 * arithmetic, pdes/gexrk_stepper.ipp:252-341, 533-819, split at the
 * exchange.)  All arrays are device arrays on the problem's stream.
 * gf_gather: dst[k] = src[idx[k]], k < n.
 * gf_dss_fold_copies: for k < nout, u[out_local[k]] = the GGFX fold (op)
 *   of point out_point[k]'s copies pool[table[point*maxc + j]], j in order
 *   while table[...] >= 0 (Sum/Smooth from 0, Smooth divided by the copy
 *   count, Max/Min as std::max/min folds): the reference's fold order when
 *   the table lists the copies in ascending global local id.
 * gf_rk_stage_sum: y = uin + ((0 + b0 K0) + b1 K1 + b2 K2) (nk terms).
 * gf_rk_update: x = dt x + uin; x = a x + b y (if y); x = a2 x + b2 y2
 *   (if y2): the SSP substep update before its Smooth.
 * gf_rk_accum: uout = uout + K ch.
 * The last three run on the problem's nlocal nodes. */
int gf_gather(gf_problem_t prob, int dtype, int64_t n, const int32_t *idx, const void *src,
              void *dst);
int gf_dss_fold_copies(gf_problem_t prob, int dtype, int op, int maxc, const int32_t *table,
                       const void *pool, int64_t nout, const int32_t *out_local,
                       const int32_t *out_point, void *u);
int gf_rk_stage_sum(gf_problem_t prob, int dtype, const void *uin, int nk, const void *K0,
                    const void *K1, const void *K2, double b0, double b1, double b2, void *y);
int gf_rk_update(gf_problem_t prob, int dtype, void *x, double dt, const void *uin, double a,
                 const void *y, double b, double a2, const void *y2, double b2);
int gf_rk_accum(gf_problem_t prob, int dtype, void *uout, const void *K, double ch);
/* Replaces the problem's inverse mass 1/Smooth(M) (used by gf_dudt and the
 * RK stepper) with the caller's host values (nlocal): the assembled values
 * when the problem is one rank's part of a partitioned grid. */
int gf_problem_set_imass(gf_problem_t prob, const double *imass);

/* ---- allocation-free integral (no counterpart in the reference) ----
 * sum_i mass[i]*u[i] over n nodes into *result, all three device pointers;
 * with mass = the local mass W (x) W (x) W Jac this is GGrid::integrate.
 * For callers that cannot call cudaMalloc where they integrate (a host
 * framework owning device memory through its own pool, a loop that must
 * not stall on an allocation, a deployment that forbids allocation after
 * start-up): nothing is allocated, the scratch is a fixed 256 KB array in
 * the library (held by every GPU that loads it until exit), so n may be at
 * most GF_NOALLOC_MAX_BLOCKS * GF_NOALLOC_CHUNK (134,217,728); larger n is
 * rejected with GF_ERR_ARG.  The first call on a device looks up the
 * array's device address; make it before any stream capture.  Calls share
 * the array: calls that overlap on the GPU race, so order them on one
 * stream.  `stream` is a cudaStream_t (NULL: legacy default stream). */
#define GF_NOALLOC_CHUNK 4096
#define GF_NOALLOC_MAX_BLOCKS 32768
int gf_integrate_noalloc(int64_t n, const double *mass, const double *u, double *result,
                         void *stream);

/* ---- spectral filters (sem/gboyd_filter.ipp, sem/gprojection_filter.ipp) ----
 * gf_filter_matrix: the 1-d filter matrix of order p, column-major
 * F[i + j*(p+1)], as GBoydFilter::init (pdelta: filtered modes above
 * ifilter = p - pdelta, strength mu in [0, 1]) or GProjectionFilter::init
 * (projection to order p - pdelta, 1 <= pdelta <= p/2, blended with
 * strength).  Host only; p = 1 bases are allowed here (the reference's
 * GLLBasis asserts on them).  gf_filter_apply: u_k <- (F3 (x) F2 (x) F1) u_k
 * in every element for the ncomp device fields u (FilterBase::apply in
 * place; the filters' D3_X_D2_X_D1(F, F^T, F^T) with a matrix per direction,
 * F3 ignored in 2-d; GMConv applies its filter list after each step). */
enum { GF_FILTER_BOYD = 0, GF_FILTER_PROJECTION = 1 };
int gf_filter_matrix(int kind, int p, int pdelta, double strength, double *F);
int gf_filter_apply(gf_problem_t prob, int dtype, const double *F1, const double *F2,
                    const double *F3, int ncomp, void *const *u);

/* ---- GIO state files (io/gio.ipp POSIX format) ----
 * One field of one rank per file: the GIO header (io/gio.ipp:459-503)
 * followed by the field's values, straight from / into device memory
 * through pinned double-buffered staging.  Ftype is the dtype (GF_F64:
 * double, GF_F32: float); the header's time is stored as Ftype. */
typedef struct {
  int ivers;             /* 0: one porder row for all elements, else one per element */
  int dim;
  uint64_t nelems;
  int gtype;             /* GElemType: 0 GE_REGULAR, 1 GE_DEFORMED, 2 GE_2DEMBEDDED */
  uint64_t cycle;
  double time;
  int multivar;
  /* filled by the readers */
  int float_bytes;       /* sizeof(Ftype) */
  uint64_t header_bytes; /* GIO::sz_header (io/gio.ipp:676-690) */
  uint64_t ndata;        /* Ftype values after the header (io/gio.ipp:416-429) */
  int64_t porder_rows;   /* 1 if ivers == 0, else nelems */
} gf_gio_header;
/* Header size in bytes for dtype's Ftype, or GF_ERR_ARG. */
int64_t gf_gio_header_bytes(int ivers, int dim, uint64_t nelems, int dtype);
/* The header alone, creating (truncating) path; GIO::write_header_posix
 * (io/gio.ipp:459-503).  ctx may be NULL. */
int gf_gio_write_header(gf_ctx_t ctx, const char *path, const gf_gio_header *h,
                        const int *porder, const uint64_t *elemids, int dtype);
/* n values of device memory u into the existing file path at byte offset
 * (no truncation): one rank's slab of a collective file
 * (GIO::write_coll, io/gio.ipp:735-790) or the data of a POSIX file. */
int gf_gio_write_data(gf_ctx_t ctx, const char *path, int dtype, const void *u, uint64_t n,
                      uint64_t offset);
/* n values from byte offset of path into device memory u (GIO::read_coll's
 * slab read, io/gio.ipp:806-860). */
int gf_gio_read_data(gf_ctx_t ctx, const char *path, int dtype, void *u, uint64_t n,
                     uint64_t offset);
/* GIO::write_posix (io/gio.ipp:347-377): porder is porder_rows x dim
 * int32, elemids nelems keys (NULL: all 0, as GGridBox leaves them); n must
 * equal the count the orders give. */
int gf_gio_write(gf_ctx_t ctx, const char *path, const gf_gio_header *h, const int *porder,
                 const uint64_t *elemids, int dtype, const void *u, uint64_t n);
/* GIO::read_header (io/gio.ipp:587-660).  dtype -1 infers Ftype from the
 * file size.  porder / elemids may be NULL; else they need porder_rows*dim
 * and nelems entries (caps checked).  ctx may be NULL (no device is
 * touched; messages then go to stderr). */
int gf_gio_read_header(gf_ctx_t ctx, const char *path, int dtype, gf_gio_header *h, int *porder,
                       int64_t porder_cap, uint64_t *elemids, int64_t elemids_cap);
/* GIO::read_posix (io/gio.ipp:392-444): reads the n values into device
 * memory u; n must equal the header's count.  hout may be NULL. */
int gf_gio_read(gf_ctx_t ctx, const char *path, int dtype, void *u, uint64_t n,
                gf_gio_header *hout);

/* ---- CUDA graphs (no reference counterpart) ---- */
/* Records nsteps RK steps of gf_rk_advance (same arguments, same result)
 * as a CUDA graph; gf_graph_launch replays them on the problem's stream in
 * one call.  The graph keeps the device pointers u, c and the problem's
 * work buffers: they must outlive it.  The capture uses a library stream,
 * so the context's stream may be the legacy default stream. */
typedef struct gf_graph *gf_graph_t;
int gf_rk_graph_create(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                       void *const *u, const void *const *c, double dt, int nsteps,
                       gf_graph_t *out);
/* One graph holding n graphs of independent problems as concurrent
 * branches (an ensemble advanced by one launch), launched on the stream of
 * parts[0]'s context. */
int gf_graph_ensemble(int n, const gf_graph_t *parts, gf_graph_t *out);
int gf_graph_launch(gf_graph_t g);
int gf_graph_nodes(gf_graph_t g);  /* kernel/copy nodes recorded */
int gf_graph_destroy(gf_graph_t g);

/* ---- adjoint (no reference counterpart) ---- */
/* Vector-Jacobian product of gf_dudt: given u (and c) and a cotangent
 * lam[nstate] on dudt, returns ubar[nstate] = (d dudt/du)^T lam. */
int gf_dudt_vjp(gf_problem_t prob, int dtype, int eqn, double nu, int nstate,
                const void *const *u, const void *const *c,
                const void *const *lam, void *const *ubar);
/* Adjoint of gf_dss (DSS Sum/Smooth are symmetric: each class is reduced
 * with one weight, so the transpose equals the forward map). */
int gf_dss_T(gf_problem_t prob, int dtype, int op, void *u);
/* VJP of one RK step: given the step input u0 and a cotangent lam on the
 * step output, returns (d step/du0)^T lam in lam (in place). */
int gf_rk_step_vjp(gf_problem_t prob, int dtype, const gf_rk_traits *traits,
                   const void *const *u0, const void *const *c, double dt,
                   void *const *lam);
/* Gradient of J = 1/2 ||u(T) - u_obs||_M^2 with respect to u(0) through
 * nsteps RK steps, with a checkpoint every `checkpoint_every` steps and
 * recomputation.  u0, u_obs, grad: device FP64 [nstate][N_local].
 * *J receives the misfit (host). */
int gf_adjoint_gradient(gf_problem_t prob, const gf_rk_traits *traits,
                        const double *const *u0, const double *const *c,
                        const double *const *u_obs, double dt, int nsteps,
                        int checkpoint_every, double *J, double *const *grad);

/* ---- ensembles of independent problems (no reference counterpart: the
 * reference runs one problem per process) ----
 * Up to 64 2-d members of orders 2..9 advanced together, one persistent
 * cooperative launch per RK stage or CG iteration, captured in CUDA graphs.
 * Members are either all deformed / embedded problems (GF_ENS_RK: e.g.
 * icosahedral-sphere advection, each member bit-identical to gf_rk_advance
 * on it alone) or all box problems with affine elements (GF_ENS_CG:
 * Helmholtz solves).  The problems must outlive the ensemble. */
typedef struct gf_ensemble *gf_ensemble_t;
enum { GF_ENS_RK = 0, GF_ENS_CG = 1 };
int gf_ensemble_create(gf_ctx_t ctx, int n, const gf_problem_t *members, gf_ensemble_t *out);
int gf_ensemble_destroy(gf_ensemble_t ens);
/* GF_ENS_RK or GF_ENS_CG */
int gf_ensemble_kind(gf_ensemble_t ens);
/* kernels launched by the ensemble so far (graph launches counted per kernel) */
uint64_t gf_ensemble_launches(gf_ensemble_t ens);
/* Advances member m's state u[m] (device, dtype, N_local) by nsteps step_b
 * steps (GExRKStepper, gexrk_stepper.ipp:252-341) of size dt[m]: traits eqn
 * GF_EQN_ADVECT (velocity c[3*m + k], k < the member's physical
 * coordinates) or GF_EQN_HEAT (c may be NULL), nstate 1, scheme RK1..RK4.
 * Returns GF_ERR_NONFINITE when a member's state is not finite after the
 * last step.  Synchronises; not callable while the stream is captured. */
int gf_ensemble_rk_advance(gf_ensemble_t ens, int dtype, const gf_rk_traits *traits,
                           void *const *u, const void *const *c, const double *dt, int nsteps);
/* Solves (p L + q M) x[m] = b[m] for every member m (device FP64 E-vectors;
 * x holds the initial guess) with the member's Dirichlet mask applied:
 * GCG::solve_impl(A, b, xb, x) with xb = 0 (gcg.ipp:239-382; the masked
 * initial guess, the masked residual; the form without xb masks nothing)
 * with the Jacobi preconditioner.  traits->precision GF_CG_FP64: FP64
 * iterations, GCG's stop test on the recurrence residual.  GF_CG_MIXED: FP32
 * iterations (FP64 dot products) and FP64 residuals: each FP32 run restarts
 * from the FP64 residual once it has reduced its own by inner_tol (default
 * 1e-4); the stop test is on the FP64 residual.  traits: precond GF_PRECOND_JACOBI,
 * normtype EUC or INF, maxit (iterations per member), tol, relative,
 * max_refine (FP64 residual evaluations, default 64).  Per member (host
 * arrays, may be NULL): iterations, the final residual norm, status 0
 * converged / 1 no convergence / 2 breakdown.  Returns 0, GF_CG_NOCONVERGE
 * if any member did not converge, or GF_ERR_NONFINITE.  Synchronises. */
int gf_ensemble_cg_solve(gf_ensemble_t ens, const gf_cg_traits *traits, double p, double q,
                         const double *const *b, double *const *x, int *iters,
                         double *final_norm, int *status);
/* The autotuner: times candidate launch shapes (threads per block, blocks
 * per SM, lanes per element for each order present) on this ensemble's
 * members, with the ensemble's own scratch as the data, and keeps the
 * fastest: best of `reps` launches of the RK stage's element phase (on the
 * equation of the last advance; advection before the first) or of one
 * whole CG iteration.  reps < 0 times the current shape |reps| times and
 * changes nothing (its time is then what gf_ensemble_shape reports). */
int gf_ensemble_tune(gf_ensemble_t ens, int dtype, int reps);
/* The current shape: threads per block, cooperative blocks, lanes per
 * element by GLL point count (team_by_n[n], n <= 10), tuned flag, and the
 * tuner's measured milliseconds per launch of the timed kernel (the RK
 * stage's element phase, or one whole CG iteration; -1 before tuning).
 * Any output may be NULL. */
int gf_ensemble_shape(gf_ensemble_t ens, int dtype, int *threads, int *blocks, int *team_by_n,
                      int *tuned, double *tuned_ms);
/* Sets a shape (threads 64..512, blocks per SM 0 = as many as fit, team
 * widths 8/16/32 by point count, or NULL to keep them). */
int gf_ensemble_set_shape(gf_ensemble_t ens, int dtype, int threads, int blocks_per_sm,
                          const int *team_by_n);

#ifdef __cplusplus
}
#endif
#endif /* GFGPU_H */

// Test infrastructure: a C entry layer over the reference's own spectral-
// element path, compiled from the reference sources into
// oracle/_ref/libgfref{2,3}.so (one library per GDIM, as the reference
// builds one executable per dimension).  It runs, unmodified:
//   GGridBox<Types>       grid construction, geometry, mask, mass
//                         (src/cdg/grid/ggrid_box.ipp, ggrid.ipp)
//   GGFX<double>::init    coordinate matching (src/cdg/comm/ggfx.hpp:169-342)
//   GGFX<double>::doOp    gather-scatter Sum/Smooth/Max/Min (ggfx.hpp:346-443)
//   GHelmholtz::opVec_prod (src/cdg/sem/ghelmholtz.ipp:77-93, 309-378)
//   GAdvect::apply        (src/cdg/sem/gadvect.ipp:58-100)
//   GCG::solve            (src/cdg/solvers/gcg.ipp:239-382)
//   GBurgers + GExRKStepper (src/cdg/pdes/gburgers.ipp, gexrk_stepper.ipp)
// with single-rank Boost stand-ins (oracle/ref/shim).  Only the tests and
// the fixture scripts load it, to pin the C oracle to the reference.
#include <cstdio>
#include <exception>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "gburgers.hpp"
#include "gcg.hpp"
#include "gcomm.hpp"
#include "ggfx.hpp"
#include "ggrid_box.hpp"
#include "ggrid_icos.hpp"
#include "ghelmholtz.hpp"
#include "gllbasis.hpp"
#include "gmass.hpp"
#include "gadvect.hpp"
#include "gtypes.h"
#include "pdeint/lin_solver_base.hpp"
#include "tbox/property_tree.hpp"

using geoflow::tbox::PropertyTree;

GINT szMatCache_ = _G_MAT_CACHE_SIZE;
GINT szVecCache_ = _G_VEC_CACHE_SIZE;

struct RefTypes {
  using State = GTVector<GTVector<GFTYPE> *>;
  using StateComp = GTVector<GFTYPE>;
  using StateInfo = GStateInfo;
  using Grid = GGrid<RefTypes>;
  using GridBox = GGridBox<RefTypes>;
  using GridIcos = GGridIcos<RefTypes>;
  using Mass = GMass<RefTypes>;
  using Ftype = GFTYPE;
  using Derivative = State;
  using Time = Ftype;
  using CompDesc = GTVector<GStateCompType>;
  using Jacobian = State;
  using Size = GSIZET;
  using EqnBase = EquationBase<RefTypes>;
  using EqnBasePtr = std::shared_ptr<EqnBase>;
  using IBdyVol = GTVector<GSIZET>;
  using TBdyVol = GTVector<GBdyType>;
  using Operator = GHelmholtz<RefTypes>;
  using GElemList = GTVector<GElem_base *>;
  using Preconditioner = GHelmholtz<RefTypes>;
  using ConnectivityOp = GGFX<Ftype>;
  using FilterBasePtr = std::shared_ptr<FilterBase<RefTypes>>;
  using FilterList = std::vector<FilterBasePtr>;
};

class RefDiagPrecond;

struct RefCGTypes {
  using Operator = GHelmholtz<RefTypes>;
  using Preconditioner = RefDiagPrecond;
  using State = RefTypes::State;
  using StateComp = RefTypes::StateComp;
  using Grid = GGrid<RefTypes>;
  using Ftype = GFTYPE;
  using ConnectivityOp = GGFX<GFTYPE>;
};

// z = dinv * r: the diagonal (Jacobi) preconditioner handed to the
// reference's GCG through its LinSolverBase preconditioner slot
// (gcg.hpp:71, gcg.ipp:263-268,295-300).  The reference ships no Jacobi
// class; dinv comes from the caller.
class RefDiagPrecond : public LinSolverBase<RefCGTypes> {
 public:
  RefDiagPrecond(Traits &t, GGrid<RefTypes> &g, GGFX<GFTYPE> &x, RefTypes::State &tmp,
                 const double *dinv, size_t n)
      : LinSolverBase<RefCGTypes>(t, g, x, tmp), dinv_(n) {
    for (size_t i = 0; i < n; i++) dinv_[i] = dinv[i];
  }

 protected:
  int solve_impl(const StateComp &b, StateComp &x) override {
    for (size_t i = 0; i < b.size(); i++) x[i] = dinv_[i] * b[i];
    return 0;
  }
  int solve_impl(Operator &, const StateComp &, StateComp &) override { return 2; }
  int solve_impl(Operator &, const StateComp &, const StateComp &, StateComp &) override {
    return 2;
  }

 private:
  GTVector<GFTYPE> dinv_;
};

// 3-d boundary configuration.  The reference's 3-d GGridBox cannot
// configure its boundaries as shipped:
//  * find_gbdy_ind (ggrid_box.ipp:1473-1487) calls find_gbdy_ind2d under
//    _G_IS3D, which asserts on the z faces (bdyid 4, 5);
//  * find_gbdy_ind3d's polygon test geoflow::in_poly (gutils.ipp:323-364)
//    records a point once per polygon edge it lies OUTSIDE of, overrunning
//    its index buffer, and face 1's fourth vertex repeats its first
//    (ggrid_box.ipp:1700-1704);
//  * elem_face_data3d (ggrid_box.ipp:1934-1967, GE_REGULAR branch) reads
//    dXdXi(r, 1) of the (nxy x 1) matrix reg_geom_init sizes
//    (ggrid.ipp:718-719).
// None of this is on the operator path: it only lists the boundary nodes
// (from which GGrid::init_bc_info builds the Dirichlet mask,
// ggrid.ipp:1410-1480) and fills face mass and normals.  So in the 3-d build
// this subclass overrides the two virtuals: config_gbdy lists, per box
// face, the nodes whose coordinate lies on that face (within eps_), typed
// GBDY_PERIODIC or GBDY_DIRICHLET from the configuration, with no update
// objects (homogeneous Dirichlet); elem_face_data uses the in-bounds face
// Jacobian dXdXi(r0,0) * dXdXi(r1,0).  Elements, geometry, mass, mask and
// every operator remain the reference's code.
class RefGridBox : public GGridBox<RefTypes> {
 public:
  using GGridBox<RefTypes>::GGridBox;
#if defined(_G_IS3D)
  int periodic_mask = 0;  // bit d: direction d periodic

  void config_gbdy(const PropertyTree &, GBOOL, GTVector<GTVector<GSIZET>> &igbdyf,
                   GTVector<GTVector<GBdyType>> &igbdyft, GTVector<GSIZET> &igbdy,
                   GTVector<GUINT> &degbdy) override {
    const double eps = 0.125 * this->minnodedist_;
    auto &X = this->xNodes_;
    const size_t n = X[0].size();
    igbdyf.resize(2 * GDIM);
    igbdyft.resize(2 * GDIM);
    this->bdy_update_list_.resize(2 * GDIM);
    std::vector<GSIZET> all;
    for (int f = 0; f < 2 * GDIM; f++) {
      const int d = f / 2;
      const double face = (f & 1) ? this->getP1()[d] : this->getP0()[d];
      std::vector<GSIZET> ids;
      for (size_t i = 0; i < n; i++)
        if (std::fabs(X[d][i] - face) < eps) ids.push_back(i);
      igbdyf[f].resize(ids.size());
      igbdyft[f].resize(ids.size());
      for (size_t k = 0; k < ids.size(); k++) {
        igbdyf[f][k] = ids[k];
        igbdyft[f][k] = ((periodic_mask >> d) & 1) ? GBDY_PERIODIC : GBDY_DIRICHLET;
      }
      all.insert(all.end(), ids.begin(), ids.end());
    }
    igbdy.resize(all.size());
    degbdy.resize(all.size());
    for (size_t k = 0; k < all.size(); k++) {
      igbdy[k] = all[k];
      degbdy[k] = 0;
    }
  }

  void elem_face_data(GTMatrix<GTVector<GFTYPE>> &dXdXi, GTVector<GSIZET> &gieface,
                      GTVector<GFTYPE> &face_mass,
                      GTVector<GTVector<GFTYPE>> &normals) override {
    const unsigned f2r[6][2] = {{0, 2}, {1, 2}, {0, 2}, {1, 2}, {0, 1}, {0, 1}};
    const unsigned f2n[6] = {0, 1, 0, 1, 2, 2};
    size_t nb = 0;
    for (size_t e = 0; e < this->gelems_.size(); e++)
      for (int j = 0; j < this->gelems_[e]->nfaces(); j++)
        nb += this->gelems_[e]->face_indices(j).size();
    gieface.resize(nb);
    face_mass.resize(nb);
    for (size_t k = 0; k < normals.size(); k++) {
      normals[k].resize(nb);
      normals[k] = 0.0;
    }
    nb = 0;
    size_t istart = 0;
    for (size_t e = 0; e < this->gelems_.size(); e++) {
      GTVector<GFTYPE> &fm = this->gelems_[e]->face_mass();
      for (int j = 0; j < this->gelems_[e]->nfaces(); j++) {
        GTVector<GINT> &fi = this->gelems_[e]->face_indices(j);
        const double sgn = (j < 4 || j == 5) ? 1.0 : -1.0;
        for (size_t i = 0; i < fi.size(); i++) {
          const size_t ib = fi[i] + istart;
          gieface[nb] = ib;
          normals[f2n[j]][nb] = sgn;
          face_mass[nb++] = fm[fi[i]] * dXdXi(f2r[j][0], 0)[ib] * dXdXi(f2r[j][1], 0)[ib];
        }
      }
      istart += this->gelems_[e]->nnodes();
    }
  }
#endif
};

namespace {

struct RefBox {
  GTVector<GNBasis<GCTYPE, GFTYPE> *> gbasis;
  GGrid<RefTypes> *grid = nullptr;
  GGFX<GFTYPE> *ggfx = nullptr;
  PropertyTree ptree;
  RefTypes::State utmp;
  size_t ndof = 0;
};

thread_local std::string g_err;

std::string box_json(const int *ne, int p, const double *x0, const double *dx, int periodic,
                     int maxit, double tol) {
  std::ostringstream js;
  js.precision(17);
  js << "{\"grid_type\": \"grid_box\", \"terrain_type\": \"none\", \"exp_order_type\": "
        "\"constant\", \"exp_order\": [";
  for (int d = 0; d < GDIM; d++) js << (d ? ", " : "") << p;
  js << "], \"grid_box\": {\"grid_name\": \"grid_box\", \"xyz0\": [";
  for (int d = 0; d < 3; d++) js << (d ? ", " : "") << (d < GDIM ? x0[d] : 0.0);
  js << "], \"delxyz\": [";
  for (int d = 0; d < 3; d++) js << (d ? ", " : "") << (d < GDIM ? dx[d] : 1.0);
  js << "], \"num_elems\": [";
  for (int d = 0; d < 3; d++) js << (d ? ", " : "") << (d < GDIM ? ne[d] : 1);
  js << "]";
  const char *names[6] = {"bdy_x_0", "bdy_x_1", "bdy_y_0", "bdy_y_1", "bdy_z_0", "bdy_z_1"};
  for (int f = 0; f < 2 * GDIM; f++)
    js << ", \"" << names[f] << "\": \"" << ((periodic >> (f / 2)) & 1 ? "gf_per" : "gf_dir")
       << "\"";
  js << ", \"maxit\": " << maxit << ", \"tol\": " << tol
     << ", \"norm_type\": \"GCG_NORM_INF\"}, "
        "\"gf_per\": {\"bdy_class\": \"uniform\", \"base_type\": [\"GBDY_PERIODIC\"], "
        "\"istate\": [[0, 1, 2]]}, "
        "\"gf_dir\": {\"bdy_class\": \"uniform\", \"base_type\": [\"GBDY_DIRICHLET\"], "
        "\"istate\": [[0, 1, 2]], \"value\": [[0.0, 0.0, 0.0]]}}";
  return js.str();
}

}  // namespace

extern "C" {

int gfr_path_dim(void) { return GDIM; }

const char *gfr_path_error(void) { return g_err.c_str(); }

// A box grid built the way the reference's executable builds it:
// GGridFactory::build (grid/ggrid_factory.ipp:22-60: GGridBox + grid_init),
// then init_ggfx (apps/geoflow_cdg.cpp:731-774): periodize, GGFX::init on
// the node coordinates with max_duplicates() and tolerance
// tol_frac * minnodedist (0.001 there), unperiodize, set_ggfx.
// periodic: bit d set = periodic in direction d, else homogeneous Dirichlet
// on both faces.
void *gfr_box_create(const int *ne, int p, const double *x0, const double *dx, int periodic,
                     double tol_frac) {
  try {
    auto *b = new RefBox;
    b->ptree.load_string(box_json(ne, p, x0, dx, periodic, 512, 1e-8));
    b->gbasis.resize(GDIM);
    for (int d = 0; d < GDIM; d++) b->gbasis[d] = new GLLBasis<GCTYPE, GFTYPE>(p);
    GC_COMM comm = GC_COMM_WORLD;
    auto *gb = new RefGridBox(b->ptree, b->gbasis, comm);
#if defined(_G_IS3D)
    gb->periodic_mask = periodic;
#endif
    b->grid = gb;
    b->grid->grid_init();
    b->ndof = b->grid->ndof();
    gb->periodize();
    const auto nxyz = b->grid->xNodes().size();
    std::vector<std::array<GFTYPE, GGFX<GFTYPE>::NDIM>> xyz(b->ndof);
    for (size_t i = 0; i < b->ndof; i++) {
      for (size_t d = 0; d < GGFX<GFTYPE>::NDIM; d++)
        xyz[i][d] = d < nxyz ? b->grid->xNodes()[d][i] : 0.0;
    }
    gb->unperiodize();
    b->ggfx = new GGFX<GFTYPE>;
    b->ggfx->init(gb->max_duplicates(), tol_frac * b->grid->minnodedist(), xyz);
    b->grid->set_ggfx(*b->ggfx);
    b->utmp.resize(24);
    for (size_t j = 0; j < b->utmp.size(); j++) b->utmp[j] = new GTVector<GFTYPE>(b->ndof);
    return b;
  } catch (std::exception &e) {
    g_err = e.what();
    return nullptr;
  }
}

#if defined(_G_IS2D)
// The 2-d icosahedral sphere of the reference's GGridIcos (GE_2DEMBEDDED):
// base icosahedron refined by refine_type (0: GICOS_BISECTION, 1:
// GICOS_LAGRANGIAN) at level `level`, each triangle split into 3 quads,
// order p, radius r; then GGFX::init on the node coordinates
// (tolerance tol_frac * minnodedist, max_duplicates of the grid).
void *gfr_icos_create(int level, int p, double radius, int refine_type, double tol_frac) {
  try {
    auto *b = new RefBox;
    std::ostringstream js;
    js.precision(17);
    js << "{\"grid_type\": \"grid_icos\", \"terrain_type\": \"none\", "
          "\"exp_order_type\": \"constant\", \"exp_order\": [" << p << ", " << p
       << "], \"grid_icos\": {\"grid_name\": \"grid_icos\", \"ilevel\": " << level
       << ", \"radius\": " << radius << ", \"refine_type\": \""
       << (refine_type == 0 ? "GICOS_BISECTION" : "GICOS_LAGRANGIAN")
       << "\", \"maxit\": 128, \"tol\": 1e-8, \"norm_type\": \"GCG_NORM_INF\"}}";
    b->ptree.load_string(js.str());
    b->gbasis.resize(GDIM);
    for (int d = 0; d < GDIM; d++) b->gbasis[d] = new GLLBasis<GCTYPE, GFTYPE>(p);
    GC_COMM comm = GC_COMM_WORLD;
    auto *gi = new GGridIcos<RefTypes>(b->ptree, b->gbasis, comm);
    b->grid = gi;
    b->grid->grid_init();
    b->ndof = b->grid->ndof();
    const auto nxyz = b->grid->xNodes().size();
    std::vector<std::array<GFTYPE, GGFX<GFTYPE>::NDIM>> xyz(b->ndof);
    for (size_t i = 0; i < b->ndof; i++)
      for (size_t d = 0; d < GGFX<GFTYPE>::NDIM; d++)
        xyz[i][d] = d < nxyz ? b->grid->xNodes()[d][i] : 0.0;
    b->ggfx = new GGFX<GFTYPE>;
    b->ggfx->init(gi->max_duplicates(), tol_frac * b->grid->minnodedist(), xyz);
    b->grid->set_ggfx(*b->ggfx);
    b->utmp.resize(24);
    for (size_t j = 0; j < b->utmp.size(); j++) b->utmp[j] = new GTVector<GFTYPE>(b->ndof);
    return b;
  } catch (std::exception &e) {
    g_err = e.what();
    return nullptr;
  }
}
#endif

// Number of coordinate components (GDIM, or 3 on an embedded surface).
int gfr_nxyz(void *h) { return (int)static_cast<RefBox *>(h)->grid->xNodes().size(); }

// dXi_i/dX_k per node into out[(i * nxy + k) * ndof + n] (i < GDIM,
// k < nxy) and the Jacobian into jac (GGrid::dXidX(), GGrid::Jac()).
// Regular grids store only the diagonal (k = i) planes, the rest are 0.
void gfr_metric(void *h, double *out, double *jac) {
  auto *b = static_cast<RefBox *>(h);
  auto &M = b->grid->dXidX();
  const size_t nxy = b->grid->xNodes().size();
  for (size_t i = 0; i < (size_t)GDIM; i++)
    for (size_t k = 0; k < nxy; k++) {
      double *o = out + (i * nxy + k) * b->ndof;
      const bool have = i < M.size(1) && k < M.size(2);
      for (size_t n = 0; n < b->ndof; n++) o[n] = have && M(i, k).size() ? M(i, k)[n] : 0.0;
    }
  auto &J = b->grid->Jac();
  for (size_t n = 0; n < b->ndof; n++) jac[n] = J[n];
}

size_t gfr_ndof(void *h) { return static_cast<RefBox *>(h)->ndof; }

// Node coordinates, xyz[d*ndof + i].
void gfr_coords(void *h, double *xyz) {
  auto *b = static_cast<RefBox *>(h);
  auto &X = b->grid->xNodes();
  for (size_t d = 0; d < X.size(); d++)
    for (size_t i = 0; i < b->ndof; i++) xyz[d * b->ndof + i] = X[d][i];
}

// Lumped local mass (massop data: W x W (x W) x J) and the Dirichlet mask.
void gfr_mass(void *h, double *m) {
  auto *b = static_cast<RefBox *>(h);
  GTVector<GFTYPE> *mv = b->grid->massop().data();
  for (size_t i = 0; i < b->ndof; i++) m[i] = (*mv)[i];
}

void gfr_mask(void *h, double *m) {
  auto *b = static_cast<RefBox *>(h);
  auto &mk = b->grid->get_mask();
  for (size_t i = 0; i < b->ndof; i++) m[i] = mk[i];
}

void gfr_imult(void *h, double *im) {
  auto *b = static_cast<RefBox *>(h);
  GTVector<GFTYPE> v(b->ndof);
  b->ggfx->get_imult(v);
  for (size_t i = 0; i < b->ndof; i++) im[i] = v[i];
}

// GGFX::doOp in place; op 0 Sum, 1 Smooth, 2 Max, 3 Min.
int gfr_dss(void *h, double *u, int op) {
  auto *b = static_cast<RefBox *>(h);
  GTVector<GFTYPE> v(b->ndof);
  for (size_t i = 0; i < b->ndof; i++) v[i] = u[i];
  GBOOL ok = FALSE;
  switch (op) {
    case 0: ok = b->ggfx->doOp(v, GGFX<GFTYPE>::Sum()); break;
    case 1: ok = b->ggfx->doOp(v, GGFX<GFTYPE>::Smooth()); break;
    case 2: ok = b->ggfx->doOp(v, GGFX<GFTYPE>::Max()); break;
    case 3: ok = b->ggfx->doOp(v, GGFX<GFTYPE>::Min()); break;
    default: return -1;
  }
  for (size_t i = 0; i < b->ndof; i++) u[i] = v[i];
  return ok ? 0 : 1;
}

// GHelmholtz::opVec_prod with p (scalar when np == 1, else per node) and,
// when q != NULL, set_mass_scalar(q) (per node).
int gfr_helmholtz(void *h, const double *u, double *out, const double *p, size_t np,
                  const double *q) {
  auto *b = static_cast<RefBox *>(h);
  GTVector<GFTYPE> vp(np), vq(q ? b->ndof : 1), vu(b->ndof), vo(b->ndof);
  for (size_t i = 0; i < np; i++) vp[i] = p[i];
  for (size_t i = 0; i < b->ndof; i++) vu[i] = u[i];
  GHelmholtz<RefTypes> H(*b->grid);
  H.set_Lap_scalar(vp);
  if (q) {
    for (size_t i = 0; i < b->ndof; i++) vq[i] = q[i];
    H.set_mass_scalar(vq);
  }
  H.init();
  H.opVec_prod(vu, b->utmp, vo);
  for (size_t i = 0; i < b->ndof; i++) out[i] = vo[i];
  return 0;
}

// GAdvect::apply: out = M * sum_j c_j d/dx_j u, c given as one vector per
// physical coordinate (GDIM, or 3 on an embedded surface).
int gfr_advect(void *h, const double *u, const double *c, double *out) {
  auto *b = static_cast<RefBox *>(h);
  const int nc = (int)b->grid->xNodes().size();
  GTVector<GFTYPE> vu(b->ndof), vo(b->ndof);
  std::vector<GTVector<GFTYPE>> cv(nc, GTVector<GFTYPE>(b->ndof));
  RefTypes::State cs(nc);
  for (size_t i = 0; i < b->ndof; i++) vu[i] = u[i];
  for (int d = 0; d < nc; d++) {
    for (size_t i = 0; i < b->ndof; i++) cv[d][i] = c[d * b->ndof + i];
    cs[d] = &cv[d];
  }
  GAdvect<RefTypes> A(*b->grid);
  A.apply(vu, cs, b->utmp, vo);
  for (size_t i = 0; i < b->ndof; i++) out[i] = vo[i];
  return 0;
}

// GCG::solve(A, b, xb, x) with A = GHelmholtz(p scalar, q per node) and,
// when dinv != NULL, the diagonal preconditioner z = dinv * r.
// norm: LinSolverBase::GNormType.  Returns the GCGERR code; iters and the
// per-iteration residual norms (up to maxit) are returned.
int gfr_cg_solve(void *h, double p, const double *q, const double *bvec, const double *xb,
                 double *x, int maxit, double tol, int norm, const double *dinv, int *iters,
                 double *resid) {
  auto *b = static_cast<RefBox *>(h);
  LinSolverBase<RefCGTypes>::Traits tr;
  tr.maxit = maxit;
  tr.tol = tol;
  tr.normtype = static_cast<LinSolverBase<RefCGTypes>::GNormType>(norm);
  GTVector<GFTYPE> vp(1), vq(b->ndof), vb(b->ndof), vxb(b->ndof), vx(b->ndof);
  vp[0] = p;
  for (size_t i = 0; i < b->ndof; i++) {
    vq[i] = q[i];
    vb[i] = bvec[i];
    vxb[i] = xb[i];
    vx[i] = x[i];
  }
  GHelmholtz<RefTypes> H(*b->grid);
  H.set_Lap_scalar(vp);
  H.set_mass_scalar(vq);
  H.init();
  RefTypes::State tmp(10);
  for (size_t j = 0; j < tmp.size(); j++) tmp[j] = b->utmp[j];
  GCG<RefCGTypes> cg(tr, *b->grid, *b->ggfx, tmp);
  std::unique_ptr<RefDiagPrecond> pc;
  if (dinv) {
    RefTypes::State ptmp(2);
    ptmp[0] = b->utmp[10];
    ptmp[1] = b->utmp[11];
    pc.reset(new RefDiagPrecond(tr, *b->grid, *b->ggfx, ptmp, dinv, b->ndof));
    cg.set_precond(*pc);
  }
  int rc = cg.solve(H, vb, vxb, vx);
  for (size_t i = 0; i < b->ndof; i++) x[i] = vx[i];
  *iters = cg.get_iteration_count();
  GTVector<GFTYPE> &r = cg.get_residuals();
  for (int i = 0; i < maxit && i < (int)r.size(); i++) resid[i] = r[i];
  return rc;
}

// GBurgers stepped with its own GExRKStepper, as the reference's
// integrator calls EquationBase::step(t, u, uf, dt) each cycle.
// kind: 0 pure advection (state = [u, c_1..c_GDIM], c prescribed),
//       1 Burgers (state = GDIM velocity components), 2 heat (state = [u]).
// order: time_deriv_order (RK stages); ssp: stab_preserving.
// u: nstate*ndof values, updated in place after nsteps steps of dt.
int gfr_burgers_run(void *h, int kind, double nu, int order, int ssp, double dt, int nsteps,
                    double *u) {
  auto *b = static_cast<RefBox *>(h);
  try {
    GBurgers<RefTypes>::Traits tr;
    tr.doheat = kind == 2;
    tr.bpureadv = kind == 0;
    tr.bconserved = FALSE;
    tr.bforced = FALSE;
    tr.variabledt = FALSE;
    tr.nsolve = (kind == 1) ? GDIM : 1;
    tr.nstate = tr.nsolve + (kind == 0 ? GDIM : 0);
    tr.itorder = order;
    tr.nstage = order;
    tr.bSSP = ssp != 0;
    tr.inorder = 2;
    tr.courant = 0.5;
    tr.nu = nu;
    tr.ssteptype = "GSTEPPER_EXRK";
    // GBurgers keeps a shared_ptr to itself (gburgers.ipp:94), so it owns
    // its own lifetime; it is created once per run and left to the process.
    auto *eq = new GBurgers<RefTypes>(*b->grid, tr);
    // the equation sets its own state size (one velocity per physical
    // coordinate: 3 on an embedded surface); the heat equation reads only
    // its evolved component
    const int nstate = kind == 2 ? 1 : eq->get_traits().nstate;
    const int ntmp = eq->tmp_size() + 4;
    RefTypes::State us(nstate), uf(nstate), tmp(ntmp);
    std::vector<GTVector<GFTYPE> *> owned;
    for (int k = 0; k < nstate; k++) {
      us[k] = new GTVector<GFTYPE>(b->ndof);
      owned.push_back(us[k]);
      for (size_t i = 0; i < b->ndof; i++) (*us[k])[i] = u[k * b->ndof + i];
      uf[k] = NULLPTR;
    }
    for (int j = 0; j < ntmp; j++) {
      tmp[j] = new GTVector<GFTYPE>(b->ndof);
      owned.push_back(tmp[j]);
    }
    eq->init(us, tmp);
    double t = 0.0;
    for (int s = 0; s < nsteps; s++) {
      eq->step(t, us, uf, dt);
      t += dt;
    }
    for (int k = 0; k < nstate; k++)
      for (size_t i = 0; i < b->ndof; i++) u[k * b->ndof + i] = (*us[k])[i];
    for (auto *v : owned) delete v;
    return 0;
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

void gfr_box_destroy(void *h) {
  auto *b = static_cast<RefBox *>(h);
  for (size_t j = 0; j < b->utmp.size(); j++) delete b->utmp[j];
  delete b->ggfx;
  delete b->grid;
  for (size_t d = 0; d < b->gbasis.size(); d++) delete b->gbasis[d];
  delete b;
}

}  // extern "C"

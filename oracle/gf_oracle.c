/*
 * gf_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the GeoFLOW
 * spectral-element hot path.  Each function restates the reference
 * algorithm it cites (paths relative to NOAA-GSL/GeoFLOW src/cdg/) in plain
 * C, keeping the reference's arithmetic order where it is defined, so that
 * FP64 results agree with the reference to rounding.  It is compiled with
 * -ffp-contract=off so that no multiply-add is fused.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, as the checker; the product library never does.
 */
#include "gf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The oracle is serial.  Built with -fopenmp (libgforacle_omp.so, the
 * bench's all-core CPU baseline only) the element, class and node loops
 * below run on every host core; dot products and norms then sum in thread
 * order, so that build is not bit-identical to the serial checker. */
#if defined(_OPENMP)
#define GFO_PRAGMA(x) _Pragma(#x)
#define GFO_PAR GFO_PRAGMA(omp parallel for schedule(static))
#define GFO_PAR_SUM(v) GFO_PRAGMA(omp parallel for schedule(static) reduction(+ : v))
#define GFO_PAR_MAX(v) GFO_PRAGMA(omp parallel for schedule(static) reduction(max : v))
#else
#define GFO_PAR
#define GFO_PAR_SUM(v)
#define GFO_PAR_MAX(v)
#endif

/* ===================================================================== */
/* GLL basis: GLLBasis<long double,double> (sem/gllbasis.ipp)            */
/* ===================================================================== */

/* computeJacobi (gllbasis.ipp:619-670) with alpha = beta = 0. */
static void jacobi(int N, long double x, long double *poly, long double *pder,
                   long double *polym1, long double *pderm1,
                   long double *polym2, long double *pderm2) {
  const long double alpha = 0.0L, beta = 0.0L;
  long double apb = alpha + beta, rv = 1.0L + alpha;
  long double polylist = 0, pderlist = 0, psave = 0, pdsave = 0;
  *poly = 1.0L;
  *pder = 0.0L;
  if (N == 0) return;
  polylist = *poly;
  pderlist = *pder;
  *poly = rv * x;
  *pder = rv;
  if (N == 1) return;
  for (int k = 2; k <= N; k++) {
    long double fk = (long double)k;
    long double a1 = 2.0 * fk * (fk + apb) * (2.0 * fk + apb - 2.0);
    long double a2 = (2.0 * fk + apb - 1.0) * (alpha * alpha - beta * beta);
    long double b3 = 2.0 * fk + apb - 2.0;
    long double a3 = b3 * (b3 + 1.0) * (b3 + 2.0);
    long double a4 = 2.0 * (fk + alpha - 1.0) * (fk + beta - 1.0) * (2.0 * fk + apb);
    long double polyn = ((a2 + a3 * x) * (*poly) - a4 * polylist) / a1;
    long double pdern = ((a2 + a3 * x) * (*pder) - a4 * pderlist + a3 * (*poly)) / a1;
    psave = polylist;
    pdsave = pderlist;
    polylist = *poly;
    *poly = polyn;
    pderlist = *pder;
    *pder = pdern;
  }
  *polym1 = polylist;
  *pderm1 = pderlist;
  *polym2 = psave;
  *pderm2 = pdsave;
}

/* computeNodes (gllbasis.ipp:411-505), computeWeights (515-535) and
 * computeDerivMatrix (580-606), then the cast to double of init()
 * (gllbasis.ipp:715-737).  D is column-major: D[l + j*n]. */
int gfo_gll(int p, double *xi_out, double *w_out, double *D_out) {
  if (p < 1 || p > 64) return -1;
  const int Np = p, np1 = p + 1;
  const long double ximin = -1.0L, ximax = 1.0L, eps = 1.0e-8;
  const long double ttiny = 100.0L * LDBL_EPSILON;
  const int kstop = 128;
  long double xi[65], Pn[65];
  long double pnp1p, pdnp1p, pnp, pdnp, pnm1p, pdnm1, pnp1m, pdnp1m, pnm, pdnm, pnm1m;
  long double d0, d1, d2, d3;

  if (Np == 1) {
    xi[0] = ximin;
    xi[1] = ximax;
  } else {
    jacobi(np1, ximax, &pnp1p, &pdnp1p, &pnp, &pdnp, &pnm1p, &pdnm1);
    jacobi(np1, ximin, &pnp1m, &pdnp1m, &pnm, &pdnm, &pnm1m, &pdnm1);
    long double det = pnp * pnm1m - pnm * pnm1p;
    long double rp = -pnp1p, rm = -pnp1m;
    long double a = (rp * pnm1m - rm * pnm1p) / det;
    long double b = (rm * pnp - rp * pnm) / det;
    xi[0] = ximax;
    xi[Np] = ximin;
    int nh = (Np + 1) / 2;
    /* initial-guess recursion: the quotient is formed in double */
    long double dth = 3.1415926535898 / (2.0 * Np + 1.0);
    long double cd = cosl(2.0 * dth), sd = sinl(2.0 * dth);
    long double cs = cosl(dth), ss = sinl(dth);
    for (int j = 1; j < nh + 1; j++) {
      long double x = cs;
      for (int k = 0; k < kstop; k++) {
        long double pnp1, pdnp1, pn, pdn, pnm1, pdnm1b;
        jacobi(np1, x, &pnp1, &pdnp1, &pn, &pdn, &pnm1, &pdnm1b);
        long double poly = pnp1 + a * pn + b * pnm1;
        long double pder = pdnp1 + a * pdn + b * pdnm1b;
        long double recsum = 0.0;
        for (int i = 0; i < j; i++) recsum += (1.0 / (x - xi[i]));
        long double delx = -poly / (pder - recsum * poly);
        x += delx;
        long double error = fabsl(delx) / fabsl(x);
        if (error < eps) break;
      }
      xi[j] = x;
      long double cssave = cs * cd - ss * sd;
      ss = cs * sd + ss * cd;
      cs = cssave;
    }
    for (int i = 0; i < nh; i++) xi[np1 - i - 1] = -xi[i];
    if (Np == (2 * (Np / 2))) xi[nh] = 0.0;
    for (int i = 0; i < nh; i++) {
      long double t = xi[Np - i];
      xi[Np - i] = xi[i];
      xi[i] = t;
    }
  }
  /* weights: fact is formed in double, as in the reference */
  long double fact = 2.0 / (Np * (Np + 1.0));
  for (int i = 0; i < np1; i++) {
    long double ppn, pder;
    d0 = d1 = d2 = d3 = 0;
    jacobi(Np, xi[i], &ppn, &pder, &d0, &d1, &d2, &d3);
    Pn[i] = ppn;
    long double wi = (Pn[i] == 0.0) ? 0.0L : fact / (Pn[i] * Pn[i]);
    if (w_out) w_out[i] = (double)wi;
    if (xi_out) xi_out[i] = (double)xi[i];
  }
  if (D_out) {
    for (int j = 0; j < np1; j++)
      for (int l = 0; l < np1; l++) {
        long double v = 0.0L;
        if (l != j) {
          long double delxi = xi[l] - xi[j];
          v = Pn[l] / (Pn[j] * delxi + ttiny);
        }
        D_out[l + (size_t)j * np1] = (double)v;
      }
    long double d00 = -0.25 * Np * (Np + 1.0);
    D_out[0] = (double)d00;
    D_out[Np + (size_t)Np * np1] = (double)(-d00);
  }
  return 0;
}

/* ===================================================================== */
/* dmxm contract (blas/cff_blas.F:846-943; blas/dmxmp.F:19-894)          */
/* C(nai,nbj) = A(nai,*) B(nbi,nbj), summed left to right over k.        */
/* ===================================================================== */
void gfo_dmxm(double *C, const double *A, size_t nai, const double *B,
              size_t nbi, size_t nbj) {
  GFO_PAR
  for (size_t j = 0; j < nbj; j++)
    for (size_t i = 0; i < nai; i++) {
      double s = A[i] * B[j * nbi];
      for (size_t k = 1; k < nbi; k++) s = s + A[i + k * nai] * B[k + j * nbi];
      C[i + j * nai] = s;
    }
}

static void fmxm(float *C, const float *A, size_t nai, const float *B,
                 size_t nbi, size_t nbj) {
  for (size_t j = 0; j < nbj; j++)
    for (size_t i = 0; i < nai; i++) {
      float s = A[i] * B[j * nbi];
      for (size_t k = 1; k < nbi; k++) s = s + A[i + k * nai] * B[k + j * nbi];
      C[i + j * nai] = s;
    }
}

/* ===================================================================== */
/* GMTK tensor products (blas/gmtk.ipp)                                  */
/* ===================================================================== */

/* I2_X_D1 (gmtk.ipp:1462-1489): y = D1 . U with U N1 x (N2 Ne). */
void gfo_I2_X_D1(const double *D1, const double *u, size_t N1, size_t N2,
                 size_t Ne, double *y) {
  gfo_dmxm(y, D1, N1, u, N1, N2 * Ne);
}

/* D2_X_I1 (gmtk.ipp:1745-1779): per element y_e = U_e . D2T. */
void gfo_D2_X_I1(const double *D2T, const double *u, size_t N1, size_t N2,
                 size_t Ne, double *y) {
  size_t Nu = N1 * N2;
  GFO_PAR
  for (size_t e = 0; e < Ne; e++) gfo_dmxm(y + e * Nu, u + e * Nu, N1, D2T, N2, N2);
}

/* I3_X_I2_X_D1 (gmtk.ipp:2055-2085): one mxm over all elements. */
void gfo_I3_X_I2_X_D1(const double *D1, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y) {
  gfo_dmxm(y, D1, N1, u, N1, N2 * N3 * Ne);
}

/* I3_X_D2_X_I1 (gmtk.ipp:2155-2197): per element, per k-plane U_k . D2T. */
void gfo_I3_X_D2_X_I1(const double *D2T, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y) {
  size_t NXY = N1 * N2, Nu = N1 * N2 * N3;
  GFO_PAR
  for (size_t e = 0; e < Ne; e++)
    for (size_t k = 0; k < N3; k++)
      gfo_dmxm(y + k * NXY + e * Nu, u + k * NXY + e * Nu, N1, D2T, N2, N2);
}

/* D3_X_I2_X_I1 (gmtk.ipp:2260-2296): per element U (NXY x N3) . D3T. */
void gfo_D3_X_I2_X_I1(const double *D3T, const double *u, size_t N1,
                      size_t N2, size_t N3, size_t Ne, double *y) {
  size_t NXY = N1 * N2, Nu = NXY * N3;
  GFO_PAR
  for (size_t e = 0; e < Ne; e++) gfo_dmxm(y + e * Nu, u + e * Nu, NXY, D3T, N3, N3);
}

/* ===================================================================== */
/* Box grid (grid/ggrid_box.ipp, grid/ggrid.ipp, sem/gelem_base.cpp)     */
/* ===================================================================== */

static size_t elem_nodes(const gfo_grid *g) {
  size_t nn = 1;
  for (int d = 0; d < g->dim; d++) nn *= (size_t)g->n[d];
  return nn;
}

size_t gfo_box_ndof(int dim, const int *ne, const int *p) {
  size_t nd = 1;
  for (int d = 0; d < dim; d++) nd *= (size_t)ne[d] * (size_t)(p[d] + 1);
  return nd;
}

/* find_rank_subdomain (ggrid_box.ipp:860-980) lexicographic element list
 * on one rank; node coordinates from the linear shape functions over the
 * element vertices (do_elems2d/3d, ggrid_box.ipp:250-463); regular-element
 * geometry dXidX = 2/L, Jac = prod(L)/2^dim (gelem_base.cpp:897-1045);
 * mask = 0 on non-periodic boundary nodes (ggrid.ipp:1458-1466). */
void gfo_box_build(int dim, const int *ne, const int *p, const double *x0,
                   const double *len, const int *periodic, double *x,
                   double *y, double *z, double *dXidX0, double *dXidX1,
                   double *dXidX2, double *Jac, double *mask) {
  int n[3] = {1, 1, 1};
  double xi[3][65];
  double dx[3] = {0, 0, 0};
  for (int d = 0; d < dim; d++) {
    n[d] = p[d] + 1;
    gfo_gll(p[d], xi[d], NULL, NULL);
    dx[d] = len[d] / (double)ne[d];
  }
  size_t nelem = 1;
  for (int d = 0; d < dim; d++) nelem *= (size_t)ne[d];
  size_t nn = (size_t)n[0] * n[1] * n[2];
  double *out[3] = {x, y, z};
  double *dxi[3] = {dXidX0, dXidX1, dXidX2};
  const int nv = 1 << dim;
  /* vertex offsets v1..v8 (ggrid_box.ipp:945-952) */
  static const int voff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  const double scale = dim == 2 ? 0.25 : 0.125;
  for (size_t e = 0; e < nelem; e++) {
    int ei[3] = {0, 0, 0};
    size_t r = e;
    for (int d = 0; d < dim; d++) {
      ei[d] = (int)(r % (size_t)ne[d]);
      r /= (size_t)ne[d];
    }
    double v0[3] = {0, 0, 0}, v[8][3] = {{0}}, L[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) v0[d] = x0[d] + ei[d] * dx[d];
    for (int m = 0; m < nv; m++)
      for (int d = 0; d < dim; d++) v[m][d] = voff[m][d] ? v0[d] + dx[d] : v0[d];
    /* L[0] = v2.x1 - v1.x1, L[1] = v3.x2 - v2.x2, L[2] = v5.x3 - v1.x3 */
    L[0] = v[1][0] - v[0][0];
    if (dim > 1) L[1] = v[2][1] - v[1][1];
    if (dim > 2) L[2] = v[4][2] - v[0][2];
    double jac = dim == 2 ? 0.25 * L[0] * L[1] : 0.125 * L[0] * L[1] * L[2];
    for (size_t a = 0; a < nn; a++) {
      int li[3] = {0, 0, 0};
      size_t rr = a;
      for (int d = 0; d < dim; d++) {
        li[d] = (int)(rr % (size_t)n[d]);
        rr /= (size_t)n[d];
      }
      size_t gi = e * nn + a;
      for (int l = 0; l < dim; l++) {
        double acc = 0.0;
        for (int m = 0; m < nv; m++) {
          double Ni = 1.0;
          for (int d = 0; d < dim; d++) {
            double s = voff[m][d] ? 1.0 : -1.0;
            Ni *= (1.0 + s * xi[d][li[d]]);
          }
          acc += Ni * (v[m][l] * scale);
        }
        out[l][gi] = acc;
        if (dxi[l]) dxi[l][gi] = 2.0 / L[l];
      }
      if (Jac) Jac[gi] = jac;
      if (mask) {
        double mk = 1.0;
        for (int d = 0; d < dim; d++) {
          if (periodic[d]) continue;
          if ((ei[d] == 0 && li[d] == 0) || (ei[d] == ne[d] - 1 && li[d] == n[d] - 1)) mk = 0.0;
        }
        mask[gi] = mk;
      }
    }
  }
}

/* GMass::init2d / init3d (gmass.ipp:134-220). */
void gfo_mass(const gfo_grid *g, double *mass) {
  size_t nn = elem_nodes(g), n = 0;
  for (size_t e = 0; e < g->Ne; e++) {
    if (g->dim == 2) {
      for (int k = 0; k < g->n[1]; k++)
        for (int j = 0; j < g->n[0]; j++, n++) mass[n] = g->W[1][k] * g->W[0][j];
    } else {
      for (int l = 0; l < g->n[2]; l++)
        for (int k = 0; k < g->n[1]; k++)
          for (int j = 0; j < g->n[0]; j++, n++)
            mass[n] = g->W[2][l] * g->W[1][k] * g->W[0][j];
    }
  }
  (void)nn;
  for (size_t i = 0; i < n; i++) mass[i] *= g->Jac[i];
}

/* GGrid::integrate (ggrid.ipp:1077-1147), single rank. */
double gfo_integrate(const gfo_grid *g, const double *u) {
  size_t n = 0, nd = g->Ne * elem_nodes(g);
  double *tmp = (double *)malloc(nd * sizeof(double));
  for (size_t e = 0; e < g->Ne; e++) {
    if (g->dim == 2) {
      for (int k = 0; k < g->n[1]; k++)
        for (int j = 0; j < g->n[0]; j++, n++) tmp[n] = g->W[1][k] * g->W[0][j] * u[n];
    } else {
      for (int k = 0; k < g->n[2]; k++)
        for (int j = 0; j < g->n[1]; j++)
          for (int i = 0; i < g->n[0]; i++, n++)
            tmp[n] = g->W[2][k] * g->W[1][j] * g->W[0][i] * u[n];
    }
  }
  double s = 0.0;
  for (size_t i = 0; i < nd; i++) {
    tmp[i] *= g->Jac[i];
    s += tmp[i];
  }
  free(tmp);
  return s;
}

/* ===================================================================== */
/* GGFX (comm/ggfx.hpp)                                                  */
/* ===================================================================== */

typedef struct {
  long long key[3];
  size_t id;
} hnode;

static int cmp_hnode(const void *a, const void *b) {
  const hnode *x = (const hnode *)a, *y = (const hnode *)b;
  for (int d = 0; d < 3; d++) {
    if (x->key[d] < y->key[d]) return -1;
    if (x->key[d] > y->key[d]) return 1;
  }
  return x->id < y->id ? -1 : (x->id > y->id ? 1 : 0);
}

/* tbox::spatial::bound::Intersects for two closed boxes of half-width tol
 * around points a and b. */
static int boxes_intersect(const double *a, const double *b, int dim, double tol) {
  for (int d = 0; d < dim; d++) {
    double amin = a[d] - tol, amax = a[d] + tol, bmin = b[d] - tol, bmax = b[d] + tol;
    if (amax < bmin || bmax < amin) return 0;
  }
  return 1;
}

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* GGFX::init, local part (ggfx.hpp:169-245): for each local id in
 * ascending order that is not yet mapped, query every bound intersecting
 * its bound and make that set the class of every member.  The R-tree query
 * is restated as a bucket search over cells of width 4*tol. */
long gfo_ggfx_init(size_t N, int dim, const double *x, const double *y,
                   const double *z, double tol, int32_t *node_class,
                   int32_t *class_ptr, int32_t *members) {
  const double *c[3] = {x, y, z};
  double cell = 4.0 * tol;
  hnode *h = (hnode *)malloc(N * sizeof(hnode));
  for (size_t i = 0; i < N; i++) {
    for (int d = 0; d < 3; d++) h[i].key[d] = d < dim ? (long long)floor(c[d][i] / cell) : 0;
    h[i].id = i;
  }
  qsort(h, N, sizeof(hnode), cmp_hnode);
  /* set of ids per class stored as a linked list of member ids */
  int32_t *owner = (int32_t *)malloc(N * sizeof(int32_t));  /* class id of node */
  unsigned char *mapped = (unsigned char *)calloc(N, 1);
  int32_t *cand = (int32_t *)malloc(4096 * sizeof(int32_t));
  int32_t *cls_first = (int32_t *)malloc(N * sizeof(int32_t));
  int32_t *cls_size = (int32_t *)malloc(N * sizeof(int32_t));
  int32_t *cls_list = (int32_t *)malloc(N * 64 * sizeof(int32_t));
  size_t nlist = 0, ncls = 0;
  for (size_t i = 0; i < N; i++) owner[i] = -1;
  for (size_t id = 0; id < N; id++) {
    if (mapped[id]) continue;
    double p[3];
    for (int d = 0; d < dim; d++) p[d] = c[d][id];
    long long kc[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) kc[d] = (long long)floor(p[d] / cell);
    int ncand = 0;
    for (int dz = (dim > 2 ? -1 : 0); dz <= (dim > 2 ? 1 : 0); dz++)
      for (int dy = (dim > 1 ? -1 : 0); dy <= (dim > 1 ? 1 : 0); dy++)
        for (int dxx = -1; dxx <= 1; dxx++) {
          hnode probe;
          probe.key[0] = kc[0] + dxx;
          probe.key[1] = kc[1] + dy;
          probe.key[2] = kc[2] + dz;
          probe.id = 0;
          /* lower bound */
          size_t lo = 0, hi = N;
          while (lo < hi) {
            size_t mid = (lo + hi) / 2;
            if (cmp_hnode(&h[mid], &probe) < 0) lo = mid + 1; else hi = mid;
          }
          for (size_t s = lo; s < N && h[s].key[0] == probe.key[0] && h[s].key[1] == probe.key[1] &&
                              h[s].key[2] == probe.key[2]; s++) {
            double q[3];
            for (int d = 0; d < dim; d++) q[d] = c[d][h[s].id];
            if (boxes_intersect(p, q, dim, tol) && ncand < 4096) cand[ncand++] = (int32_t)h[s].id;
          }
        }
    qsort(cand, (size_t)ncand, sizeof(int32_t), cmp_i32);
    cls_first[ncls] = (int32_t)nlist;
    cls_size[ncls] = ncand;
    for (int k = 0; k < ncand; k++) {
      cls_list[nlist++] = cand[k];
      owner[cand[k]] = (int32_t)ncls;
      mapped[cand[k]] = 1;
    }
    ncls++;
  }
  /* A node's reduction buffer holds the values of every set that contains
   * it (ggfx.hpp:401-405); with separated classes that is exactly its own
   * class.  Emit the CSR of the final owner sets. */
  size_t pos = 0, nout = 0;
  int32_t *remap = (int32_t *)malloc(ncls * sizeof(int32_t));
  for (size_t k = 0; k < ncls; k++) remap[k] = -1;
  for (size_t k = 0; k < ncls; k++) {
    /* keep only members still owned by this class */
    int keep = 0;
    for (int m = 0; m < cls_size[k]; m++)
      if (owner[cls_list[cls_first[k] + m]] == (int32_t)k) keep++;
    if (!keep) continue;
    remap[k] = (int32_t)nout;
    class_ptr[nout] = (int32_t)pos;
    for (int m = 0; m < cls_size[k]; m++) {
      int32_t id = cls_list[cls_first[k] + m];
      if (owner[id] == (int32_t)k) {
        members[pos++] = id;
        node_class[id] = (int32_t)nout;
      }
    }
    nout++;
  }
  class_ptr[nout] = (int32_t)pos;
  free(remap);
  free(h);
  free(owner);
  free(mapped);
  free(cand);
  free(cls_first);
  free(cls_size);
  free(cls_list);
  return (long)nout;
}

/* GGFX::doOp (ggfx.hpp:346-443) single rank: every node's buffer holds the
 * values of its class in ascending local id; Sum/Smooth accumulate from 0
 * (std::accumulate), Max/Min fold with std::max/std::min from
 * lowest()/max() (ggfx.hpp:36-76).  Values are all read before any is
 * written. */
void gfo_ggfx_doop(double *u, size_t nclass, const int32_t *class_ptr,
                   const int32_t *members, int op) {
  GFO_PAR
  for (size_t c = 0; c < nclass; c++) {
    int32_t b = class_ptr[c], e = class_ptr[c + 1];
    double acc;
    if (op == GFO_SUM || op == GFO_SMOOTH) {
      acc = 0.0;
      for (int32_t k = b; k < e; k++) acc = acc + u[members[k]];
      if (op == GFO_SMOOTH) acc = acc / (double)(size_t)(e - b);
    } else if (op == GFO_MAX) {
      acc = -DBL_MAX;
      for (int32_t k = b; k < e; k++) {
        double v = u[members[k]];
        acc = (acc < v) ? v : acc;
      }
    } else {
      acc = DBL_MAX;
      for (int32_t k = b; k < e; k++) {
        double v = u[members[k]];
        acc = (v < acc) ? v : acc;
      }
    }
    for (int32_t k = b; k < e; k++) u[members[k]] = acc;
  }
}

void gfo_ggfx_doop_f(float *u, size_t nclass, const int32_t *class_ptr,
                     const int32_t *members, int op) {
  for (size_t c = 0; c < nclass; c++) {
    int32_t b = class_ptr[c], e = class_ptr[c + 1];
    float acc;
    if (op == GFO_SUM || op == GFO_SMOOTH) {
      acc = 0.0f;
      for (int32_t k = b; k < e; k++) acc = acc + u[members[k]];
      if (op == GFO_SMOOTH) acc = acc / (float)(size_t)(e - b);
    } else if (op == GFO_MAX) {
      acc = -FLT_MAX;
      for (int32_t k = b; k < e; k++) {
        float v = u[members[k]];
        acc = (acc < v) ? v : acc;
      }
    } else {
      acc = FLT_MAX;
      for (int32_t k = b; k < e; k++) {
        float v = u[members[k]];
        acc = (v < acc) ? v : acc;
      }
    }
    for (int32_t k = b; k < e; k++) u[members[k]] = acc;
  }
}

/* GGFX::get_mult (ggfx.hpp:453-475). */
void gfo_ggfx_mult(size_t N, size_t nclass, const int32_t *class_ptr,
                   const int32_t *members, double *mult) {
  for (size_t i = 0; i < N; i++) mult[i] = 0.0;
  for (size_t c = 0; c < nclass; c++)
    for (int32_t k = class_ptr[c]; k < class_ptr[c + 1]; k++)
      mult[members[k]] = (double)(class_ptr[c + 1] - class_ptr[c]);
}

/* ===================================================================== */
/* Reference-space derivatives (grid/ggrid.ipp)                          */
/* ===================================================================== */

static void transpose(const double *A, int n, double *AT) {
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) AT[j + i * n] = A[i + j * n];
}

/* Applies the 1-d operator for direction idir (1-based), following
 * grefderiv_varp (ggrid.ipp:2094-2181): direction 1 uses
 * getDerivMatrix(dotrans) through I*_X_D1, directions 2 and 3 use
 * getDerivMatrix(!dotrans) through the right-multiplied forms. */
static void apply_dir(const gfo_grid *g, const double *Dmat, int nd,
                      const double *u, int idir, int dotrans, double *du) {
  double DT[4096];
  transpose(Dmat, nd, DT);
  size_t N1 = g->n[0], N2 = g->n[1], N3 = g->dim > 2 ? g->n[2] : 1;
  const double *Dop;
  if (idir == 1) Dop = dotrans ? DT : Dmat;
  else Dop = dotrans ? Dmat : DT;
  if (g->dim == 2) {
    if (idir == 1) gfo_I2_X_D1(Dop, u, N1, N2, g->Ne, du);
    else gfo_D2_X_I1(Dop, u, N1, N2, g->Ne, du);
  } else {
    if (idir == 1) gfo_I3_X_I2_X_D1(Dop, u, N1, N2, N3, g->Ne, du);
    else if (idir == 2) gfo_I3_X_D2_X_I1(Dop, u, N1, N2, N3, g->Ne, du);
    else gfo_D3_X_I2_X_I1(Dop, u, N1, N2, N3, g->Ne, du);
  }
}

/* compute_grefderiv (ggrid.ipp:2046-2062). */
void gfo_grefderiv(const gfo_grid *g, const double *u, int idir, int dotrans,
                   double *du) {
  apply_dir(g, g->D[idir - 1], g->n[idir - 1], u, idir, dotrans, du);
}

/* compute_grefdiv (ggrid.ipp:1847-1927): divu = 0; divu += D1 u1; ...
 * In 3-d the third operator is taken from basis 1 (ggrid.ipp:1906), which
 * only matters for anisotropic orders; it is kept as in the reference. */
void gfo_grefdiv(const gfo_grid *g, const double *const *u, int dotrans,
                 double *divu) {
  size_t nd = g->Ne * elem_nodes(g);
  double *etmp = (double *)malloc(nd * sizeof(double));
  GFO_PAR
  for (size_t i = 0; i < nd; i++) divu[i] = 0.0;
  for (int k = 0; k < g->dim; k++) {
    if (!u[k]) continue;
    int src = (g->dim == 3 && k == 2) ? 1 : k;
    apply_dir(g, g->D[src], g->n[src], u[k], k + 1, dotrans, etmp);
    GFO_PAR
    for (size_t i = 0; i < nd; i++) divu[i] += etmp[i];
  }
  free(etmp);
}

/* GGrid::deriv (ggrid.ipp:1163-1190), GE_REGULAR branch. */
void gfo_deriv(const gfo_grid *g, const double *u, int idir, double *du) {
  size_t nd = g->Ne * elem_nodes(g);
  gfo_grefderiv(g, u, idir, 0, du);
  for (size_t i = 0; i < nd; i++) du[i] *= g->dXidX[idir - 1][i];
}

/* ===================================================================== */
/* GHelmholtz::reg_prod (sem/ghelmholtz.ipp:309-378), reg_init 531-578    */
/* ===================================================================== */
void gfo_helmholtz(const gfo_grid *g, const double *u, double p_scalar,
                   const double *p_vec, const double *q_vec, double *uo) {
  size_t nd = g->Ne * elem_nodes(g);
  double *gdu[3] = {NULL, NULL, NULL};
  for (int k = 0; k < g->dim; k++) {
    gdu[k] = (double *)malloc(nd * sizeof(double));
    gfo_grefderiv(g, u, k + 1, 0, gdu[k]);
  }
  for (int k = 0; k < g->dim; k++) {
    GFO_PAR
    for (size_t i = 0; i < nd; i++) {
      double G = g->dXidX[k][i] * g->dXidX[k][i];
      gdu[k][i] *= G;
      if (p_vec) gdu[k][i] *= p_vec[i];
      uo[i] = g->mass[i] * gdu[k][i];
      gdu[k][i] = uo[i];
    }
  }
  gfo_grefdiv(g, (const double *const *)gdu, 1, uo);
  if (!p_vec && p_scalar != 1.0) {
    GFO_PAR
    for (size_t i = 0; i < nd; i++) uo[i] *= p_scalar;
  }
  if (q_vec) {
    GFO_PAR
    for (size_t i = 0; i < nd; i++) {
      double t = g->mass[i] * u[i];
      t *= q_vec[i];
      uo[i] += t;
    }
  }
  for (int k = 0; k < g->dim; k++) free(gdu[k]);
}

/* FP32 instantiation of reg_prod on an affine box: gscale[e*(dim+1)+k] =
 * dXidX_k^2 for element e, gscale[e*(dim+1)+dim] = Jac. */
void gfo_helmholtz_f(int dim, size_t Ne, int n, const float *D,
                     const float *W, const float *gscale, float p_scalar,
                     const float *q_vec, const float *u, float *uo) {
  size_t nn = (size_t)n * n * (dim > 2 ? n : 1), nd = Ne * nn;
  float DT[4096];
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) DT[j + i * n] = D[i + j * n];
  float *gdu[3], *mass = (float *)malloc(nd * sizeof(float));
  float *etmp = (float *)malloc(nd * sizeof(float));
  for (size_t e = 0, m = 0; e < Ne; e++)
    for (size_t a = 0; a < nn; a++, m++) {
      size_t i = a % n, j = (a / n) % n, k = a / ((size_t)n * n);
      float w = dim == 2 ? W[j] * W[i] : W[k] * W[j] * W[i];
      mass[m] = w * gscale[e * (dim + 1) + dim];
    }
  for (int k = 0; k < dim; k++) {
    gdu[k] = (float *)malloc(nd * sizeof(float));
    for (size_t e = 0; e < Ne; e++) {
      const float *ue = u + e * nn;
      float *ye = gdu[k] + e * nn;
      if (k == 0) fmxm(ye, D, n, ue, n, nn / n);
      else if (k == 1) {
        if (dim == 2) fmxm(ye, ue, n, DT, n, n);
        else for (int z = 0; z < n; z++) fmxm(ye + z * n * n, ue + z * n * n, n, DT, n, n);
      } else fmxm(ye, ue, (size_t)n * n, DT, n, n);
      float G = gscale[e * (dim + 1) + k];
      for (size_t a = 0; a < nn; a++) ye[a] = mass[e * nn + a] * (ye[a] * G);
    }
  }
  for (size_t i = 0; i < nd; i++) uo[i] = 0.0f;
  for (int k = 0; k < dim; k++) {
    for (size_t e = 0; e < Ne; e++) {
      const float *ge = gdu[k] + e * nn;
      float *ye = etmp + e * nn;
      if (k == 0) fmxm(ye, DT, n, ge, n, nn / n);
      else if (k == 1) {
        if (dim == 2) fmxm(ye, ge, n, D, n, n);
        else for (int z = 0; z < n; z++) fmxm(ye + z * n * n, ge + z * n * n, n, D, n, n);
      } else fmxm(ye, ge, (size_t)n * n, D, n, n);
    }
    for (size_t i = 0; i < nd; i++) uo[i] += etmp[i];
  }
  if (p_scalar != 1.0f)
    for (size_t i = 0; i < nd; i++) uo[i] *= p_scalar;
  if (q_vec)
    for (size_t i = 0; i < nd; i++) {
      float t = mass[i] * u[i];
      t *= q_vec[i];
      uo[i] += t;
    }
  for (int k = 0; k < dim; k++) free(gdu[k]);
  free(mass);
  free(etmp);
}

/* Assembled diagonal of H = p L + q M: sum over directions of
 * D(m,a_d)^2 G_d M(node with a_d -> m), then DSS Sum.  (The reference ships
 * no preconditioner; this is the Jacobi diagonal.) */
void gfo_helmholtz_diag(const gfo_grid *g, double p_scalar,
                        const double *q_vec, size_t nclass,
                        const int32_t *class_ptr, const int32_t *members,
                        double *diag) {
  size_t nn = elem_nodes(g);
  for (size_t e = 0; e < g->Ne; e++)
    for (size_t a = 0; a < nn; a++) {
      int li[3] = {0, 0, 0};
      size_t r = a;
      for (int d = 0; d < g->dim; d++) {
        li[d] = (int)(r % (size_t)g->n[d]);
        r /= (size_t)g->n[d];
      }
      size_t gi = e * nn + a;
      double s = 0.0;
      for (int d = 0; d < g->dim; d++) {
        int nd = g->n[d];
        size_t stride = 1;
        for (int q = 0; q < d; q++) stride *= (size_t)g->n[q];
        for (int m = 0; m < nd; m++) {
          double Dm = g->D[d][m + (size_t)li[d] * nd];
          size_t gb = gi + ((size_t)m - (size_t)li[d]) * stride;
          double G = g->dXidX[d][gb] * g->dXidX[d][gb];
          s += Dm * Dm * G * g->mass[gb];
        }
      }
      s *= p_scalar;
      if (q_vec) s += q_vec[gi] * g->mass[gi];
      diag[gi] = s;
    }
  gfo_ggfx_doop(diag, nclass, class_ptr, members, GFO_SUM);
}

/* ===================================================================== */
/* GAdvect::apply (sem/gadvect.ipp:58-100), regular grid                 */
/* ===================================================================== */
void gfo_advect(const gfo_grid *g, const double *p, int ncomp,
                const double *const *c, double *po) {
  size_t nd = g->Ne * elem_nodes(g);
  double *t = (double *)malloc(nd * sizeof(double));
  gfo_deriv(g, p, 1, po);
  for (size_t i = 0; i < nd; i++) po[i] *= c[0][i];
  for (int j = 1; j < ncomp; j++) {
    gfo_deriv(g, p, j + 1, t);
    for (size_t i = 0; i < nd; i++) {
      t[i] *= c[j][i];
      po[i] += t[i];
    }
  }
  for (size_t i = 0; i < nd; i++) po[i] *= g->mass[i];
  free(t);
}

/* ===================================================================== */
/* GBurgers::dudt_impl (pdes/gburgers.ipp:203-257)                       */
/* ===================================================================== */
void gfo_dudt(const gfo_grid *g, int kind, double nu, const double *imass,
              int nstate, const double *const *u, const double *const *c,
              double *const *dudt) {
  size_t nd = g->Ne * elem_nodes(g);
  double *urhs = (double *)malloc(nd * sizeof(double));
  if (kind == 2) { /* heat */
    for (int k = 0; k < nstate; k++) {
      gfo_helmholtz(g, u[k], nu, NULL, NULL, urhs);
      for (size_t i = 0; i < nd; i++) urhs[i] *= -1.0;
      for (size_t i = 0; i < nd; i++) dudt[k][i] = imass[i] * urhs[i];
    }
  } else if (kind == 0) { /* pure linear advection */
    gfo_advect(g, u[0], g->dim, c, dudt[0]);
    gfo_helmholtz(g, u[0], nu, NULL, NULL, urhs);
    for (size_t i = 0; i < nd; i++) urhs[i] = -1.0 * urhs[i] + -1.0 * dudt[0][i];
    for (size_t i = 0; i < nd; i++) dudt[0][i] = imass[i] * urhs[i];
  } else { /* nonlinear advection */
    for (int k = 0; k < g->dim; k++) {
      gfo_advect(g, u[k], nstate, u, dudt[k]);
      gfo_helmholtz(g, u[k], nu, NULL, NULL, urhs);
      for (size_t i = 0; i < nd; i++) urhs[i] = -1.0 * urhs[i] + -1.0 * dudt[k][i];
      for (size_t i = 0; i < nd; i++) dudt[k][i] = imass[i] * urhs[i];
    }
  }
  free(urhs);
}

/* ===================================================================== */
/* GExRKStepper (pdes/gexrk_stepper.ipp), GButcherRK (gbutcherrk.ipp)     */
/* ===================================================================== */

static void butcher(int order, double *alpha, double beta[4][4], double *c) {
  memset(beta, 0, sizeof(double) * 16);
  for (int i = 0; i < 4; i++) alpha[i] = c[i] = 0.0;
  /* gbutcherrk.ipp:86-125 */
  if (order == 1) {
    alpha[0] = 0;
    c[0] = 1.0;
  } else if (order == 3) {
    alpha[0] = 0; c[0] = 0.25;
    alpha[1] = 1.0 / 3.0; c[1] = 0.0;
    alpha[2] = 2.0 / 3.0; c[2] = 0.75;
    beta[1][0] = 1.0 / 3.0;
    beta[2][1] = 2.0 / 3.0;
  } else if (order == 2) {
    alpha[0] = 0; c[0] = 0.5;
    alpha[1] = 1.0; c[1] = 0.5;
    beta[1][0] = 1.0;
  } else {
    alpha[0] = 0; c[0] = 1.0 / 6.0;
    alpha[1] = 0.5; c[1] = 1.0 / 3.0;
    alpha[2] = 0.5; c[2] = 1.0 / 3.0;
    alpha[3] = 1.0; c[3] = 1.0 / 6.0;
    beta[1][0] = 0.5;
    beta[2][1] = 0.5;
    beta[3][2] = 1.0;
  }
}

static void rhs(const gfo_burgers *b, int nstate, double *const *u, double *const *k) {
  gfo_dudt(b->g, b->kind, b->nu, b->imass, nstate, (const double *const *)u, b->c, k);
}

static void smooth(const gfo_burgers *b, double *v) {
  gfo_ggfx_doop(v, b->nclass, b->class_ptr, b->members, GFO_SMOOTH);
}

/* step_b (1) (gexrk_stepper.ipp:252-341), the live Butcher step. */
static void step_b(const gfo_burgers *b, int order, int nstate,
                   double *const *uin, double dt, double *const *uout, size_t nd) {
  double alpha[4], beta[4][4], c[4];
  butcher(order, alpha, beta, c);
  int nstage = order;
  double h = dt;
  double *u[3], *K[4][3];
  double *isum = (double *)malloc(nd * sizeof(double));
  for (int n = 0; n < nstate; n++) {
    u[n] = (double *)malloc(nd * sizeof(double));
    memcpy(uout[n], uin[n], nd * sizeof(double));
  }
  int nk = nstage - 1 > 1 ? nstage - 1 : 1;
  for (int j = 0; j < nk; j++)
    for (int n = 0; n < nstate; n++) K[j][n] = (double *)malloc(nd * sizeof(double));
  for (int m = 0; m < nstage - 1; m++) {
    for (int n = 0; n < nstate; n++) {
      for (size_t i = 0; i < nd; i++) isum[i] = 0.0;
      for (int j = 0; j < m; j++) {
        double bh = beta[m][j] * h;
        for (size_t i = 0; i < nd; i++) isum[i] = 1.0 * isum[i] + bh * K[j][n][i];
      }
      for (size_t i = 0; i < nd; i++) {
        u[n][i] = uin[n][i];
        u[n][i] += isum[i];
      }
    }
    rhs(b, nstate, u, K[m]);
    for (int n = 0; n < nstate; n++) {
      smooth(b, K[m][n]);
      double ch = c[m] * h;
      for (size_t i = 0; i < nd; i++) {
        isum[i] = K[m][n][i];
        isum[i] *= ch;
        uout[n][i] += isum[i];
      }
    }
  }
  for (int n = 0; n < nstate; n++) {
    for (size_t i = 0; i < nd; i++) isum[i] = 0.0;
    for (int j = 0; j < nstage - 1; j++) {
      double bh = beta[nstage - 1][j] * h;
      for (size_t i = 0; i < nd; i++) isum[i] = 1.0 * isum[i] + bh * K[j][n][i];
    }
    for (size_t i = 0; i < nd; i++) {
      u[n][i] = uin[n][i];
      u[n][i] += isum[i];
    }
    smooth(b, u[n]);
  }
  rhs(b, nstate, u, K[0]);
  for (int n = 0; n < nstate; n++) smooth(b, K[0][n]);
  for (int n = 0; n < nstate; n++) {
    double ch = c[nstage - 1] * h;
    for (size_t i = 0; i < nd; i++) {
      isum[i] = K[0][n][i];
      isum[i] *= ch;
      uout[n][i] += isum[i];
    }
    smooth(b, uout[n]);
  }
  for (int j = 0; j < nk; j++)
    for (int n = 0; n < nstate; n++) free(K[j][n]);
  for (int n = 0; n < nstate; n++) free(u[n]);
  free(isum);
}

/* step_euler (gexrk_stepper.ipp:809-819): uout = dt*RHS(uin) + uin. */
static void euler(const gfo_burgers *b, int nstate, double *const *uin, double dt,
                  double *const *uout, size_t nd) {
  rhs(b, nstate, uin, uout);
  for (int n = 0; n < nstate; n++)
    for (size_t i = 0; i < nd; i++) uout[n][i] = dt * uout[n][i] + 1.0 * uin[n][i];
}

static void axpby(double *x, double a, const double *y, double bcoef, size_t nd) {
  for (size_t i = 0; i < nd; i++) x[i] = a * x[i] + bcoef * y[i];
}

/* step_ssp22 (718-780), step_ssp33 (635-712), step_ssp34 (533-620). */
static void step_ssp(const gfo_burgers *b, int scheme, int nstate,
                     double *const *uin, double dt, double *const *uout, size_t nd) {
  double *K[3][3];
  for (int j = 0; j < 3; j++)
    for (int n = 0; n < nstate; n++) K[j][n] = (double *)malloc(nd * sizeof(double));
  if (scheme == 22) {
    euler(b, nstate, uin, dt, K[0], nd);
    for (int n = 0; n < nstate; n++) smooth(b, K[0][n]);
    euler(b, nstate, K[0], dt, uout, nd);
    for (int n = 0; n < nstate; n++) {
      axpby(uout[n], 0.5, uin[n], 0.5, nd);
      smooth(b, uout[n]);
    }
  } else if (scheme == 33) {
    euler(b, nstate, uin, dt, K[0], nd);
    for (int n = 0; n < nstate; n++) smooth(b, K[0][n]);
    euler(b, nstate, K[0], dt, K[1], nd);
    for (int n = 0; n < nstate; n++) {
      axpby(K[1][n], 0.25, uin[n], 0.75, nd);
      smooth(b, K[1][n]);
    }
    euler(b, nstate, K[1], dt, uout, nd);
    for (int n = 0; n < nstate; n++) {
      axpby(uout[n], 2.0 / 3.0, uin[n], 1.0 / 3.0, nd);
      smooth(b, uout[n]);
    }
  } else { /* 34 */
    euler(b, nstate, uin, dt, K[0], nd);
    for (int n = 0; n < nstate; n++) {
      axpby(K[0][n], 0.5, uin[n], 0.5, nd);
      smooth(b, K[0][n]);
    }
    euler(b, nstate, K[0], dt, K[1], nd);
    for (int n = 0; n < nstate; n++) {
      axpby(K[1][n], 0.5, K[0][n], 0.5, nd);
      smooth(b, K[1][n]);
    }
    euler(b, nstate, K[1], dt, K[2], nd);
    for (int n = 0; n < nstate; n++) {
      axpby(K[2][n], 1.0 / 6.0, K[1][n], 1.0 / 6.0, nd);
      axpby(K[2][n], 1.0, uin[n], 2.0 / 3.0, nd);
      smooth(b, K[2][n]);
    }
    euler(b, nstate, K[2], dt, uout, nd);
    for (int n = 0; n < nstate; n++) {
      axpby(uout[n], 0.5, K[2][n], 0.5, nd);
      smooth(b, uout[n]);
    }
  }
  for (int j = 0; j < 3; j++)
    for (int n = 0; n < nstate; n++) free(K[j][n]);
}

/* GBurgers::step_impl -> step_exrk -> GExRKStepper::step
 * (gburgers.ipp:275-405, gexrk_stepper.ipp:101-114): uold = u; step. */
void gfo_rk_advance(const gfo_burgers *b, int scheme, int nstate,
                    double *const *u, double t0, double dt, int nsteps) {
  const gfo_grid *g = b->g;
  size_t nd = g->Ne * elem_nodes(g);
  double *uold[3];
  (void)t0;
  for (int n = 0; n < nstate; n++) uold[n] = (double *)malloc(nd * sizeof(double));
  for (int s = 0; s < nsteps; s++) {
    for (int n = 0; n < nstate; n++) memcpy(uold[n], u[n], nd * sizeof(double));
    if (scheme >= 1 && scheme <= 4) step_b(b, scheme, nstate, uold, dt, u, nd);
    else step_ssp(b, scheme, nstate, uold, dt, u, nd);
  }
  for (int n = 0; n < nstate; n++) free(uold[n]);
}

/* ===================================================================== */
/* GCG (solvers/gcg.ipp:239-429)                                         */
/* ===================================================================== */

static double cg_norm(const gfo_grid *g, int normtype, const double *x, size_t nd, double ivol) {
  if (normtype == GFO_NORM_INF) {
    double m = 0.0;
    GFO_PAR_MAX(m)
    for (size_t i = 0; i < nd; i++) {
      double a = fabs(x[i]);
      m = m > a ? m : a;
    }
    return m;
  }
  double *t = (double *)malloc(nd * sizeof(double));
  double r;
  if (normtype == GFO_NORM_EUC) {
    double s = 0.0;
    GFO_PAR_SUM(s)
    for (size_t i = 0; i < nd; i++) s += x[i] * x[i];
    r = sqrt(s / (double)nd);
  } else if (normtype == GFO_NORM_L2) {
    for (size_t i = 0; i < nd; i++) t[i] = x[i] * x[i];
    r = sqrt(gfo_integrate(g, t) * ivol);
  } else {
    for (size_t i = 0; i < nd; i++) t[i] = fabs(x[i]);
    r = gfo_integrate(g, t) * ivol;
  }
  free(t);
  return r;
}

int gfo_cg_solve(const gfo_grid *g, double p_scalar, const double *q_vec,
                 const double *mask, size_t nclass, const int32_t *class_ptr,
                 const int32_t *members, const double *dinv,
                 const gfo_cg_traits *tr, const double *b, const double *xb,
                 double *x, int *iters, double *residuals) {
  size_t nd = g->Ne * elem_nodes(g);
  int bbv = xb != NULL;
  double *q = (double *)malloc(nd * sizeof(double));
  double *r = (double *)malloc(nd * sizeof(double));
  double *w = (double *)malloc(nd * sizeof(double));
  double *z = (double *)malloc(nd * sizeof(double));
  double *imult = (double *)malloc(nd * sizeof(double));
  double *ones = (double *)malloc(nd * sizeof(double));
  for (size_t i = 0; i < nd; i++) ones[i] = 1.0;
  ones[0] = 1.0;
  double ivol = 1.0 / gfo_integrate(g, ones);
  gfo_ggfx_mult(nd, nclass, class_ptr, members, imult);
  for (size_t i = 0; i < nd; i++) imult[i] = 1.0 / imult[i];
  /* solve_impl (2) prologue (gcg.ipp:362-382) */
  if (bbv) {
    for (size_t i = 0; i < nd; i++) x[i] *= mask[i];
    for (size_t i = 0; i < nd; i++) x[i] += xb[i];
  }
  int iret = GFO_CG_NONE, iter = 0;
  double alpha, beta, rnorm, rho, rhom, rtol;
  memcpy(r, b, nd * sizeof(double));
  gfo_helmholtz(g, x, p_scalar, NULL, q_vec, w);
  for (size_t i = 0; i < nd; i++) r[i] -= w[i];
  gfo_ggfx_doop(r, nclass, class_ptr, members, GFO_SUM);
  if (bbv) for (size_t i = 0; i < nd; i++) r[i] *= mask[i];
  if (dinv) for (size_t i = 0; i < nd; i++) z[i] = dinv[i] * r[i];
  else memcpy(z, r, nd * sizeof(double));
  memcpy(w, z, nd * sizeof(double));
  rho = 0.0;
  for (size_t i = 0; i < nd; i++) rho += r[i] * z[i] * imult[i];
  rnorm = cg_norm(g, tr->normtype, b, nd, ivol);
  rtol = rnorm < 1.0 ? tr->tol : tr->tol * rnorm;
  rnorm = 10.0 * rtol;
  while (iret == GFO_CG_NONE && iter < tr->maxit && rnorm > rtol) {
    gfo_helmholtz(g, w, p_scalar, NULL, q_vec, q);
    gfo_ggfx_doop(q, nclass, class_ptr, members, GFO_SUM);
    if (bbv) {
      GFO_PAR
      for (size_t i = 0; i < nd; i++) q[i] *= mask[i];
    }
    double wq = 0.0;
    GFO_PAR_SUM(wq)
    for (size_t i = 0; i < nd; i++) wq += w[i] * q[i] * imult[i];
    alpha = rho / wq;
    GFO_PAR
    for (size_t i = 0; i < nd; i++) {
      x[i] = 1.0 * x[i] + alpha * w[i];
      r[i] = 1.0 * r[i] + (-alpha) * q[i];
      z[i] = dinv ? dinv[i] * r[i] : r[i];
    }
    rhom = rho;
    rho = 0.0;
    GFO_PAR_SUM(rho)
    for (size_t i = 0; i < nd; i++) rho += r[i] * z[i] * imult[i];
    beta = rho / rhom;
    GFO_PAR
    for (size_t i = 0; i < nd; i++) w[i] = beta * w[i] + 1.0 * z[i];
    rnorm = cg_norm(g, tr->normtype, r, nd, ivol);
    if (residuals) residuals[iter] = rnorm;
    iter++;
  }
  if (bbv) for (size_t i = 0; i < nd; i++) x[i] *= mask[i];
  if (iret == GFO_CG_NONE && iter >= tr->maxit && rnorm > tr->tol) iret = GFO_CG_NOCONVERGE;
  if (bbv) for (size_t i = 0; i < nd; i++) x[i] += xb[i];
  if (iters) *iters = iter;
  free(q); free(r); free(w); free(z); free(imult); free(ones);
  return iret;
}

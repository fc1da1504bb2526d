// Test infrastructure: a C entry layer over the reference's own
// GLLBasis<GCTYPE,GFTYPE> (src/cdg/sem/gllbasis.ipp) and GMTK tensor
// products (src/cdg/blas/gmtk.ipp), compiled from the reference sources
// into oracle/_ref/libgfref.so.  The tests use it to pin the C oracle.
#include "gllbasis.hpp"
#include "gmtk.hpp"

GINT szMatCache_ = 16;
GINT szVecCache_ = 16;

extern "C" {

// GLL nodes, weights and column-major D(l,j) as getDerivMatrix(FALSE).
int gfr_gll(int p, double *xi, double *w, double *D) {
  GLLBasis<GCTYPE, GFTYPE> b(p);
  GTVector<GFTYPE> *x = b.getXiNodes();
  GTVector<GFTYPE> *ww = b.getWeights();
  GTMatrix<GFTYPE> *d = b.getDerivMatrix(FALSE);
  int n = p + 1;
  for (int i = 0; i < n; i++) { xi[i] = (*x)[i]; w[i] = (*ww)[i]; }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) D[i + j * n] = (*d)(i, j);
  return 0;
}

static void tomat(GTMatrix<GFTYPE> &M, const double *a, size_t n1, size_t n2) {
  M.resize(n1, n2);
  for (size_t j = 0; j < n2; j++)
    for (size_t i = 0; i < n1; i++) M(i, j) = a[i + j * n1];
}

static void tovec(GTVector<GFTYPE> &v, const double *a, size_t n) {
  v.resize(n);
  for (size_t i = 0; i < n; i++) v[i] = a[i];
}

// which: 0 I2_X_D1, 1 D2_X_I1, 2 I3_X_I2_X_D1, 3 I3_X_D2_X_I1,
//        4 D3_X_I2_X_I1, 5 D2_X_D1, 6 D3_X_D2_X_D1.
// A/B/C are the 1-d matrices in the argument order of the GMTK routine.
int gfr_gmtk(int which, const double *A, const double *B, const double *C,
             const size_t *N, size_t Ne, const double *u, double *y) {
  GTMatrix<GFTYPE> MA, MB, MC;
  GTVector<GFTYPE> vu, vy, tmp;
  size_t nn = N[0] * N[1] * (which == 2 || which == 3 || which == 4 || which == 6 ? N[2] : 1);
  tovec(vu, u, nn * Ne);
  vy.resize(nn * Ne);
  tmp.resize(nn * Ne);
  GCBLAS::cuMatBlockDat cudat;
  switch (which) {
    case 0: tomat(MA, A, N[0], N[0]); GMTK::I2_X_D1<GFTYPE>(MA, vu, N[0], N[1], Ne, cudat, vy); break;
    case 1: tomat(MA, A, N[1], N[1]); GMTK::D2_X_I1<GFTYPE>(MA, vu, N[0], N[1], Ne, cudat, vy); break;
    case 2: tomat(MA, A, N[0], N[0]); GMTK::I3_X_I2_X_D1<GFTYPE>(MA, vu, N[0], N[1], N[2], Ne, cudat, vy); break;
    case 3: tomat(MA, A, N[1], N[1]); GMTK::I3_X_D2_X_I1<GFTYPE>(MA, vu, N[0], N[1], N[2], Ne, cudat, vy); break;
    case 4: tomat(MA, A, N[2], N[2]); GMTK::D3_X_I2_X_I1<GFTYPE>(MA, vu, N[0], N[1], N[2], Ne, cudat, vy); break;
    case 5: tomat(MA, A, N[0], N[0]); tomat(MB, B, N[1], N[1]); GMTK::D2_X_D1<GFTYPE>(MA, MB, vu, tmp, vy); break;
    case 6: tomat(MA, A, N[0], N[0]); tomat(MB, B, N[1], N[1]); tomat(MC, C, N[2], N[2]);
            GMTK::D3_X_D2_X_D1<GFTYPE>(MA, MB, MC, vu, tmp, vy); break;
    default: return -1;
  }
  for (size_t i = 0; i < nn * Ne; i++) y[i] = vy[i];
  return 0;
}

// Boyd filter matrix, column-major, as GBoydFilter::init
// (sem/gboyd_filter.ipp:150-200) computes it from the basis' Legendre
// transform: F = L Lambda L^-1 (the compiled Lambda branch).
int gfr_boyd_filter(int p, int pdelta, double strength, double *F) {
  GLLBasis<GCTYPE, GFTYPE> b(p);
  GTMatrix<GFTYPE> *L = b.getLegTransform(), *iL = b.getiLegTransform();
  const int n = p + 1, ifilter = n - pdelta - 1;
  if (!(ifilter > 0 && ifilter < n)) return -1;
  GTMatrix<GFTYPE> Lambda(n, n), tmp(n, n), Fm(n, n);
  Lambda = 0.0;
  for (int i = 0; i < n; i++) {
    Lambda(i, i) = 1.0;
    if (i >= ifilter)
      Lambda(i, i) = strength * pow(fabs((GFTYPE)(i - ifilter) / ((GFTYPE)(n - ifilter))), 2.0);
  }
  tmp = Lambda * (*iL);
  Fm = (*L) * tmp;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) F[i + j * n] = Fm(i, j);
  return 0;
}

// Projection filter matrix, column-major, as GProjectionFilter::init
// (sem/gprojection_filter.ipp:156-202).
int gfr_projection_filter(int p, int pdelta, double strength, double *F) {
  GLLBasis<GCTYPE, GFTYPE> hi(p);
  const int n = p + 1, nlow = n - pdelta;
  if (!(pdelta >= 1 && pdelta <= (n - 1) / 2)) return -1;
  GLLBasis<GCTYPE, GFTYPE> lo(nlow - 1);
  GTVector<GFTYPE> xihi, xilow;
  hi.getXiNodes(xihi);
  lo.getXiNodes(xilow);
  GTMatrix<GFTYPE> Ilow(nlow, n), Ihi(n, nlow), M(n, n), Fm(n, n), Id(n, n);
  Id.createIdentity();
  hi.evalBasis(xilow, Ilow);
  lo.evalBasis(xihi, Ihi);
  M = Ihi * Ilow;
  Fm = M * strength;
  Fm += (Id * (1.0 - strength));
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) F[i + j * n] = Fm(i, j);
  return 0;
}

}  // extern "C"

/* Test infrastructure for the oracle/_ref build.  gfortran is absent, so
 * the Fortran kernels the reference's GMTK calls through its C ABI
 * (cff_blas.h:62,66,108: dmxm/dmxv/fmxm/qmxm) are restated here with the same
 * contract and summation order as cff_blas.F:846-943 and dmxmp.F: the
 * column-major C(nai,nbj) = A(nai,:) B(nbi,nbj), summed left to right. */
#include <stddef.h>
#define MXM(NAME, T)                                                         \
  void NAME(T *C, T *A, size_t *nai, size_t *naj, T *B, size_t *nbi,        \
            size_t *nbj, int *isz) {                                         \
    size_t na = *nai, nb = *nbi, nc = *nbj;                                  \
    (void)naj; (void)isz;                                                    \
    for (size_t j = 0; j < nc; j++)                                          \
      for (size_t i = 0; i < na; i++) {                                      \
        T s = A[i] * B[j * nb];                                              \
        for (size_t k = 1; k < nb; k++) s = s + A[i + k * na] * B[k + j * nb]; \
        C[i + j * na] = s;                                                   \
      }                                                                      \
  }
MXM(dmxm, double)
MXM(fmxm, float)
MXM(qmxm, long double)

/* dmxv (cff_blas.F:1022-1056): y(ny) = A(ny,nx) x(nx), column-major; each
 * y(i) starts at 0 and accumulates A(i,j) x(j) in ascending j (the isz
 * blocking changes no per-row order). */
void dmxv(double *y, double *A, double *x, size_t *nx, size_t *ny, int *isz) {
  size_t m = *ny, n = *nx;
  (void)isz;
  for (size_t i = 0; i < m; i++) {
    double s = 0.0;
    for (size_t j = 0; j < n; j++) s = s + A[i + j * m] * x[j];
    y[i] = s;
  }
}

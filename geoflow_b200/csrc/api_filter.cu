// api_filter.cu -- 1-d matrices of the spectral filters (host).
//
// GBoydFilter::init (sem/gboyd_filter.ipp:150-200), after Giraldo & Rosmond
// (2004):  F = L Lambda L^-1, with L the basis' Legendre transform as
// GLLBasis::computeLegTransform(2) builds it (sem/gllbasis.ipp:783-820) from
// LegMatrix(i, j) = P_i(xi_j) (computeLegendreMatrix, 752-778):
//   L(i, j) = LegMatrix(i, j)                        j < 2
//           = LegMatrix(i, j) - LegMatrix(i, j - 2)  j >= 2
// and Lambda = diag(1 for i < ifilter, strength ((i - ifilter)/(n - ifilter))^2
// for i >= ifilter), ifilter = n - pdelta - 1 (the expression the reference
// compiles, gboyd_filter.ipp:186-189).
// GProjectionFilter::init (sem/gprojection_filter.ipp:156-202):
//   F = strength Ihi Ilow + (1 - strength) I,
// Ilow(i, j) = phi_j^(p)(xi^low_i) interpolates to the GLL nodes of order
// p - pdelta, Ihi(i, j) = phi_j^(p - pdelta)(xi_i) back, with the GLL
// cardinal functions of GLLBasis::evalBasis (1341-1370).
// The filters act along every direction of every element, u <- (F (x) F (x)
// F) u (gf_filter_apply, api_tensor.cu); F is returned column-major like the
// other 1-d operators, F(i, j) = F[i + j n].  Computed in long double.
#include <cfloat>
#include <cmath>
#include <vector>

#include "gf_common.cuh"

namespace {

using LD = long double;

// P_0..P_N at x, and P_N'(x)
void legendre(int N, LD x, std::vector<LD> &P, LD *dPN) {
  P.assign(N + 1, 0.0L);
  P[0] = 1.0L;
  if (N >= 1) P[1] = x;
  for (int k = 2; k <= N; k++) P[k] = ((2 * k - 1) * x * P[k - 1] - (k - 1) * P[k - 2]) / k;
  if (dPN) {  // P_N' from the derivative recurrence
    LD d0 = 0.0L, d1 = 1.0L;
    if (N == 0) {
      *dPN = 0.0L;
    } else {
      for (int k = 2; k <= N; k++) {
        const LD dk = d0 + (2 * k - 1) * P[k - 1];  // P_k' = P_{k-2}' + (2k-1) P_{k-1}
        d0 = d1;
        d1 = dk;
      }
      *dPN = d1;
    }
  }
}

// inverse by Gauss-Jordan with partial pivoting; false when singular
bool invert(int n, std::vector<LD> A, std::vector<LD> &inv) {
  inv.assign((size_t)n * n, 0.0L);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0L;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (fabsl(A[(size_t)r * n + c]) > fabsl(A[(size_t)piv * n + c])) piv = r;
    if (A[(size_t)piv * n + c] == 0.0L) return false;
    if (piv != c)
      for (int k = 0; k < n; k++) {
        std::swap(A[(size_t)piv * n + k], A[(size_t)c * n + k]);
        std::swap(inv[(size_t)piv * n + k], inv[(size_t)c * n + k]);
      }
    const LD d = A[(size_t)c * n + c];
    for (int k = 0; k < n; k++) {
      A[(size_t)c * n + k] /= d;
      inv[(size_t)c * n + k] /= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const LD f = A[(size_t)r * n + c];
      if (f == 0.0L) continue;
      for (int k = 0; k < n; k++) {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
  return true;
}

// GLL cardinal function j of order N (nodes x) at xi (evalBasis (3))
LD cardinal(int N, const std::vector<double> &x, int j, LD xi) {
  const LD tetiny = 100.0L * (LD)DBL_EPSILON;
  if (xi < -1.0L || xi > 1.0L) return 0.0L;
  if (fabsl(xi - (LD)x[j]) <= tetiny) return 1.0L;
  std::vector<LD> P;
  LD dPN = 0.0L, PNj = 0.0L;
  legendre(N, (LD)x[j], P, nullptr);
  PNj = P[N];
  legendre(N, xi, P, &dPN);
  const LD fact = -1.0L / ((LD)N * (N + 1.0L));
  return fact * ((1.0L - xi * xi) / (xi - (LD)x[j])) * dPN / PNj;
}

}  // namespace

extern "C" int gf_filter_matrix(int kind, int p, int pdelta, double strength, double *F) {
  if (p < 1 || p > GF_MAXN - 1 || !F || !(strength >= 0.0 && strength <= 1.0)) return GF_ERR_ARG;
  const int n = p + 1;
  std::vector<double> xi(n);
  if (gf_gll_basis(p, xi.data(), nullptr, nullptr)) return GF_ERR_ARG;
  std::vector<LD> Fm((size_t)n * n, 0.0L);  // row-major F(i, j)
  if (kind == GF_FILTER_BOYD) {
    const int ifilter = n - pdelta - 1;
    if (!(ifilter > 0 && ifilter < n)) return GF_ERR_ARG;
    std::vector<LD> Lm((size_t)n * n), L((size_t)n * n), iL, P;
    for (int j = 0; j < n; j++) {
      legendre(p, (LD)xi[j], P, nullptr);
      for (int i = 0; i < n; i++) Lm[(size_t)i * n + j] = P[i];  // P_i(xi_j)
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        L[(size_t)i * n + j] =
            j < 2 ? Lm[(size_t)i * n + j] : Lm[(size_t)i * n + j] - Lm[(size_t)i * n + j - 2];
    if (!invert(n, L, iL)) return GF_ERR_UNSUPPORTED;
    std::vector<LD> lam(n);
    for (int i = 0; i < n; i++) {
      const LD r = (LD)(i - ifilter) / (LD)(n - ifilter);
      lam[i] = i < ifilter ? 1.0L : (LD)strength * r * r;
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        LD s = 0.0L;
        for (int k = 0; k < n; k++) s += L[(size_t)i * n + k] * lam[k] * iL[(size_t)k * n + j];
        Fm[(size_t)i * n + j] = s;
      }
  } else if (kind == GF_FILTER_PROJECTION) {
    if (!(pdelta >= 1 && pdelta <= (n - 1) / 2)) return GF_ERR_ARG;
    const int nlow = n - pdelta;
    std::vector<double> xl(nlow);
    if (gf_gll_basis(nlow - 1, xl.data(), nullptr, nullptr)) return GF_ERR_ARG;
    std::vector<LD> Ilow((size_t)nlow * n), Ihi((size_t)n * nlow);
    for (int i = 0; i < nlow; i++)
      for (int j = 0; j < n; j++) Ilow[(size_t)i * n + j] = cardinal(p, xi, j, (LD)xl[i]);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < nlow; j++)
        Ihi[(size_t)i * nlow + j] = cardinal(nlow - 1, xl, j, (LD)xi[i]);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        LD s = 0.0L;
        for (int k = 0; k < nlow; k++) s += Ihi[(size_t)i * nlow + k] * Ilow[(size_t)k * n + j];
        Fm[(size_t)i * n + j] = (LD)strength * s + (i == j ? 1.0L - (LD)strength : 0.0L);
      }
  } else {
    return GF_ERR_ARG;
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) F[i + j * n] = (double)Fm[(size_t)i * n + j];
  return GF_OK;
}

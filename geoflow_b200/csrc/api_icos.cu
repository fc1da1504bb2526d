// api_icos.cu -- the 2-d icosahedral sphere of GGridIcos (GE_2DEMBEDDED),
// host-side set-up: node coordinates and the embedded-surface metric that
// the library's GF_GEOM_EMBEDDED problems take as node_geom.
//
// Construction (grid/ggrid_icos.ipp):
//   init2d (134-225)        the base icosahedron: 12 vertices (a vertex at
//                           the pole), 20 faces
//   lagrefine (252-320)     every face cut into rows of sub-triangles
//                           (nrows = 2^level - 1 for GICOS_BISECTION,
//                           level for GICOS_LAGRANGIAN), vertices projected
//                           to the unit sphere, each triangle flagged as
//                           pointing up or down (order_triangles, 2210-2260)
//   do_elems2d (378-515)    3 quadrilaterals per triangle (vertex, edge
//                           midpoints, centroid), vertices projected and
//                           reordered in gnomonic coordinates about the
//                           quad centroid (reorderverts2d, 1925-1970), the
//                           GLL nodes placed by the bilinear map of the 4
//                           vertices and projected to the sphere of `radius`
//   GElem_base::dogeom2d    rij = [dX/dxi, dX/deta, X] (the embedded shape
//     (sem/gelem_base.cpp:  function's third derivative is the position),
//      877-970, Jac/inv     Jac = |det rij| / |X|, dXi/dX = rij^-1
//      1046-1175, 1250-1300)
// The arithmetic follows those steps in their order, including two
// behaviours of the reference's index sort that decide vertex orders:
// GTVector::sortincreasing sorts the values in place with a quicksort
// (gtvector.ipp:2940-3050) while also returning the permutation, and
// order_triangles reads the sorted longitudes through that permutation.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/gfgpu.h"

namespace {

constexpr double kPI = 3.14159265358979323846264338328;

struct P3 {
  double x, y, z;
};
inline P3 operator+(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 operator-(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 operator*(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double norm(P3 a) {
  double s = 0.0;
  s += a.x * a.x;
  s += a.y * a.y;
  s += a.z * a.z;
  return std::sqrt(s);
}

// the point on the sphere of radius rad through p (lat/long round trip)
inline P3 to_sphere(P3 v, double rad) {
  const double r = norm(v);
  const double lat = std::asin(v.z / r);
  double lon = std::atan2(v.y, v.x);
  lon = lon < 0.0 ? 2.0 * kPI + lon : lon;
  return {rad * std::cos(lat) * std::cos(lon), rad * std::cos(lat) * std::sin(lon),
          rad * std::sin(lat)};
}

// quicksort of a[start..end] with the permutation isort, small to large
int64_t partition_s2l(double *a, int64_t *isort, int64_t start, int64_t end) {
  const int64_t pi = start + (end - start) / 2;
  const double pivot = a[pi];
  std::swap(a[pi], a[start]);
  std::swap(isort[pi], isort[start]);
  int64_t i = start + 1, j = end;
  while (i <= j) {
    while (i <= j && a[i] <= pivot) i++;
    while (i <= j && a[j] > pivot) j--;
    if (i < j) {
      std::swap(a[i], a[j]);
      std::swap(isort[i], isort[j]);
    }
  }
  std::swap(a[i - 1], a[start]);
  std::swap(isort[i - 1], isort[start]);
  return i - 1;
}
void quicksort_s2l(double *a, int64_t *isort, int64_t start, int64_t end) {
  if (start >= end) return;
  const int64_t p = partition_s2l(a, isort, start, end);
  quicksort_s2l(a, isort, start, p - 1);
  quicksort_s2l(a, isort, p + 1, end);
}
// values sorted in place, isort the permutation (isort starts as identity)
void sort_increasing(double *a, int64_t *isort, int n) {
  for (int i = 0; i < n; i++) isort[i] = i;
  quicksort_s2l(a, isort, 0, n - 1);
}

struct Tri {
  P3 v[3];
};

// row I of the refinement of triangle (a, b, c) into nrows+1 rows
void row_points(P3 a, P3 b, P3 c, int I, int nrows, std::vector<P3> &R) {
  R.resize(I + 1);
  double fact = 1.0 / (double)(nrows + 1);
  const double xI = (double)I;
  const P3 rL = a + ((b - a) * (xI * fact));
  const P3 rR = a + ((c - a) * (xI * fact));
  fact = I > 0 ? 1.0 / (double)I : 1.0;
  for (int j = 0; j < I + 1; j++) R[j] = rL + ((rR - rL) * ((double)j * fact));
}

// order_triangles: vertex order by longitude, up/down flag from latitude
int order_triangle(Tri &t) {
  P3 cv[3] = {t.v[0], t.v[1], t.v[2]};
  double lon[3], lat[3];
  for (int j = 0; j < 3; j++) {
    const P3 v = cv[j];
    const double r = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    lat[j] = std::asin(v.z / r);
    double l = std::atan2(v.y, v.x);
    lon[j] = l < 0.0 ? 2.0 * kPI + l : l;
  }
  int64_t is[3];
  sort_increasing(lon, is, 3);
  if (std::fabs(lon[is[0]] - lon[is[2]]) < kPI) {
    for (int j = 0; j < 3; j++)
      if (lon[j] > 1.5 * kPI && lon[j] <= 2.0 * kPI) lon[j] -= 2.0 * kPI;
  }
  sort_increasing(lon, is, 3);
  int up = 0;
  if (lat[is[1]] > lat[is[0]] && lat[is[1]] > lat[is[2]]) {
    t.v[0] = cv[is[0]];
    t.v[1] = cv[is[2]];
    t.v[2] = cv[is[1]];
    up = 1;
  }
  if (lat[is[1]] < lat[is[0]] && lat[is[1]] < lat[is[2]]) {
    t.v[0] = cv[is[1]];
    t.v[1] = cv[is[2]];
    t.v[2] = cv[is[0]];
  }
  return up;
}

// reorderverts2d: the quad's vertices in shape-function order, from their
// gnomonic coordinates about the quad centroid
void reorder_quad(const P3 (&u)[4], P3 (&o)[4]) {
  const P3 c = (((u[0] + u[1]) + u[2]) + u[3]) * 0.25;
  const double latc = std::asin(c.z);
  double lonc = std::atan2(c.y, c.x);
  lonc = lonc < 0.0 ? 2 * kPI + lonc : lonc;
  const double eps = 10.0 * 2.220446049250313e-16;
  double gx[4], gy[4];
  for (int i = 0; i < 4; i++) {
    const double r = norm(u[i]);
    const double lat = std::asin(u[i].z / r);
    double lon = std::atan2(u[i].y, u[i].x);
    lon = lon < 0.0 ? 2.0 * kPI + lon : lon;
    double den = std::sin(latc) * std::sin(lat) + std::cos(latc) * std::cos(lat) * std::cos(lon - lonc);
    den = std::fabs(den) < eps ? 0.0 : 1.0 / den;
    gx[i] = 1.0 * std::cos(lat) * std::sin(lon - lonc) * den;
    gy[i] = 1.0 * (std::cos(latc) * std::sin(lat) - std::sin(latc) * std::cos(lat) * std::cos(lon - lonc)) * den;
  }
  double x[4] = {gx[0], gx[1], gx[2], gx[3]};
  int64_t I[4], s[4];
  sort_increasing(x, I, 4);
  if (gy[I[0]] < gy[I[1]]) {
    s[0] = I[0];
    s[3] = I[1];
  } else {
    s[0] = I[1];
    s[3] = I[0];
  }
  if (gy[I[2]] < gy[I[3]]) {
    s[1] = I[2];
    s[2] = I[3];
  } else {
    s[1] = I[3];
    s[2] = I[2];
  }
  for (int j = 0; j < 4; j++) o[j] = u[s[j]];
}

int nrows_of(int level, int refine) {
  if (refine == GF_ICOS_BISECTION) return (1 << level) - 1;
  return level;
}

// base icosahedron of init2d (vertex at the pole), scaled by 1/sqrt(phi^2+1)
void base_mesh(std::vector<Tri> &tb) {
  static const double V[12][3] = {
      {0.000000000000000, 0.000000000000000, 1.000000000000000},
      {0.894427190999916, 0.000000000000000, 0.447213595499958},
      {-0.894427190999916, 0.000000000000000, -0.447213595499958},
      {0.000000000000000, 0.000000000000000, -1.000000000000000},
      {-0.723606797749979, 0.525731112119134, 0.447213595499958},
      {-0.723606797749979, -0.525731112119134, 0.447213595499958},
      {0.723606797749979, 0.525731112119134, -0.447213595499958},
      {0.723606797749979, -0.525731112119134, -0.447213595499958},
      {0.276393202250021, 0.850650808352040, 0.447213595499958},
      {0.276393202250021, -0.850650808352040, 0.447213595499958},
      {-0.276393202250021, 0.850650808352040, -0.447213595499958},
      {-0.276393202250021, -0.850650808352040, -0.447213595499958}};
  static const int F[20][3] = {{0, 1, 8},  {0, 8, 4},   {0, 4, 5},  {0, 5, 9},  {0, 9, 1},
                               {1, 6, 8},  {8, 6, 10},  {8, 10, 4}, {4, 10, 2}, {4, 2, 5},
                               {5, 2, 11}, {5, 11, 9},  {9, 11, 7}, {9, 7, 1},  {1, 7, 6},
                               {3, 6, 7},  {3, 7, 11},  {3, 11, 2}, {3, 2, 10}, {3, 10, 6}};
  const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
  const double fact = 1.0 / std::sqrt(phi * phi + 1.0);
  tb.resize(20);
  for (int i = 0; i < 20; i++)
    for (int j = 0; j < 3; j++) {
      const double *v = V[F[i][j]];
      tb[i].v[j] = {v[0] * fact, v[1] * fact, v[2] * fact};
    }
}

}  // namespace

extern "C" int gf_icos_sizes(int level, int p, int refine, int64_t *nelems, int64_t *nlocal) {
  if (level < 0 || level > 8 || p < 1 || p > 11 ||
      (refine != GF_ICOS_BISECTION && refine != GF_ICOS_LAGRANGIAN))
    return GF_ERR_ARG;
  const int64_t nr = nrows_of(level, refine);
  const int64_t ntri = 20 * (nr * (nr + 2) + 1);
  if (nelems) *nelems = 3 * ntri;
  if (nlocal) *nlocal = 3 * ntri * (int64_t)(p + 1) * (p + 1);
  return GF_OK;
}

extern "C" int gf_icos_grid(int level, int p, double radius, int refine, double *const *xyz,
                            double *node_geom) {
  int64_t ne = 0, nl = 0;
  int rc = gf_icos_sizes(level, p, refine, &ne, &nl);
  if (rc) return rc;
  if (!(radius > 0.0) || !xyz || !xyz[0] || !xyz[1] || !xyz[2]) return GF_ERR_ARG;
  const int nrows = nrows_of(level, refine);
  const int n = p + 1, nn = n * n;
  std::vector<double> xi(n), w(n), D(nn);
  if ((rc = gf_gll_basis(p, xi.data(), w.data(), D.data()))) return rc;

  // lagrefine
  std::vector<Tri> tb, tm;
  base_mesh(tb);
  tm.reserve((size_t)ne / 3);
  std::vector<P3> R0, R1, Rz(2 * (nrows + 1) + 1);
  for (size_t t = 0; t < tb.size(); t++) {
    const P3 a = tb[t].v[0], b = tb[t].v[1], c = tb[t].v[2];
    for (int l = 0; l < nrows + 1; l++) {
      row_points(a, b, c, l, nrows, R0);
      row_points(a, b, c, l + 1, nrows, R1);
      for (int j = 0; j < 2 * l + 3; j++) Rz[j] = (j % 2 == 0) ? R1[j / 2] : R0[(j - 1) / 2];
      for (int m = 0; m < 2 * l + 1; m++) tm.push_back(Tri{{Rz[m], Rz[m + 1], Rz[m + 2]}});
    }
  }
  for (auto &t : tm)
    for (int j = 0; j < 3; j++) t.v[j] = to_sphere(t.v[j], 1.0);
  std::vector<int> up(tm.size());
  for (size_t i = 0; i < tm.size(); i++) up[i] = order_triangle(tm[i]);

  // do_elems2d + dogeom2d
  std::vector<double> X[3];
  for (int k = 0; k < 3; k++) X[k].resize(nn);
  const double third = 1.0 / 3.0;
  int64_t e = 0;
  for (size_t i = 0; i < tm.size(); i++) {
    const P3 v1 = tm[i].v[0], v2 = tm[i].v[1], v3 = tm[i].v[2];
    const P3 ct = (v1 + (v2 + v3)) * third;
    const P3 m12 = (v1 + v2) * 0.5, m13 = (v1 + v3) * 0.5, m23 = (v2 + v3) * 0.5;
    for (int j = 0; j < 3; j++, e++) {
      P3 cv[4];
      if (up[i] == 1) {
        if (j == 0) { cv[0] = v1; cv[1] = m12; cv[2] = ct; cv[3] = m13; }
        else if (j == 1) { cv[0] = m12; cv[1] = v2; cv[2] = m23; cv[3] = ct; }
        else { cv[0] = ct; cv[1] = m23; cv[2] = v3; cv[3] = m13; }
      } else {
        if (j == 0) { cv[0] = v1; cv[1] = m12; cv[2] = ct; cv[3] = m13; }
        else if (j == 1) { cv[0] = ct; cv[1] = m12; cv[2] = v2; cv[3] = m23; }
        else { cv[0] = m13; cv[1] = ct; cv[2] = m23; cv[3] = v3; }
      }
      for (int m = 0; m < 4; m++) cv[m] = to_sphere(cv[m], 1.0);
      P3 gv[4];
      reorder_quad(cv, gv);
      // bilinear map at the GLL nodes (vertex m: (-,-), (+,-), (+,+), (-,+))
      for (int k = 0; k < 3; k++) {
        for (int q = 0; q < nn; q++) X[k][q] = 0.0;
        for (int m = 0; m < 4; m++) {
          const double gvk = (k == 0 ? gv[m].x : (k == 1 ? gv[m].y : gv[m].z)) * 0.25;
          for (int b = 0, q = 0; b < n; b++) {
            const double sm = 1.0 - xi[b], sp = 1.0 + xi[b];
            for (int a = 0; a < n; a++, q++) {
              const double rm = 1.0 - xi[a], rp = 1.0 + xi[a];
              const double Ni = m == 0 ? rm * sm : (m == 1 ? rp * sm : (m == 2 ? rp * sp : rm * sp));
              X[k][q] += Ni * gvk;
            }
          }
        }
      }
      for (int q = 0; q < nn; q++) {
        const double x = X[0][q], y = X[1][q], z = X[2][q];
        const double r = std::sqrt(x * x + y * y + z * z);
        const double lat = std::asin(z / r);
        double lon = std::atan2(y, x);
        lon = lon < 0.0 ? 2.0 * kPI + lon : lon;
        X[0][q] = radius * std::cos(lat) * std::cos(lon);
        X[1][q] = radius * std::cos(lat) * std::sin(lon);
        X[2][q] = radius * std::sin(lat);
      }
      const int64_t base = e * nn;
      for (int k = 0; k < 3; k++) std::memcpy(xyz[k] + base, X[k].data(), sizeof(double) * nn);
      if (!node_geom) continue;
      for (int b = 0, q = 0; b < n; b++)
        for (int a = 0; a < n; a++, q++) {
          double G[3][3];  // G(k, m) = dX_k / dxi_m, m = 2: X_k
          for (int k = 0; k < 3; k++) {
            double s0 = 0.0, s1 = 0.0;
            for (int ii = 0; ii < n; ii++) s0 += D[a + ii * n] * X[k][ii + b * n];
            for (int jj = 0; jj < n; jj++) s1 += D[b + jj * n] * X[k][a + jj * n];
            G[k][0] = s0;
            G[k][1] = s1;
            G[k][2] = X[k][q];
          }
          double det = G[0][0] * (G[1][1] * G[2][2] - G[1][2] * G[2][1]) -
                       G[0][1] * (G[1][0] * G[2][2] - G[1][2] * G[2][0]) +
                       G[0][2] * (G[1][0] * G[2][1] - G[1][1] * G[2][0]);
          const double ij = 1.0 / det;
          const double xr = G[0][2], yr = G[1][2], zr = G[2][2];
          const double jac = std::fabs(det) / std::sqrt(xr * xr + yr * yr + zr * zr);
          // rows 0 and 1 of G^-1: dXi_i/dX_k
          double iG[2][3];
          iG[0][0] = (G[1][1] * G[2][2] - G[1][2] * G[2][1]) * ij;
          iG[0][1] = -(G[0][1] * G[2][2] - G[2][1] * G[0][2]) * ij;
          iG[0][2] = (G[0][1] * G[1][2] - G[0][2] * G[1][1]) * ij;
          iG[1][0] = -(G[1][0] * G[2][2] - G[2][0] * G[1][2]) * ij;
          iG[1][1] = (G[0][0] * G[2][2] - G[2][0] * G[0][2]) * ij;
          iG[1][2] = -(G[0][0] * G[1][2] - G[0][2] * G[1][0]) * ij;
          for (int ii = 0; ii < 2; ii++)
            for (int k = 0; k < 3; k++) node_geom[(int64_t)(ii * 3 + k) * nl + base + q] = iG[ii][k];
          node_geom[(int64_t)6 * nl + base + q] = jac;
        }
    }
  }
  return GF_OK;
}

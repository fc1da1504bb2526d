/* gf_oracle_def.c -- CPU oracle (test infrastructure only) for deformed
 * (GE_DEFORMED) and 2-d embedded (GE_2DEMBEDDED) elements: the metric of
 * GHelmholtz::def_init, def_prod / embed_prod, the deformed branch of
 * GGrid::deriv, GAdvect::apply with nxy velocity components, the Burgers
 * right-hand side built from them, and GMTK::constrain2sphere (2).
 * Plain C, -ffp-contract=off, operations in the reference's order. */
#include <stdlib.h>
#include <string.h>

#include "gf_oracle.h"

static size_t nodes_per_elem(const gfo_grid *g) {
  size_t nn = 1;
  for (int d = 0; d < g->dim; d++) nn *= (size_t)g->n[d];
  return nn;
}

/* ghelmholtz.ipp:416-519 (formula of its comment; see the header). */
void gfo_def_metric(const gfo_defgrid *g, double *const G[3][3]) {
  const gfo_grid *b = g->base;
  const int dim = b->dim;
  const size_t nn = nodes_per_elem(b);
  for (int i = 0; i < dim; i++)
    for (int j = 0; j < dim; j++) memset(G[i][j], 0, b->Ne * nn * sizeof(double));
  for (size_t e = 0; e < b->Ne; e++)
    for (size_t a = 0; a < nn; a++) {
      const size_t node = e * nn + a;
      const int l = (int)(a % b->n[0]), m = (int)((a / b->n[0]) % b->n[1]);
      const int pz = dim > 2 ? (int)(a / ((size_t)b->n[0] * b->n[1])) : 0;
      for (int j = 0; j < dim; j++)
        for (int i = j; i < dim; i++) {
          double s = G[i][j][node];
          for (int k = 0; k < g->nxy; k++) {
            double t = g->X[i][k][node] * g->X[j][k][node] * b->W[0][l] * b->W[1][m];
            if (dim > 2) t = t * b->W[2][pz];
            s += t * b->Jac[node];
          }
          G[i][j][node] = s;
          G[j][i][node] = s;
        }
    }
}

/* ghelmholtz.ipp:109-191 (def_prod) and 207-293 (embed_prod). */
void gfo_def_helmholtz(const gfo_defgrid *g, const double *const G[3][3], const double *u,
                       double p_scalar, const double *p_vec, const double *q_vec,
                       double *uo) {
  const gfo_grid *b = g->base;
  const int dim = b->dim;
  const size_t nd = b->Ne * nodes_per_elem(b);
  double *du[3] = {NULL, NULL, NULL}, *gdu[3] = {NULL, NULL, NULL};
  for (int i = 0; i < dim; i++) {
    du[i] = (double *)malloc(nd * sizeof(double));
    gdu[i] = (double *)malloc(nd * sizeof(double));
    gfo_grefderiv(b, u, i + 1, 0, du[i]);
  }
  for (int j = 0; j < dim; j++) {
    for (size_t n = 0; n < nd; n++) gdu[j][n] = 0.0;
    for (int i = 0; i < dim; i++)
      for (size_t n = 0; n < nd; n++) {
        double t = du[i][n] * G[i][j][n];
        gdu[j][n] += t;
      }
    if (p_vec)
      for (size_t n = 0; n < nd; n++) gdu[j][n] *= p_vec[n];
  }
  gfo_grefdiv(b, (const double *const *)gdu, 1, uo);
  if (!p_vec && p_scalar != 1.0)
    for (size_t n = 0; n < nd; n++) uo[n] *= p_scalar;
  if (q_vec)
    for (size_t n = 0; n < nd; n++) {
      double t = b->mass[n] * u[n];
      t *= q_vec[n];
      uo[n] += t;
    }
  for (int i = 0; i < dim; i++) {
    free(du[i]);
    free(gdu[i]);
  }
}

/* ggrid.ipp:1177-1186 */
void gfo_def_deriv(const gfo_defgrid *g, const double *u, int idir, double *du) {
  const gfo_grid *b = g->base;
  const size_t nd = b->Ne * nodes_per_elem(b);
  double *t = (double *)malloc(nd * sizeof(double));
  gfo_grefderiv(b, u, 1, 0, du);
  for (size_t n = 0; n < nd; n++) du[n] *= g->X[0][idir - 1][n];
  for (int j = 1; j < b->dim; j++) {
    gfo_grefderiv(b, u, j + 1, 0, t);
    for (size_t n = 0; n < nd; n++) {
      t[n] *= g->X[j][idir - 1][n];
      du[n] += t[n];
    }
  }
  free(t);
}

/* gadvect.ipp:58-100 */
void gfo_def_advect(const gfo_defgrid *g, const double *p, const double *const *c,
                    double *po) {
  const gfo_grid *b = g->base;
  const size_t nd = b->Ne * nodes_per_elem(b);
  double *t = (double *)malloc(nd * sizeof(double));
  gfo_def_deriv(g, p, 1, po);
  for (size_t n = 0; n < nd; n++) po[n] *= c[0][n];
  for (int j = 1; j < g->nxy; j++) {
    gfo_def_deriv(g, p, j + 1, t);
    for (size_t n = 0; n < nd; n++) {
      t[n] *= c[j][n];
      po[n] += t[n];
    }
  }
  for (size_t n = 0; n < nd; n++) po[n] *= b->mass[n];
  free(t);
}

/* gburgers.ipp:203-257 on the deformed operators */
void gfo_def_dudt(const gfo_defgrid *g, const double *const G[3][3], int kind, double nu,
                  const double *imass, int nstate, const double *const *u,
                  const double *const *c, double *const *dudt) {
  const gfo_grid *b = g->base;
  const size_t nd = b->Ne * nodes_per_elem(b);
  double *urhs = (double *)malloc(nd * sizeof(double));
  for (int k = 0; k < nstate; k++) {
    gfo_def_helmholtz(g, G, u[k], nu, NULL, NULL, urhs);
    if (kind == 2) {
      for (size_t n = 0; n < nd; n++) urhs[n] *= -1.0;
    } else {
      gfo_def_advect(g, u[k], kind == 0 ? c : u, dudt[k]);
      for (size_t n = 0; n < nd; n++) urhs[n] = -1.0 * urhs[n] + -1.0 * dudt[k][n];
    }
    for (size_t n = 0; n < nd; n++) dudt[k][n] = imass[n] * urhs[n];
  }
  free(urhs);
}

/* gmtk.ipp:2957-2976 */
void gfo_constrain2sphere(size_t N, const double *const *xyz, double *const *v) {
  if (N == 0) return;
  double x = xyz[0][0], y = xyz[1][0], z = xyz[2][0];
  const double r2 = x * x + y * y + z * z;
  const double ri = 1.0 / r2;
  for (size_t j = 0; j < N; j++) {
    x = xyz[0][j];
    y = xyz[1][j];
    z = xyz[2][j];
    v[0][j] = (v[0][j] * (r2 - x * x) - v[1][j] * x * y - v[2][j] * x * z) * ri;
    v[1][j] = (-v[0][j] * y * x + v[1][j] * (r2 - y * y) - v[2][j] * y * z) * ri;
    v[2][j] = (-v[0][j] * z * x - v[1][j] * z * y + v[2][j] * (r2 - z * z)) * ri;
  }
}

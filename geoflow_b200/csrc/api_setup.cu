// api_setup.cu -- context lifetime, host-side set-up helpers (GLL basis,
// box grid, gather-scatter classes) and problem creation.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <numeric>

#include "gf_common.cuh"

// ---------------------------------------------------------------------
// errors and scratch
// ---------------------------------------------------------------------
int gf_fail(gf_context *ctx, int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->last_error = buf;
  else fprintf(stderr, "gfgpu: %s\n", buf);
  return code;
}

namespace gfk {
// K1(l,m) = sum_i D(i,l) W_i D(i,m), D(i,m) = D[i + m*n], accumulated in
// long double, then averaged with its centro-reflection K1(n-1-l, n-1-m)
// (equal in exact arithmetic) so that the even-odd form is exact.
void gf_k1_matrix(int n, const double *D, const double *W, double *K1) {
  std::vector<long double> K((size_t)n * n);
  for (int l = 0; l < n; l++)
    for (int m = 0; m < n; m++) {
      long double s = 0.0L;
      for (int i = 0; i < n; i++)
        s += ((long double)D[i + l * n] * (long double)D[i + m * n]) * (long double)W[i];
      K[l + m * n] = s;
    }
  for (int l = 0; l < n; l++)
    for (int m = 0; m < n; m++)
      K1[l + m * n] = (double)(0.5L * (K[l + m * n] + K[(n - 1 - l) + (n - 1 - m) * n]));
}
}  // namespace gfk

void *gf_work(gf_problem *prob, int slot, size_t bytes) {
  if ((int)prob->work.size() <= slot) prob->work.resize(slot + 1);
  gf_buffer &b = prob->work[slot];
  if (b.bytes < bytes) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    if (cudaMalloc(&b.ptr, bytes) != cudaSuccess) return nullptr;
    b.bytes = bytes;
  }
  return b.ptr;
}

extern "C" int gf_abi_version(void) { return GFGPU_ABI_VERSION; }

extern "C" int gf_ctx_create(int device, void *stream, gf_ctx_t *out) {
  if (!out) return GF_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || device < 0 || device >= ndev)
    return gf_fail(nullptr, GF_ERR_CUDA, "no CUDA device %d (%s)", device,
                   e == cudaSuccess ? "out of range" : cudaGetErrorString(e));
  if (cudaSetDevice(device) != cudaSuccess) return GF_ERR_CUDA;
  gf_context *ctx = new gf_context();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  // NULL selects the legacy default stream, which orders the library's
  // work with every other blocking stream of the process (torch's default)
  ctx->stream = (cudaStream_t)stream;
  ctx->own_stream = false;
  *out = ctx;
  return GF_OK;
}

extern "C" int gf_ctx_destroy(gf_ctx_t ctx) {
  if (!ctx) return GF_ERR_ARG;
  if (ctx->nprob > 0) {  // freed with its last problem
    ctx->destroy_pending = true;
    return GF_OK;
  }
  cudaSetDevice(ctx->device);
  if (ctx->own_stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return GF_OK;
}

extern "C" const char *gf_ctx_last_error(gf_ctx_t ctx) {
  if (!ctx) return "null context";
  ctx->returned_error = ctx->last_error;
  ctx->last_error.clear();
  return ctx->returned_error.c_str();
}

extern "C" int gf_ctx_synchronize(gf_ctx_t ctx) {
  if (!ctx) return GF_ERR_ARG;
  GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GF_OK;
}

// ---------------------------------------------------------------------
// GLL basis.  The construction follows GLLBasis<long double,double>
// (sem/gllbasis.ipp): Legendre values by the three-term recurrence
// (computeJacobi, 619-670), interior nodes by Newton iteration with
// deflation from Chebyshev-like starting points (computeNodes, 411-505),
// weights 2/(N(N+1) P_N^2) (515-535), D(l,j) = P_N(l)/(P_N(j)(x_l-x_j)+tiny)
// with D(0,0) = -D(N,N) = -N(N+1)/4 (580-606); all in long double, then
// rounded to double.  Matching the reference's constants and order makes
// the doubles bit-identical to the reference's.
// ---------------------------------------------------------------------
namespace {
struct Leg {
  long double p, dp, pm1, dpm1;  // P_N, P_N', P_{N-1}, P'_{N-1}
};

Leg legendre(int N, long double x) {
  Leg r{1.0L, 0.0L, 0.0L, 0.0L};
  if (N == 0) return r;
  long double p0 = 1.0L, d0 = 0.0L, p1 = x, d1 = 1.0L;
  if (N == 1) return Leg{p1, d1, p0, d0};
  for (int k = 2; k <= N; k++) {
    long double fk = (long double)k;
    long double a1 = 2.0 * fk * fk * (2.0 * fk - 2.0);
    long double b3 = 2.0 * fk - 2.0;
    long double a3 = b3 * (b3 + 1.0) * (b3 + 2.0);
    long double a4 = 2.0 * (fk - 1.0) * (fk - 1.0) * (2.0 * fk);
    long double a2 = (2.0 * fk - 1.0) * 0.0L;
    long double pn = ((a2 + a3 * x) * p1 - a4 * p0) / a1;
    long double dn = ((a2 + a3 * x) * d1 - a4 * d0 + a3 * p1) / a1;
    p0 = p1; d0 = d1; p1 = pn; d1 = dn;
  }
  return Leg{p1, d1, p0, d0};
}
}  // namespace

extern "C" int gf_gll_basis(int p, double *xi_out, double *w_out, double *D_out) {
  if (p < 1 || p > 32) return GF_ERR_ARG;
  const int N = p, n = p + 1;
  std::vector<long double> x(n), PN(n);
  if (N == 1) {
    x[0] = -1.0L;
    x[1] = 1.0L;
  } else {
    // combination of P_{N+1}, P_N, P_{N-1} vanishing at +-1
    Leg hp = legendre(N + 1, 1.0L), hm = legendre(N + 1, -1.0L);
    long double pnp1p = hp.p, pnp = hp.pm1, pnp1m = hm.p, pnm = hm.pm1;
    long double pnm1p = legendre(N - 1, 1.0L).p, pnm1m = legendre(N - 1, -1.0L).p;
    long double det = pnp * pnm1m - pnm * pnm1p;
    long double rp = -pnp1p, rm = -pnp1m;
    long double ca = (rp * pnm1m - rm * pnm1p) / det;
    long double cb = (rm * pnp - rp * pnm) / det;
    std::vector<long double> r(n);
    r[0] = 1.0L;
    r[N] = -1.0L;
    const int nh = (N + 1) / 2;
    long double th = 3.1415926535898 / (2.0 * N + 1.0);
    long double c2 = cosl(2.0 * th), s2 = sinl(2.0 * th), c1 = cosl(th), s1 = sinl(th);
    for (int j = 1; j <= nh; j++) {
      long double xx = c1;
      for (int it = 0; it < 128; it++) {
        Leg a = legendre(N + 1, xx);
        Leg b = legendre(N - 1, xx);
        // P_{N} and P'_{N} at xx come with the N+1 evaluation
        long double f = a.p + ca * a.pm1 + cb * b.p;
        long double fd = a.dp + ca * a.dpm1 + cb * b.dp;
        long double defl = 0.0;
        for (int i = 0; i < j; i++) defl += (1.0 / (xx - r[i]));
        long double step = -f / (fd - defl * f);
        xx += step;
        if (fabsl(step) / fabsl(xx) < 1.0e-8) break;
      }
      r[j] = xx;
      long double cn = c1 * c2 - s1 * s2;
      s1 = c1 * s2 + s1 * c2;
      c1 = cn;
    }
    for (int i = 0; i < nh; i++) r[n - i - 1] = -r[i];
    if (N % 2 == 0) r[nh] = 0.0;
    for (int i = 0; i < nh; i++) std::swap(r[N - i], r[i]);
    x = r;
  }
  long double fact = 2.0 / (N * (N + 1.0));
  for (int i = 0; i < n; i++) {
    PN[i] = legendre(N, x[i]).p;
    if (xi_out) xi_out[i] = (double)x[i];
    if (w_out) w_out[i] = (double)(PN[i] == 0.0 ? 0.0L : fact / (PN[i] * PN[i]));
  }
  if (D_out) {
    const long double tiny = 100.0L * LDBL_EPSILON;
    for (int j = 0; j < n; j++)
      for (int l = 0; l < n; l++)
        D_out[l + j * n] = (l == j) ? 0.0 : (double)(PN[l] / (PN[j] * (x[l] - x[j]) + tiny));
    long double d00 = -0.25 * N * (N + 1.0);
    D_out[0] = (double)d00;
    D_out[N + N * n] = (double)(-d00);
  }
  return GF_OK;
}

// ---------------------------------------------------------------------
// Box grid (GGridBox): lexicographic elements, x fastest
// ---------------------------------------------------------------------
extern "C" int gf_box_grid(int dim, const int *ne, int p, const double *x0, const double *len,
                           const int *periodic, double *const *xyz, double *elem_geom,
                           double *mask) {
  if ((dim != 2 && dim != 3) || !ne || !x0 || !len || p < 1 || p > 32) return GF_ERR_ARG;
  const int n = p + 1;
  std::vector<double> xi(n);
  gf_gll_basis(p, xi.data(), nullptr, nullptr);
  int64_t nelem = 1, nn = 1;
  double h[3] = {0, 0, 0};
  for (int d = 0; d < dim; d++) {
    if (ne[d] < 1) return GF_ERR_ARG;
    nelem *= ne[d];
    nn *= n;
    h[d] = len[d] / (double)ne[d];
  }
  // vertex offsets in the GGridBox hex/quad order (ggrid_box.ipp:945-952)
  static const int voff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  const int nv = 1 << dim;
  const double vscale = dim == 2 ? 0.25 : 0.125;
  for (int64_t e = 0; e < nelem; e++) {
    int ei[3] = {0, 0, 0};
    int64_t r = e;
    for (int d = 0; d < dim; d++) {
      ei[d] = (int)(r % ne[d]);
      r /= ne[d];
    }
    double v[8][3] = {{0}};
    for (int m = 0; m < nv; m++)
      for (int d = 0; d < dim; d++) {
        double lo = x0[d] + ei[d] * h[d];
        v[m][d] = voff[m][d] ? lo + h[d] : lo;
      }
    double L[3] = {v[1][0] - v[0][0], dim > 1 ? v[2][1] - v[1][1] : 1.0,
                   dim > 2 ? v[4][2] - v[0][2] : 1.0};
    if (elem_geom) {
      for (int d = 0; d < dim; d++) elem_geom[e * (dim + 1) + d] = 2.0 / L[d];
      elem_geom[e * (dim + 1) + dim] = dim == 2 ? 0.25 * L[0] * L[1] : 0.125 * L[0] * L[1] * L[2];
    }
    for (int64_t a = 0; a < nn; a++) {
      int li[3] = {0, 0, 0};
      int64_t rr = a;
      for (int d = 0; d < dim; d++) {
        li[d] = (int)(rr % n);
        rr /= n;
      }
      const int64_t gi = e * nn + a;
      if (xyz) {
        for (int l = 0; l < dim; l++) {
          if (!xyz[l]) continue;
          double acc = 0.0;
          for (int m = 0; m < nv; m++) {
            double Ni = 1.0;
            for (int d = 0; d < dim; d++) Ni *= (1.0 + (voff[m][d] ? 1.0 : -1.0) * xi[li[d]]);
            acc += Ni * (v[m][l] * vscale);
          }
          xyz[l][gi] = acc;
        }
      }
      if (mask) {
        double mk = 1.0;
        for (int d = 0; d < dim; d++) {
          if (periodic && periodic[d]) continue;
          if ((ei[d] == 0 && li[d] == 0) || (ei[d] == ne[d] - 1 && li[d] == n - 1)) mk = 0.0;
        }
        mask[gi] = mk;
      }
    }
  }
  return GF_OK;
}

// Emits the CSR of classes given a class key per node: classes ordered by
// their smallest member, members ascending.
static int64_t csr_from_keys(const std::vector<int64_t> &key, int64_t nkeys, int32_t *node_class,
                             int32_t *class_ptr, int32_t *members) {
  const int64_t N = (int64_t)key.size();
  std::vector<int32_t> cls_of_key(nkeys, -1);
  std::vector<int32_t> count;
  count.reserve(N);
  int32_t ncls = 0;
  std::vector<int32_t> cls(N);
  for (int64_t i = 0; i < N; i++) {
    int64_t k = key[i];
    if (cls_of_key[k] < 0) {
      cls_of_key[k] = ncls++;
      count.push_back(0);
    }
    cls[i] = cls_of_key[k];
    count[cls[i]]++;
  }
  std::vector<int32_t> pos(ncls + 1, 0);
  for (int32_t c = 0; c < ncls; c++) pos[c + 1] = pos[c] + count[c];
  if (class_ptr) std::memcpy(class_ptr, pos.data(), sizeof(int32_t) * (ncls + 1));
  std::vector<int32_t> fill(pos.begin(), pos.end() - 1);
  for (int64_t i = 0; i < N; i++) {
    if (members) members[fill[cls[i]]] = (int32_t)i;
    fill[cls[i]]++;
    if (node_class) node_class[i] = cls[i];
  }
  return ncls;
}

extern "C" int64_t gf_box_classes(int dim, const int *ne, int p, const int *periodic,
                                  int32_t *node_class, int32_t *class_ptr, int32_t *members) {
  if ((dim != 2 && dim != 3) || !ne || p < 1) return GF_ERR_ARG;
  const int n = p + 1;
  int64_t M[3] = {1, 1, 1}, nelem = 1, nn = 1;
  for (int d = 0; d < dim; d++) {
    M[d] = (int64_t)ne[d] * p + ((periodic && periodic[d]) ? 0 : 1);
    nelem *= ne[d];
    nn *= n;
  }
  if (nelem * nn > INT32_MAX) return GF_ERR_UNSUPPORTED;
  std::vector<int64_t> key(nelem * nn);
  for (int64_t e = 0; e < nelem; e++) {
    int ei[3] = {0, 0, 0};
    int64_t r = e;
    for (int d = 0; d < dim; d++) {
      ei[d] = (int)(r % ne[d]);
      r /= ne[d];
    }
    for (int64_t a = 0; a < nn; a++) {
      int64_t rr = a, k = 0, stride = 1;
      for (int d = 0; d < dim; d++) {
        int64_t li = rr % n;
        rr /= n;
        int64_t gidx = (int64_t)ei[d] * p + li;
        if (periodic && periodic[d] && gidx == (int64_t)ne[d] * p) gidx = 0;
        k += gidx * stride;
        stride *= M[d];
      }
      key[e * nn + a] = k;
    }
  }
  return csr_from_keys(key, M[0] * M[1] * M[2], node_class, class_ptr, members);
}

extern "C" int64_t gf_classes_from_coords(int dim, int64_t n, const double *const *xyz,
                                          double tol, int32_t *node_class, int32_t *class_ptr,
                                          int32_t *members) {
  if ((dim < 1 || dim > 3) || n < 0 || !xyz || !(tol > 0)) return GF_ERR_ARG;
  // cells of width 4*tol; two tolerance boxes intersect iff every
  // coordinate differs by at most 2*tol, so matches lie in adjacent cells.
  const double cell = 4.0 * tol;
  struct Item {
    int64_t c[3];
    int64_t id;
  };
  std::vector<Item> items(n);
  for (int64_t i = 0; i < n; i++) {
    items[i].id = i;
    for (int d = 0; d < 3; d++) items[i].c[d] = d < dim ? (int64_t)std::floor(xyz[d][i] / cell) : 0;
  }
  auto less = [](const Item &a, const Item &b) {
    if (a.c[0] != b.c[0]) return a.c[0] < b.c[0];
    if (a.c[1] != b.c[1]) return a.c[1] < b.c[1];
    if (a.c[2] != b.c[2]) return a.c[2] < b.c[2];
    return a.id < b.id;
  };
  std::sort(items.begin(), items.end(), less);
  std::vector<int64_t> key(n, -1);
  std::vector<int64_t> found;
  int64_t nk = 0;
  for (int64_t id = 0; id < n; id++) {
    if (key[id] >= 0) continue;
    int64_t c0[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) c0[d] = (int64_t)std::floor(xyz[d][id] / cell);
    found.clear();
    for (int dz = (dim > 2 ? -1 : 0); dz <= (dim > 2 ? 1 : 0); dz++)
      for (int dy = (dim > 1 ? -1 : 0); dy <= (dim > 1 ? 1 : 0); dy++)
        for (int dx = -1; dx <= 1; dx++) {
          Item probe{{c0[0] + dx, c0[1] + dy, c0[2] + dz}, -1};
          auto it = std::lower_bound(items.begin(), items.end(), probe, less);
          for (; it != items.end() && it->c[0] == probe.c[0] && it->c[1] == probe.c[1] &&
                 it->c[2] == probe.c[2];
               ++it) {
            bool hit = true;
            for (int d = 0; d < dim; d++) {
              double a = xyz[d][id], b = xyz[d][it->id];
              if (a + tol < b - tol || b + tol < a - tol) hit = false;
            }
            if (hit) found.push_back(it->id);
          }
        }
    for (int64_t m : found) key[m] = nk;
    nk++;
  }
  if (n > INT32_MAX) return GF_ERR_UNSUPPORTED;
  return csr_from_keys(key, nk, node_class, class_ptr, members);
}

// ---------------------------------------------------------------------
// problem
// ---------------------------------------------------------------------
template <typename T>
static T *upload(const std::vector<T> &h) {
  T *d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(T)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  return d;
}

static std::vector<float> to_f32(const std::vector<double> &v) {
  std::vector<float> f(v.size());
  for (size_t i = 0; i < v.size(); i++) f[i] = (float)v[i];
  return f;
}

extern "C" int gf_problem_destroy(gf_problem_t prob) {
  if (!prob) return GF_ERR_ARG;
  cudaSetDevice(prob->ctx->device);
  cudaStreamSynchronize(prob->ctx->stream);
  if (prob->mg && prob->mg_free) prob->mg_free(prob->mg);
  void *ptrs[] = {prob->egeom_d, prob->egeom_f, prob->ngeom_d, prob->ngeom_f, prob->mask_d,
                  prob->mask_f, prob->imass_d, prob->imass_f, prob->mass_d, prob->imult_d,
                  prob->imult_f, prob->class_ptr, prob->members, prob->node_class, prob->sh_ptr,
                  prob->sh_members, prob->scal_d, prob->partials, prob->counter,
                  prob->massL, prob->maskL8, prob->multL8, prob->dgeom_d, prob->dgeom_f,
                  prob->gmet_d, prob->gmet_f, prob->xyz_d, prob->xyz_f};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (prob->scal_h) cudaFreeHost(prob->scal_h);
  for (auto &b : prob->work)
    if (b.ptr) cudaFree(b.ptr);
  gf_context *ctx = prob->ctx;
  delete prob;
  if (--ctx->nprob == 0 && ctx->destroy_pending) {
    ctx->destroy_pending = false;
    gf_ctx_destroy(ctx);
  }
  return GF_OK;
}

extern "C" int gf_problem_create(gf_ctx_t ctx, const gf_problem_desc *d, gf_problem_t *out) {
  if (!ctx || !d || !out) return GF_ERR_ARG;
  *out = nullptr;
  GF_REQUIRE(ctx, d->dim == 2 || d->dim == 3, "dim must be 2 or 3 (got %d)", d->dim);
  GF_REQUIRE(ctx, d->n >= 2 && d->n <= GF_MAXN, "n must be in [2,%d] (got %d)", GF_MAXN, d->n);
  GF_REQUIRE(ctx, d->ne >= 1, "ne must be positive");
  GF_REQUIRE(ctx, d->D && d->W, "D and W are required");
  GF_REQUIRE(ctx, d->geom >= GF_GEOM_AFFINE && d->geom <= GF_GEOM_EMBEDDED, "unknown geometry kind");
  GF_REQUIRE(ctx, d->geom != GF_GEOM_AFFINE || d->elem_geom, "elem_geom required for AFFINE");
  GF_REQUIRE(ctx, d->geom == GF_GEOM_AFFINE || d->node_geom, "node_geom required");
  GF_REQUIRE(ctx, d->geom != GF_GEOM_EMBEDDED || d->dim == 2, "EMBEDDED grids are 2-d surfaces");
  GF_REQUIRE(ctx, d->class_ptr && d->members && d->nclass >= 1, "gather-scatter CSR required");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  const int dim = d->dim, n = d->n;
  int64_t nn = 1;
  for (int k = 0; k < dim; k++) nn *= n;
  const int64_t N = d->ne * nn;
  GF_REQUIRE(ctx, N <= INT32_MAX, "N_local %lld exceeds int32 indexing", (long long)N);
  GF_REQUIRE(ctx, d->class_ptr[0] == 0 && d->class_ptr[d->nclass] == N,
             "class_ptr must span all %lld local nodes", (long long)N);
  // validate the CSR: every node exactly once, ascending inside a class
  {
    std::vector<char> seen(N, 0);
    for (int64_t c = 0; c < d->nclass; c++) {
      GF_REQUIRE(ctx, d->class_ptr[c + 1] > d->class_ptr[c], "empty class %lld", (long long)c);
      for (int32_t k = d->class_ptr[c]; k < d->class_ptr[c + 1]; k++) {
        int32_t m = d->members[k];
        GF_REQUIRE(ctx, m >= 0 && m < N && !seen[m], "bad or repeated member %d", m);
        GF_REQUIRE(ctx, k == d->class_ptr[c] || d->members[k - 1] < m,
                   "members of class %lld not ascending", (long long)c);
        seen[m] = 1;
      }
    }
  }
  gf_problem *p = new gf_problem();
  p->ctx = ctx;
  ctx->nprob++;
  p->dim = dim;
  p->ne = d->ne;
  p->n = n;
  p->nlocal = N;
  p->nclass = d->nclass;
  p->geom = d->geom;
  std::memcpy(p->D, d->D, sizeof(double) * n * n);
  std::memcpy(p->W, d->W, sizeof(double) * n);
  gfk::gf_k1_matrix(n, p->D, p->W, p->K1);

  // geometry
  std::vector<double> jac(N), X0(N);
  if (d->geom == GF_GEOM_AFFINE) {
    std::vector<double> eg(d->elem_geom, d->elem_geom + d->ne * (dim + 1));
    p->egeom_d = upload(eg);
    p->egeom_f = upload(to_f32(eg));
    for (int64_t e = 0; e < d->ne; e++)
      for (int64_t a = 0; a < nn; a++) jac[e * nn + a] = eg[e * (dim + 1) + dim];
  } else if (d->geom == GF_GEOM_REGULAR) {
    std::vector<double> ng(d->node_geom, d->node_geom + (dim + 1) * N);
    p->ngeom_d = upload(ng);
    p->ngeom_f = upload(to_f32(ng));
    for (int64_t i = 0; i < N; i++) jac[i] = ng[dim * N + i];
  } else {
    // deformed / embedded: full dXi/dX, Jac, and the metric
    // G_ij = sum_k X_ik X_jk W Jac (GHelmholtz::def_init, ghelmholtz.ipp:416-519,
    // in its 2-d branch's order: each (i,j) accumulated once)
    const int nxy = d->geom == GF_GEOM_EMBEDDED ? 3 : dim;
    p->nxy = nxy;
    const double *X = d->node_geom;
    for (int64_t i = 0; i < N; i++) jac[i] = X[(int64_t)dim * nxy * N + i];
    std::vector<double> xg(X, X + (int64_t)dim * nxy * N);
    p->dgeom_d = upload(xg);
    p->dgeom_f = upload(to_f32(xg));
    std::vector<double> ng((dim + 1) * N, 0.0);  // zero diagonal planes, then Jac
    for (int64_t i = 0; i < N; i++) ng[dim * N + i] = jac[i];
    p->ngeom_d = upload(ng);
    p->ngeom_f = upload(to_f32(ng));
    const int npack = dim == 2 ? 3 : 6;
    std::vector<double> gm((size_t)npack * N, 0.0);
    const int pk3[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}}, pk2[3][3] = {{0, 1, 0}, {1, 2, 0}};
    for (int64_t e = 0; e < d->ne; e++)
      for (int64_t a = 0; a < nn; a++) {
        const int64_t node = e * nn + a;
        const int l = (int)(a % n), m = (int)((a / n) % n), pz = (int)(a / ((int64_t)n * n));
        for (int j = 0; j < dim; j++)
          for (int i = j; i < dim; i++) {
            double s = 0.0;
            for (int k = 0; k < nxy; k++) {
              double t = X[((int64_t)i * nxy + k) * N + node] * X[((int64_t)j * nxy + k) * N + node] *
                         d->W[l] * d->W[m];
              if (dim > 2) t = t * d->W[pz];
              s += t * jac[node];
            }
            gm[(size_t)(dim == 2 ? pk2[i][j] : pk3[i][j]) * N + node] = s;
          }
      }
    p->gmet_d = upload(gm);
    p->gmet_f = upload(to_f32(gm));
  }
  if (d->node_xyz) {
    std::vector<double> xyz(d->node_xyz, d->node_xyz + 3 * N);
    p->xyz_d = upload(xyz);
    p->xyz_f = upload(to_f32(xyz));
  }
  // local mass W (x) W (x) W * Jac (gmass.ipp:134-220)
  std::vector<double> mass(N);
  for (int64_t e = 0; e < d->ne; e++)
    for (int64_t a = 0; a < nn; a++) {
      int i = (int)(a % n), j = (int)((a / n) % n), k = (int)(a / ((int64_t)n * n));
      double w = dim == 2 ? d->W[j] * d->W[i] : d->W[k] * d->W[j] * d->W[i];
      mass[e * nn + a] = w * jac[e * nn + a];
    }
  p->volume = 0.0;
  for (int64_t i = 0; i < N; i++) p->volume += mass[i];
  // inverse mass 1/Smooth(M) (gmass.ipp:65-92) and 1/multiplicity
  std::vector<double> imass(N), imult(N);
  int64_t nshared = 0, nshm = 0;
  for (int64_t c = 0; c < d->nclass; c++) {
    int32_t b = d->class_ptr[c], e = d->class_ptr[c + 1];
    double s = 0.0;
    for (int32_t k = b; k < e; k++) s = s + mass[d->members[k]];
    s = s / (double)(size_t)(e - b);
    for (int32_t k = b; k < e; k++) {
      imass[d->members[k]] = 1.0 / s;
      imult[d->members[k]] = 1.0 / (double)(e - b);
    }
    if (e - b > 1) {
      nshared++;
      nshm += e - b;
    }
  }
  std::vector<int32_t> shp(nshared + 1), shm(nshm), ncls(N);
  {
    int64_t c2 = 0, pos = 0;
    for (int64_t c = 0; c < d->nclass; c++) {
      int32_t b = d->class_ptr[c], e = d->class_ptr[c + 1];
      for (int32_t k = b; k < e; k++) ncls[d->members[k]] = (int32_t)c;
      if (e - b < 2) continue;
      shp[c2++] = (int32_t)pos;
      for (int32_t k = b; k < e; k++) shm[pos++] = d->members[k];
    }
    shp[nshared] = (int32_t)pos;
  }
  p->nshared = nshared;
  // Unique-node indexing.  For a regular box the unique nodes are the
  // lattice points; the CSR must then be exactly the lattice classes.
  std::vector<int64_t> lofc(d->nclass);  // unique-node index of each class
  for (int64_t c = 0; c < d->nclass; c++) lofc[c] = c;
  if (d->box_ne[0] > 0) {
    gfk::BoxLattice L{};
    L.dim = dim;
    L.p = n - 1;
    int64_t nel = 1;
    for (int k = 0; k < 3; k++) {
      L.ne[k] = k < dim ? d->box_ne[k] : 1;
      L.per[k] = k < dim ? (d->box_periodic[k] != 0) : 0;
      L.M[k] = k < dim ? (int64_t)L.ne[k] * L.p + (L.per[k] ? 0 : 1) : 1;
      if (k < dim) nel *= L.ne[k];
    }
    if (nel != d->ne || L.size() != d->nclass) {
      gf_problem_destroy(p);
      return gf_fail(ctx, GF_ERR_ARG, "box description does not match the element or class count");
    }
    // every class must be one lattice point
    for (int64_t c = 0; c < d->nclass; c++) {
      int64_t key = -1;
      for (int32_t k = d->class_ptr[c]; k < d->class_ptr[c + 1]; k++) {
        const int64_t i = d->members[k], e = i / nn;
        const int a = (int)(i % nn);
        int ec[3];
        L.elem_coords(e, ec);
        int64_t g = L.g1(0, ec[0], a % n) + L.M[0] * L.g1(1, ec[1], (a / n) % n);
        if (dim > 2) g += L.M[0] * L.M[1] * L.g1(2, ec[2], a / (n * n));
        if (key >= 0 && g != key) {
          gf_problem_destroy(p);
          return gf_fail(ctx, GF_ERR_ARG, "gather-scatter classes are not the box lattice classes");
        }
        key = g;
      }
      lofc[c] = key;
    }
    p->box = L;
    p->has_box = true;
  }
  {
    std::vector<double> massL(d->nclass, 0.0);
    std::vector<uint8_t> maskL(d->nclass, 1), multL(d->nclass, 1);
    for (int64_t c = 0; c < d->nclass; c++) {
      double s = 0.0;
      for (int32_t k = d->class_ptr[c]; k < d->class_ptr[c + 1]; k++) s += mass[d->members[k]];
      massL[lofc[c]] = s;
      multL[lofc[c]] = (uint8_t)std::min<int32_t>(255, d->class_ptr[c + 1] - d->class_ptr[c]);
      if (d->mask) maskL[lofc[c]] = d->mask[d->members[d->class_ptr[c]]] != 0.0;
    }
    p->massL = upload(massL);
    p->multL8 = upload(multL);
    if (d->mask) p->maskL8 = upload(maskL);
  }
  p->mass_d = upload(mass);
  p->imass_d = upload(imass);
  p->imass_f = upload(to_f32(imass));
  p->imult_d = upload(imult);
  p->imult_f = upload(to_f32(imult));
  if (d->mask) {
    std::vector<double> mk(d->mask, d->mask + N);
    p->mask_d = upload(mk);
    p->mask_f = upload(to_f32(mk));
  }
  p->class_ptr = upload(std::vector<int32_t>(d->class_ptr, d->class_ptr + d->nclass + 1));
  p->members = upload(std::vector<int32_t>(d->members, d->members + N));
  p->node_class = upload(ncls);
  p->sh_ptr = upload(shp);
  if (nshm) p->sh_members = upload(shm);
  p->npartials = 2048;
  cudaMalloc(&p->partials, sizeof(double) * 4 * p->npartials);
  cudaMalloc(&p->counter, sizeof(unsigned int) * 8);
  cudaMemsetAsync(p->counter, 0, sizeof(unsigned int) * 8, ctx->stream);
  cudaMalloc(&p->scal_d, sizeof(double) * 64);
  cudaMemsetAsync(p->scal_d, 0, sizeof(double) * 64, ctx->stream);
  cudaMallocHost(&p->scal_h, sizeof(double) * 64);
  // uploads went through the legacy stream; finish them before any work
  // on the context's (non-blocking) stream can read the arrays
  cudaDeviceSynchronize();
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess || !p->mass_d || !p->imass_d || !p->class_ptr || !p->members ||
      !p->partials || !p->scal_d) {
    gf_problem_destroy(p);
    return gf_fail(ctx, GF_ERR_NOMEM, "device allocation failed in gf_problem_create (%s)",
                   cudaGetErrorString(err));
  }
  *out = p;
  return GF_OK;
}

extern "C" int gf_problem_sizes(gf_problem_t prob, int64_t *nlocal, int64_t *nclass) {
  if (!prob) return GF_ERR_ARG;
  if (nlocal) *nlocal = prob->nlocal;
  if (nclass) *nclass = prob->nclass;
  return GF_OK;
}

extern "C" int gf_problem_stats(gf_problem_t prob, int64_t *kernel_launches) {
  if (!prob) return GF_ERR_ARG;
  if (kernel_launches) *kernel_launches = (int64_t)prob->launches;
  return GF_OK;
}

// The inverse mass 1/Smooth(M) of a problem that is one rank's part of a
// partitioned grid: its own classes miss the copies on other ranks, so the
// caller supplies the assembled values (host, nlocal).
extern "C" int gf_problem_set_imass(gf_problem_t prob, const double *imass) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, imass, "imass is required");
  const int64_t n = prob->nlocal;
  std::vector<float> f(n);
  for (int64_t i = 0; i < n; i++) f[i] = (float)imass[i];
  GF_CUDA(ctx, cudaMemcpy(prob->imass_d, imass, sizeof(double) * n, cudaMemcpyHostToDevice));
  GF_CUDA(ctx, cudaMemcpy(prob->imass_f, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  return GF_OK;
}

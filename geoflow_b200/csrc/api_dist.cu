// api_dist.cu -- device building blocks of the element-partitioned
// (multi-GPU) gather-scatter and RK stepping (geoflow_b200/dist.py).
//
// A box partitioned by contiguous element ranges (GGridBox's
// find_rank_subdomain, grid/ggrid_box.ipp:855-980) leaves the copies of an
// interface lattice point on several ranks.  GGFX::doOp (comm/ggfx.hpp:
// 346-443) folds a point's copies in ascending global local id, so a rank
// that holds the copies' values (its own and those received from its
// peers) folds each shared point exactly as the single-GPU gather-scatter
// does: gf_dss_fold_copies, with the plan's index tables resident on the
// device.  gf_gather packs values by index (the copies a rank sends, its
// own copies before the local fold).  The three elementwise stage
// operations are the ones the single-GPU stepper fuses with its Smooth
// passes, so a partitioned step (update, exchange-and-fold) gives the same
// bits as gf_rk_advance.
#include "gf_common.cuh"
#include "k_dss.cuh"
#include "k_vec.cuh"

using namespace gfk;

namespace {

template <typename T>
__global__ void k_gather(int64_t n, const int32_t *__restrict__ idx, const T *__restrict__ src,
                         T *__restrict__ dst) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = src[idx[k]];
}

// u[out_local[k]] = fold over the copies of point out_point[k]:
// pool[table[point * maxc + j]] for j < maxc while table >= 0, in order.
template <typename T, int OP>
__global__ void k_fold_copies(int64_t nout, int maxc, const int32_t *__restrict__ table,
                              const T *__restrict__ pool, const int32_t *__restrict__ out_local,
                              const int32_t *__restrict__ out_point, T *__restrict__ u) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nout;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t *row = table + (int64_t)out_point[k] * maxc;
    T acc;
    int cnt = 0;
    if (OP == GF_DSS_SUM || OP == GF_DSS_SMOOTH) acc = T(0);
    else if (OP == GF_DSS_MAX) acc = Lim<T>::lowest();
    else acc = Lim<T>::highest();
    for (int j = 0; j < maxc; j++) {
      const int32_t s = row[j];
      if (s < 0) continue;
      const T v = pool[s];
      cnt++;
      if (OP == GF_DSS_SUM || OP == GF_DSS_SMOOTH) acc = __fadd_rn_t(acc, v);
      else if (OP == GF_DSS_MAX) acc = (acc < v) ? v : acc;
      else acc = (v < acc) ? v : acc;
    }
    if (OP == GF_DSS_SMOOTH) acc = acc / (T)cnt;
    u[out_local[k]] = acc;
  }
}

template <typename T>
__global__ void k_rk_update(int64_t n, T *__restrict__ x, T dt, const T *__restrict__ uin, T a,
                            const T *__restrict__ y, T b, T a2, const T *__restrict__ y2, T b2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = rk_euler_point(x[i], dt, uin[i], a, y, b, a2, y2, b2, i);
}

template <typename T>
__global__ void k_rk_accum(int64_t n, T *__restrict__ uout, const T *__restrict__ K, T ch) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    uout[i] = rk_accum_point(uout[i], K[i], ch);
}

inline unsigned blocks(gf_problem *p, int64_t n) {
  return grid_for(n, 256, p->ctx->sm_count * 8);
}

template <typename T>
int fold_copies(gf_problem *p, int op, int64_t nout, int maxc, const int32_t *table,
                const T *pool, const int32_t *out_local, const int32_t *out_point, T *u) {
  cudaStream_t st = p->ctx->stream;
  const unsigned g = blocks(p, nout);
  p->launches++;
  switch (op) {
    case GF_DSS_SUM:
      k_fold_copies<T, GF_DSS_SUM><<<g, 256, 0, st>>>(nout, maxc, table, pool, out_local, out_point, u);
      break;
    case GF_DSS_SMOOTH:
      k_fold_copies<T, GF_DSS_SMOOTH><<<g, 256, 0, st>>>(nout, maxc, table, pool, out_local, out_point, u);
      break;
    case GF_DSS_MAX:
      k_fold_copies<T, GF_DSS_MAX><<<g, 256, 0, st>>>(nout, maxc, table, pool, out_local, out_point, u);
      break;
    default:
      k_fold_copies<T, GF_DSS_MIN><<<g, 256, 0, st>>>(nout, maxc, table, pool, out_local, out_point, u);
  }
  return GF_OK;
}

}  // namespace

extern "C" int gf_gather(gf_problem_t prob, int dtype, int64_t n, const int32_t *idx,
                         const void *src, void *dst) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, n >= 0 && (n == 0 || (idx && src && dst)), "gather needs idx, src, dst");
  if (n == 0) return GF_OK;
  prob->launches++;
  if (dtype == GF_F64)
    k_gather<double><<<blocks(prob, n), 256, 0, ctx->stream>>>(n, idx, (const double *)src,
                                                               (double *)dst);
  else if (dtype == GF_F32)
    k_gather<float><<<blocks(prob, n), 256, 0, ctx->stream>>>(n, idx, (const float *)src,
                                                              (float *)dst);
  else
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_dss_fold_copies(gf_problem_t prob, int dtype, int op, int maxc,
                                  const int32_t *table, const void *pool, int64_t nout,
                                  const int32_t *out_local, const int32_t *out_point, void *u) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, op >= GF_DSS_SUM && op <= GF_DSS_MIN, "unknown op %d", op);
  GF_REQUIRE(ctx, maxc >= 1 && maxc <= 8, "1..8 copies per point");
  GF_REQUIRE(ctx, nout >= 0 && (nout == 0 || (table && pool && out_local && out_point && u)),
             "fold needs its tables, the pool and u");
  if (nout == 0) return GF_OK;
  int rc;
  if (dtype == GF_F64)
    rc = fold_copies<double>(prob, op, nout, maxc, table, (const double *)pool, out_local,
                             out_point, (double *)u);
  else if (dtype == GF_F32)
    rc = fold_copies<float>(prob, op, nout, maxc, table, (const float *)pool, out_local,
                            out_point, (float *)u);
  else
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  if (rc) return rc;
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_rk_update(gf_problem_t prob, int dtype, void *x, double dt, const void *uin,
                            double a, const void *y, double b, double a2, const void *y2,
                            double b2) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, x && uin, "x and uin are required");
  const int64_t n = prob->nlocal;
  prob->launches++;
  if (dtype == GF_F64)
    k_rk_update<double><<<blocks(prob, n), 256, 0, ctx->stream>>>(
        n, (double *)x, dt, (const double *)uin, a, (const double *)y, b, a2,
        (const double *)y2, b2);
  else if (dtype == GF_F32)
    k_rk_update<float><<<blocks(prob, n), 256, 0, ctx->stream>>>(
        n, (float *)x, (float)dt, (const float *)uin, (float)a, (const float *)y, (float)b,
        (float)a2, (const float *)y2, (float)b2);
  else
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

extern "C" int gf_rk_accum(gf_problem_t prob, int dtype, void *uout, const void *K, double ch) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, uout && K, "uout and K are required");
  const int64_t n = prob->nlocal;
  prob->launches++;
  if (dtype == GF_F64)
    k_rk_accum<double><<<blocks(prob, n), 256, 0, ctx->stream>>>(n, (double *)uout,
                                                                 (const double *)K, ch);
  else if (dtype == GF_F32)
    k_rk_accum<float><<<blocks(prob, n), 256, 0, ctx->stream>>>(n, (float *)uout,
                                                                (const float *)K, (float)ch);
  else
    return gf_fail(ctx, GF_ERR_ARG, "unknown dtype %d", dtype);
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

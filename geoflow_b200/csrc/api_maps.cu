// api_maps.cu -- gather-scatter classes built on the device.
//
// The same classes, numbering and CSR as the host builders gf_box_classes
// and gf_classes_from_coords (api_setup.cu), bit for bit, written into
// device arrays:
//   node_class[i]  class of node i; classes are numbered in the order of
//                  their smallest node id (first appearance in node order)
//   class_ptr[c]   start of class c in members (class_ptr[ncls] = n)
//   members        node ids grouped by class, ascending within a class
// GGFX::init (comm/ggfx.hpp:169-342) finds the classes by matching node
// coordinates within a tolerance through an R-tree on the host; here
//   box:    each node's class key is its lattice point (closed form);
//   coords: nodes are binned in cells of width 4 tol (matches lie in
//           adjacent cells), sorted by (cell, id), and each node's key is
//           the smallest id among the nodes whose tolerance boxes meet its
//           own -- the class representative when matches are transitive,
//           as for any grid whose tolerance is below half the node spacing.
// Then: first[key] = smallest node of each key, ranks of the first nodes
// by a scan, node_class by lookup, members by a stable radix sort of the
// node ids on their class, class_ptr from the class boundaries.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "gf_common.cuh"

namespace {

#define GS(i, n)                                                                 \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);     \
       i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_box_keys(int64_t n, int dim, int ne0, int ne1, int ne2, int p, int per0,
                           int per1, int per2, int64_t M0, int64_t M1, int32_t *key) {
  const int nb = p + 1;
  const int nn = dim == 3 ? nb * nb * nb : nb * nb;
  const int ne[3] = {ne0, ne1, ne2}, per[3] = {per0, per1, per2};
  GS(i, n) {
    const int64_t e = i / nn;
    int a = (int)(i - e * nn);
    int64_t r = e, k = 0, stride = 1;
    const int64_t M[3] = {M0, M1, 1};
    for (int d = 0; d < dim; d++) {
      const int ei = (int)(r % ne[d]);
      r /= ne[d];
      const int li = a % nb;
      a /= nb;
      int64_t g = (int64_t)ei * p + li;
      if (per[d] && g == (int64_t)ne[d] * p) g = 0;
      k += g * stride;
      stride *= M[d];
    }
    key[i] = (int32_t)k;
  }
}

__global__ void k_fill(int64_t n, int32_t v, int32_t *a) {
  GS(i, n) a[i] = v;
}

__global__ void k_iota(int64_t n, int32_t *a) {
  GS(i, n) a[i] = (int32_t)i;
}

// first[key[i]] = min i
__global__ void k_first(int64_t n, const int32_t *key, int32_t *first) {
  GS(i, n) atomicMin(&first[key[i]], (int32_t)i);
}

__global__ void k_is_first(int64_t n, const int32_t *key, const int32_t *first, int32_t *flag) {
  GS(i, n) flag[i] = first[key[i]] == (int32_t)i ? 1 : 0;
}

// node_class[i] = rank of the first node of i's key
__global__ void k_node_class(int64_t n, const int32_t *key, const int32_t *first,
                             const int32_t *rank, int32_t *node_class) {
  GS(i, n) node_class[i] = rank[first[key[i]]];
}

// class_ptr from the class-sorted node classes
__global__ void k_class_ptr(int64_t n, int64_t ncls, const int32_t *sorted_cls,
                            int32_t *class_ptr) {
  GS(i, n) {
    if (i == 0 || sorted_cls[i] != sorted_cls[i - 1]) class_ptr[sorted_cls[i]] = (int32_t)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) class_ptr[ncls] = (int32_t)n;
}

// cell coordinates (cells of width `cell`), packed 21 bits per direction
// after subtracting the smallest cell; out-of-range packing is reported
__global__ void k_cells(int64_t n, int dim, const double *x, const double *y, const double *z,
                        double cell, int64_t c0x, int64_t c0y, int64_t c0z, uint64_t *ckey,
                        int *overflow) {
  GS(i, n) {
    const double *X[3] = {x, y, z};
    const int64_t c0[3] = {c0x, c0y, c0z};
    uint64_t k = 0;
    for (int d = 0; d < 3; d++) {
      int64_t c = 0;
      if (d < dim) c = (int64_t)floor(X[d][i] / cell) - c0[d];
      if (c < 0 || c >= (1 << 21)) *overflow = 1;
      k |= (uint64_t)(c & ((1 << 21) - 1)) << (21 * d);
    }
    ckey[i] = k;
  }
}

// smallest cell coordinate per direction (atomicMin on int64 via
// unsigned offset)
__global__ void k_cell_min(int64_t n, int dim, const double *x, const double *y, const double *z,
                           double cell, unsigned long long *cmin) {
  GS(i, n) {
    const double *X[3] = {x, y, z};
    for (int d = 0; d < dim; d++) {
      const int64_t c = (int64_t)floor(X[d][i] / cell);
      atomicMin(&cmin[d], (unsigned long long)(c + ((int64_t)1 << 62)));
    }
  }
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t *a, int64_t n, uint64_t v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// key[i] = smallest id among the nodes whose tolerance boxes meet node i's
// (the host test: boxes miss iff a + tol < b - tol or b + tol < a - tol in
// some direction), found in the 3^dim neighbouring cells
__global__ void k_match(int64_t n, int dim, const double *x, const double *y, const double *z,
                        double tol, const uint64_t *skey, const int32_t *sid,
                        const uint64_t *ckey, int32_t *key) {
  GS(i, n) {
    const double *X[3] = {x, y, z};
    const uint64_t k = ckey[i];
    const int64_t c[3] = {(int64_t)(k & 0x1FFFFF), (int64_t)((k >> 21) & 0x1FFFFF),
                          (int64_t)((k >> 42) & 0x1FFFFF)};
    double a[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) a[d] = X[d][i];
    int32_t best = (int32_t)i;
    const int zr = dim > 2 ? 1 : 0, yr = dim > 1 ? 1 : 0;
    for (int dz = -zr; dz <= zr; dz++)
      for (int dy = -yr; dy <= yr; dy++) {
        const int64_t cy = c[1] + dy, cz = c[2] + dz;
        if (cy < 0 || cz < 0 || cy >= (1 << 21) || cz >= (1 << 21)) continue;
        const int64_t cxl = c[0] > 0 ? c[0] - 1 : 0;
        const int64_t cxh = c[0] + 1 < (1 << 21) ? c[0] + 1 : (1 << 21) - 1;
        const uint64_t lo = (uint64_t)cxl | ((uint64_t)cy << 21) | ((uint64_t)cz << 42);
        const uint64_t hi = (uint64_t)cxh | ((uint64_t)cy << 21) | ((uint64_t)cz << 42);
        for (int64_t j = lower_bound_u64(skey, n, lo); j < n && skey[j] <= hi; j++) {
          const int32_t m = sid[j];
          if (m >= best) continue;
          bool hit = true;
          for (int d = 0; d < dim; d++) {
            const double b = X[d][m];
            if (a[d] + tol < b - tol || b + tol < a[d] - tol) hit = false;
          }
          if (hit) best = m;
        }
      }
    key[i] = best;
  }
}

// scratch owned by one call
struct Scratch {
  std::vector<void *> p;
  template <typename T>
  T *get(size_t n) {
    void *q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    p.push_back(q);
    return (T *)q;
  }
  ~Scratch() {
    for (void *q : p) cudaFree(q);
  }
};

// keys (< nkeys) -> node_class, class_ptr, members; returns the class count
int64_t classes_from_keys(gf_context *ctx, int64_t n, int64_t nkeys, int32_t *key,
                          int32_t *node_class, int32_t *class_ptr, int32_t *members) {
  cudaStream_t st = ctx->stream;
  const unsigned grid = grid_for(n, 256, ctx->sm_count * 16);
  Scratch S;
  int32_t *first = S.get<int32_t>(nkeys), *flag = S.get<int32_t>(n + 1),
          *rank = S.get<int32_t>(n + 1), *ids = S.get<int32_t>(n), *scls = S.get<int32_t>(n);
  if (!first || !flag || !rank || !ids || !scls)
    return gf_fail(ctx, GF_ERR_NOMEM, "class construction allocation failed");
  k_fill<<<grid_for(nkeys, 256, ctx->sm_count * 16), 256, 0, st>>>(nkeys, INT32_MAX, first);
  k_first<<<grid, 256, 0, st>>>(n, key, first);
  k_is_first<<<grid, 256, 0, st>>>(n, key, first, flag);
  GF_CUDA(ctx, cudaMemsetAsync(flag + n, 0, sizeof(int32_t), st));
  size_t tb = 0;
  GF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, rank, (int)(n + 1), st));
  void *tmp = S.get<char>(tb);
  if (!tmp) return gf_fail(ctx, GF_ERR_NOMEM, "scan allocation failed");
  GF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp, tb, flag, rank, (int)(n + 1), st));
  int32_t ncls = 0;
  GF_CUDA(ctx, cudaMemcpyAsync(&ncls, rank + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  k_node_class<<<grid, 256, 0, st>>>(n, key, first, rank, node_class);
  // members: node ids stably sorted on their class (ascending within a class)
  k_iota<<<grid, 256, 0, st>>>(n, ids);
  int bits = 1;
  while (bits < 31 && ((int64_t)1 << bits) < n) bits++;
  size_t ts = 0;
  GF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, ts, node_class, scls, ids, members,
                                               (int)n, 0, bits, st));
  void *tmp2 = S.get<char>(ts);
  if (!tmp2) return gf_fail(ctx, GF_ERR_NOMEM, "sort allocation failed");
  GF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp2, ts, node_class, scls, ids, members, (int)n,
                                               0, bits, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  k_class_ptr<<<grid, 256, 0, st>>>(n, ncls, scls, class_ptr);
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  GF_CHECK_LAUNCH(ctx);
  return ncls;
}

}  // namespace

extern "C" int64_t gf_box_classes_device(gf_ctx_t ctx, int dim, const int *ne, int p,
                                         const int *periodic, int32_t *node_class,
                                         int32_t *class_ptr, int32_t *members) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, (dim == 2 || dim == 3) && ne && p >= 1, "bad box description");
  GF_REQUIRE(ctx, node_class && class_ptr && members, "output arrays are required");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  const int n1 = p + 1;
  int64_t M[3] = {1, 1, 1}, nelem = 1, nn = 1;
  for (int d = 0; d < dim; d++) {
    GF_REQUIRE(ctx, ne[d] >= 1, "element counts must be positive");
    M[d] = (int64_t)ne[d] * p + ((periodic && periodic[d]) ? 0 : 1);
    nelem *= ne[d];
    nn *= n1;
  }
  const int64_t n = nelem * nn;
  GF_REQUIRE(ctx, n <= INT32_MAX, "%lld nodes exceed int32 indexing", (long long)n);
  Scratch S;
  int32_t *key = S.get<int32_t>(n);
  if (!key) return gf_fail(ctx, GF_ERR_NOMEM, "key allocation failed");
  k_box_keys<<<grid_for(n, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
      n, dim, ne[0], ne[1], dim > 2 ? ne[2] : 1, p, periodic ? periodic[0] : 0,
      periodic ? periodic[1] : 0, (periodic && dim > 2) ? periodic[2] : 0, M[0], M[1], key);
  return classes_from_keys(ctx, n, M[0] * M[1] * M[2], key, node_class, class_ptr, members);
}

extern "C" int64_t gf_classes_from_coords_device(gf_ctx_t ctx, int dim, int64_t n,
                                                 const double *const *xyz, double tol,
                                                 int32_t *node_class, int32_t *class_ptr,
                                                 int32_t *members) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, dim >= 1 && dim <= 3 && n >= 1 && xyz && tol > 0, "bad arguments");
  GF_REQUIRE(ctx, node_class && class_ptr && members, "output arrays are required");
  GF_REQUIRE(ctx, n <= INT32_MAX, "%lld nodes exceed int32 indexing", (long long)n);
  for (int d = 0; d < dim; d++) GF_REQUIRE(ctx, xyz[d], "coordinate %d missing", d);
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const double *x = xyz[0], *y = dim > 1 ? xyz[1] : xyz[0], *z = dim > 2 ? xyz[2] : xyz[0];
  const double cell = 4.0 * tol;
  const unsigned grid = grid_for(n, 256, ctx->sm_count * 16);
  Scratch S;
  unsigned long long *cmin = S.get<unsigned long long>(3);
  int *ovf = S.get<int>(1);
  uint64_t *ckey = S.get<uint64_t>(n), *skey = S.get<uint64_t>(n);
  int32_t *ids = S.get<int32_t>(n), *sid = S.get<int32_t>(n), *key = S.get<int32_t>(n);
  if (!cmin || !ovf || !ckey || !skey || !ids || !sid || !key)
    return gf_fail(ctx, GF_ERR_NOMEM, "matching allocation failed");
  std::vector<unsigned long long> hmin(3, ~0ull);
  GF_CUDA(ctx, cudaMemcpyAsync(cmin, hmin.data(), 3 * sizeof(unsigned long long),
                               cudaMemcpyHostToDevice, st));
  GF_CUDA(ctx, cudaMemsetAsync(ovf, 0, sizeof(int), st));
  k_cell_min<<<grid, 256, 0, st>>>(n, dim, x, y, z, cell, cmin);
  GF_CUDA(ctx, cudaMemcpyAsync(hmin.data(), cmin, 3 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  int64_t c0[3] = {0, 0, 0};
  // one cell of margin below the smallest, so that neighbours stay >= 0
  for (int d = 0; d < dim; d++) c0[d] = (int64_t)(hmin[d] - (1ull << 62)) - 1;
  k_cells<<<grid, 256, 0, st>>>(n, dim, x, y, z, cell, c0[0], c0[1], c0[2], ckey, ovf);
  int hovf = 0;
  GF_CUDA(ctx, cudaMemcpyAsync(&hovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
  GF_CUDA(ctx, cudaStreamSynchronize(st));
  GF_REQUIRE(ctx, hovf == 0, "coordinate extent exceeds 2^21 - 2 cells of width 4 tol");
  k_iota<<<grid, 256, 0, st>>>(n, ids);
  size_t ts = 0;
  GF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, ts, ckey, skey, ids, sid, (int)n, 0,
                                               21 * dim, st));
  void *tmp = S.get<char>(ts);
  if (!tmp) return gf_fail(ctx, GF_ERR_NOMEM, "sort allocation failed");
  GF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, ts, ckey, skey, ids, sid, (int)n, 0,
                                               21 * dim, st));
  k_match<<<grid, 256, 0, st>>>(n, dim, x, y, z, tol, skey, sid, ckey, key);
  return classes_from_keys(ctx, n, n, key, node_class, class_ptr, members);
}

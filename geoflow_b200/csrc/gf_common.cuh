// gf_common.cuh -- shared definitions of libgfgpu: context and problem
// objects, error handling, the per-order basis parameter block and the
// compile-time dispatch over the GLL point count n.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/gfgpu.h"
#include "lattice.cuh"

#define GF_MAXN 12  // largest GLL point count compiled (p = 11)

struct gf_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nprob = 0;                // live problems created on this context
  bool destroy_pending = false; // destroyed while problems were alive
  int sm_count = 148;
  std::string last_error;
  std::string returned_error;  // storage for gf_ctx_last_error
};

// Device scratch owned by a problem, grown on demand and reused.
struct gf_buffer {
  void *ptr = nullptr;
  size_t bytes = 0;
};

struct gf_problem {
  gf_context *ctx = nullptr;
  int dim = 3;
  int64_t ne = 0;
  int n = 0;
  int64_t nlocal = 0;  // Ne * n^dim
  int64_t nclass = 0;  // unique nodes
  int geom = GF_GEOM_AFFINE;
  double volume = 0.0;  // sum of the local mass (integral of 1)
  double D[GF_MAXN * GF_MAXN];
  double W[GF_MAXN];
  double K1[GF_MAXN * GF_MAXN];  // D^T diag(W) D (affine-element apply)
  // device geometry (both precisions)
  double *egeom_d = nullptr;  // ne*(dim+1) (AFFINE)
  float *egeom_f = nullptr;
  double *ngeom_d = nullptr;  // (dim+1)*nlocal (REGULAR; DEFORMED/EMBEDDED: 0 planes + Jac)
  float *ngeom_f = nullptr;
  // DEFORMED / EMBEDDED: full dXi/dX (dim*nxy planes), packed metric G_ij
  // with W and Jac (dim(dim+1)/2 planes), node coordinates (optional)
  int nxy = 0;
  double *dgeom_d = nullptr, *gmet_d = nullptr, *xyz_d = nullptr;
  float *dgeom_f = nullptr, *gmet_f = nullptr, *xyz_f = nullptr;
  double *mask_d = nullptr;   // nlocal or null
  float *mask_f = nullptr;
  double *imass_d = nullptr;  // 1/Smooth(mass), nlocal
  float *imass_f = nullptr;
  double *mass_d = nullptr;   // local mass, nlocal
  double *imult_d = nullptr;  // 1/multiplicity, nlocal
  float *imult_f = nullptr;
  // gather-scatter map
  int32_t *class_ptr = nullptr;  // nclass+1
  int32_t *members = nullptr;    // nlocal
  int32_t *node_class = nullptr; // nlocal
  // regular box lattice (GGridBox): unique nodes indexed by lattice point
  bool has_box = false;
  gfk::BoxLattice box{};
  // unique-node (L) vectors, indexed by lattice point (box) or class (CSR)
  double *massL = nullptr;      // assembled mass (L2/L1 norms)
  uint8_t *multL8 = nullptr;    // multiplicity per unique node (EUC norm)
  uint8_t *maskL8 = nullptr;    // Dirichlet mask per unique node: 1 keep, 0 masked
  // classes with more than one member (shared nodes) and the singletons
  int64_t nshared = 0;
  int32_t *sh_ptr = nullptr;
  int32_t *sh_members = nullptr;
  // scratch
  std::vector<gf_buffer> work;
  double *scal_d = nullptr;      // device scalar block (CG/RK state)
  double *scal_h = nullptr;      // pinned host mirror
  double *partials = nullptr;    // block partial sums
  unsigned int *counter = nullptr;
  int npartials = 0;
  uint64_t launches = 0;  // kernels launched on this problem (instrumentation)
  // cached multigrid hierarchy of the CG preconditioner (api_cg.cu)
  void *mg = nullptr;
  void (*mg_free)(void *) = nullptr;
};

// ---- error helpers ----
int gf_fail(gf_context *ctx, int code, const char *fmt, ...);

#define GF_CUDA(ctx, call)                                                     \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess)                                                     \
      return gf_fail((ctx), GF_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,   \
                     #call, cudaGetErrorString(_e));                          \
  } while (0)

#define GF_CHECK_LAUNCH(ctx) GF_CUDA(ctx, cudaGetLastError())

#define GF_REQUIRE(ctx, cond, ...)                                             \
  do {                                                                         \
    if (!(cond)) return gf_fail((ctx), GF_ERR_ARG, __VA_ARGS__);               \
  } while (0)

// Velocity components of the advection terms: one per physical coordinate
// (3 on a 2-d surface embedded in 3-d space).
inline int gf_nvel(const gf_problem *p) { return p->nxy ? p->nxy : p->dim; }

// Returns a device buffer of at least `bytes` from slot `slot` of the
// problem's scratch list (allocated once, reused).
void *gf_work(gf_problem *prob, int slot, size_t bytes);

namespace gfk {
// K1 = D^T diag(W) D of a GLL basis (n points), exactly symmetric and
// centro-symmetric; column-major like D.
void gf_k1_matrix(int n, const double *D, const double *W, double *K1);
}  // namespace gfk

// ---- per-order constants passed by value to kernels ----
// D is stored column-major: D(l,j) = D[l + j*N].
template <typename T, int N>
struct Basis {
  T D[N * N];
  T W[N];
};

template <typename T, int N>
inline Basis<T, N> make_basis(const gf_problem *p) {
  Basis<T, N> b;
  for (int i = 0; i < N * N; i++) b.D[i] = (T)p->D[i];
  for (int i = 0; i < N; i++) b.W[i] = (T)p->W[i];
  return b;
}

// Geometry view handed to kernels.
template <typename T>
struct Geom {
  const T *egeom;  // per element: dXidX_0..dim-1, Jac (AFFINE), or null
  const T *ngeom;  // per node planes (REGULAR), or null
  int64_t nlocal;
};

template <typename T>
inline Geom<T> geom_of(const gf_problem *p);
template <>
inline Geom<double> geom_of<double>(const gf_problem *p) {
  return Geom<double>{p->egeom_d, p->ngeom_d, p->nlocal};
}
template <>
inline Geom<float> geom_of<float>(const gf_problem *p) {
  return Geom<float>{p->egeom_f, p->ngeom_f, p->nlocal};
}

template <typename T> inline const T *mask_of(const gf_problem *p);
template <> inline const double *mask_of<double>(const gf_problem *p) { return p->mask_d; }
template <> inline const float *mask_of<float>(const gf_problem *p) { return p->mask_f; }
template <typename T> inline const T *imass_of(const gf_problem *p);
template <> inline const double *imass_of<double>(const gf_problem *p) { return p->imass_d; }
template <> inline const float *imass_of<float>(const gf_problem *p) { return p->imass_f; }
template <typename T> inline const T *imult_of(const gf_problem *p);
template <> inline const double *imult_of<double>(const gf_problem *p) { return p->imult_d; }
template <> inline const float *imult_of<float>(const gf_problem *p) { return p->imult_f; }

// Dispatch a functor templated on N over the compiled range.
template <template <int> class F, typename... Args>
inline int dispatch_n(int n, Args &&...args) {
  switch (n) {
    case 2: return F<2>::run(args...);
    case 3: return F<3>::run(args...);
    case 4: return F<4>::run(args...);
    case 5: return F<5>::run(args...);
    case 6: return F<6>::run(args...);
    case 7: return F<7>::run(args...);
    case 8: return F<8>::run(args...);
    case 9: return F<9>::run(args...);
    case 10: return F<10>::run(args...);
    case 11: return F<11>::run(args...);
    case 12: return F<12>::run(args...);
    default: return GF_ERR_UNSUPPORTED;
  }
}

inline unsigned grid_for(int64_t n, int threads, int max_blocks) {
  int64_t b = (n + threads - 1) / threads;
  if (b > max_blocks) b = max_blocks;
  if (b < 1) b = 1;
  return (unsigned)b;
}

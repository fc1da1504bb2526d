// k_dss.cuh -- direct-stiffness gather-scatter (GGFX::doOp) kernels.
//
// One thread per equivalence class (a lattice point on box grids, a node
// of a singleton class or a shared class on CSR grids): it gathers the
// class members in ascending local id, folds them exactly as the
// reference's reduction functors do (comm/ggfx.hpp:36-76: std::accumulate
// from 0 for Sum and Smooth, std::max/std::min folds from lowest()/max()),
// and scatters the result to every member.  The fold order is fixed, so
// FP64 results are bit-identical to the reference's and independent of the
// launch shape.
#pragma once
#include <cfloat>

#include "gf_common.cuh"
#include "k_vec.cuh"

namespace gfk {

template <typename T> struct Lim;
template <> struct Lim<double> {
  static __device__ __forceinline__ double lowest() { return -DBL_MAX; }
  static __device__ __forceinline__ double highest() { return DBL_MAX; }
};
template <> struct Lim<float> {
  static __device__ __forceinline__ float lowest() { return -FLT_MAX; }
  static __device__ __forceinline__ float highest() { return FLT_MAX; }
};

// The box-lattice walk of a problem whose gather-scatter can take the box
// kernels below: a GGridBox problem (classes = lattice points) with no
// periodic direction of a single element (members then come in the
// (z, y, x) nesting in ascending local id).
inline bool dss_box_walk(const gf_problem *prob, BoxWalk &w) {
  if (!prob->has_box) return false;
  w = BoxWalk::make(prob->box);
  return w.sorted;
}

// The GGFX fold over the copies of one box-lattice point (ascending local id)
template <typename T, int OP>
__device__ __forceinline__ T box_fold(const T *__restrict__ u, const BoxCopies &k) {
  T acc;
  if (OP == GF_DSS_SUM || OP == GF_DSS_SMOOTH) {
    acc = T(0);
    k.each([&](int m) { acc = __fadd_rn_t(acc, u[m]); });
    if (OP == GF_DSS_SMOOTH) acc = acc / (T)k.count();
  } else if (OP == GF_DSS_MAX) {
    acc = Lim<T>::lowest();
    k.each([&](int m) {
      const T v = u[m];
      acc = (acc < v) ? v : acc;
    });
  } else {
    acc = Lim<T>::highest();
    k.each([&](int m) {
      const T v = u[m];
      acc = (v < acc) ? v : acc;
    });
  }
  return acc;
}

// Box-lattice form of k_dss_split (GGridBox problems, whose classes are the
// lattice points; no periodic direction with a single element): one thread
// per lattice point in lattice order, the members computed from the
// point's coordinates (BoxWalk) in ascending local id, so no index arrays
// are read and a point costs one memory round trip.  Same folds, same
// order: bit-identical to the CSR form.
template <typename T, int OP>
__global__ void __launch_bounds__(256) k_dss_box(T *__restrict__ u, BoxWalk w) {
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w.nL;
       c = (c < w.nL - stride) ? c + stride : w.nL) {
    const BoxCopies k = w.copies(c);
    const T acc = box_fold<T, OP>(u, k);
    k.each([&](int m) { u[m] = acc; });
  }
}

// The classes of a CSR problem split by size: a class with one member (an
// interior node, most of them on icosahedral and deformed grids) is folded
// by the thread of that node, in node order (coalesced, no index arrays;
// imult = 1 marks it), and a class with several members by one thread from
// the shared-class list (sh_ptr / sh_members, members in ascending local
// id).  Items: the n nodes, then the nsh shared classes.  Each class is
// folded exactly as the full CSR walk folds it.
struct SplitCls {
  int64_t n;              // element-local nodes
  const float *imult;     // 1/multiplicity per node
  const int32_t *shp;     // nsh + 1
  const int32_t *shm;
  int64_t nsh;
};

inline SplitCls split_of(const gf_problem *p) {
  return SplitCls{p->nlocal, p->imult_f, p->sh_ptr, p->sh_members, p->nshared};
}

// f(get, cnt): get(k) is the k-th member (ascending local id) of item it's
// class, cnt the member count; nothing for a node of a shared class.
template <class F>
__device__ __forceinline__ void split_item(const SplitCls &s, int64_t it, F f) {
  if (it < s.n) {
    if (s.imult[it] != 1.0f) return;
    f([&](int) { return it; }, 1);
  } else {
    const int64_t c = it - s.n;
    const int32_t b = s.shp[c], e = s.shp[c + 1];
    f([&](int k) { return (int64_t)s.shm[b + k]; }, e - b);
  }
}

template <typename T, int OP>
__global__ void __launch_bounds__(256) k_dss_split(T *__restrict__ u, SplitCls s) {
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < s.n + s.nsh;
       it += (int64_t)gridDim.x * blockDim.x)
    split_item(s, it, [&](auto get, int cnt) {
      T acc;
      if (OP == GF_DSS_SUM || OP == GF_DSS_SMOOTH) {
        acc = T(0);
        for (int k = 0; k < cnt; k++) acc = __fadd_rn_t(acc, u[get(k)]);
        if (OP == GF_DSS_SMOOTH) acc = acc / (T)cnt;
      } else if (OP == GF_DSS_MAX) {
        acc = Lim<T>::lowest();
        for (int k = 0; k < cnt; k++) {
          const T v = u[get(k)];
          acc = (acc < v) ? v : acc;
        }
      } else {
        acc = Lim<T>::highest();
        for (int k = 0; k < cnt; k++) {
          const T v = u[get(k)];
          acc = (v < acc) ? v : acc;
        }
      }
      for (int k = 0; k < cnt; k++) u[get(k)] = acc;
    });
}

// ---- gather-scatter fused with the RK stage updates (api_rk.cu) ----
// The stage arithmetic of GExRKStepper, with explicit round-to-nearest
// operations so that it rounds the same wherever it runs:
//   step_euler + saxpby (gexrk_stepper.ipp:809-819, 533-780):
//     v = dt x + 1 uin;  v = a v + b y (if y);  v = a2 v + b2 y2 (if y2)
//   step_b accumulation (252-341): uout += (K * ch)
// (y[i] and y2[i] are read before the arithmetic, so that a caller's loads
// of several points are all in flight together; measured on the FP64
// stage-update pass at 64^3 p = 5: 1.68 -> 1.57 ms)
template <typename T>
__device__ __forceinline__ T rk_euler_vals(T x, T dt, T uin, T a, bool has_y, T yv, T b, T a2,
                                           bool has_y2, T y2v, T b2) {
  T v = add_rn(mul_rn(dt, x), mul_rn(T(1), uin));
  if (has_y) v = add_rn(mul_rn(a, v), mul_rn(b, yv));
  if (has_y2) v = add_rn(mul_rn(a2, v), mul_rn(b2, y2v));
  return v;
}
template <typename T>
__device__ __forceinline__ T rk_euler_point(T x, T dt, T uin, T a, const T *y, T b, T a2,
                                            const T *y2, T b2, int64_t i) {
  return rk_euler_vals(x, dt, uin, a, y != nullptr, y ? y[i] : T(0), b, a2, y2 != nullptr,
                       y2 ? y2[i] : T(0), b2);
}
template <typename T>
__device__ __forceinline__ T rk_accum_point(T uout, T K, T ch) {
  return add_rn(uout, mul_rn(K, ch));
}
// step_b stage input (252-341): y = uin + ((0 + b0 K0) + b1 K1 + ...), the
// isum accumulation over the nk earlier slopes
template <typename T>
__device__ __forceinline__ T rk_stage_point(T uin, int nk, const T *__restrict__ K0,
                                            const T *__restrict__ K1, const T *__restrict__ K2,
                                            T b0, T b1, T b2, int64_t i) {
  T s = T(0);
  if (nk > 0) s = T(1) * s + b0 * K0[i];
  if (nk > 1) s = T(1) * s + b1 * K1[i];
  if (nk > 2) s = T(1) * s + b2 * K2[i];
  T v = uin;
  v += s;
  return v;
}

enum { FUSE_EULER = 0, FUSE_ACCUM_AFTER = 1, FUSE_ACCUM_BEFORE = 2 };

// One class per item (SplitCls), members in ascending local id, Smooth fold:
//   FUSE_EULER:        x_m <- rk_euler_point(x_m, ...) folded           (SSP substep)
//   FUSE_ACCUM_AFTER:  x_m <- fold(x);  acc_m <- rk_accum_point(acc_m, fold, ch)
//                      (Smooth K_m, then uout += c_m h K_m)
//   FUSE_ACCUM_BEFORE: x_m <- fold(rk_accum_point(x_m, K_m, ch))
//                      (uout += c h K, then Smooth uout)
template <typename T, int MODE>
__global__ void __launch_bounds__(256)
    k_dss_rk_split(T *__restrict__ x, SplitCls s, T dt, const T *__restrict__ uin, T a,
                   const T *__restrict__ y, T b, T a2, const T *__restrict__ y2, T b2,
                   T *__restrict__ acc_out, const T *__restrict__ K, T ch) {
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < s.n + s.nsh;
       it += (int64_t)gridDim.x * blockDim.x)
    split_item(s, it, [&](auto get, int cnt) {
      T acc = T(0);
      for (int k = 0; k < cnt; k++) {
        const int64_t m = get(k);
        T v = x[m];
        if (MODE == FUSE_EULER) v = rk_euler_point(v, dt, uin[m], a, y, b, a2, y2, b2, m);
        if (MODE == FUSE_ACCUM_BEFORE) v = rk_accum_point(v, K[m], ch);
        acc = __fadd_rn_t(acc, v);
      }
      acc = acc / (T)cnt;
      for (int k = 0; k < cnt; k++) {
        const int64_t m = get(k);
        x[m] = acc;
        if (MODE == FUSE_ACCUM_AFTER) acc_out[m] = rk_accum_point(acc_out[m], acc, ch);
      }
    });
}

// The state components of one fused stage update (pointers per component;
// y, y2, uin, K, acc may be null as in k_dss_rk_split).
template <typename T>
struct RKComps {
  T *x[3];
  const T *uin[3], *y[3], *y2[3], *K[3];
  T *acc[3];
};

// Box-lattice form of k_dss_rk_split (conditions of k_dss_box) on every
// state component in one pass: the copies of a lattice point are computed
// once, and every component's members are read before any is written (all
// loads of a point in one memory round trip).  Per component the same
// stage arithmetic, Smooth fold and order as k_dss_rk_split: bit-identical.
template <typename T, int MODE, int NC>
__global__ void __launch_bounds__(256, 5)
    k_dss_rk_box_n(RKComps<T> p, BoxWalk w, T dt, T a, T b, T a2, T b2, T ch) {
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w.nL;
       c = (c < w.nL - stride) ? c + stride : w.nL) {
    const BoxCopies k = w.copies(c);
    T acc[NC];
#pragma unroll
    for (int j = 0; j < NC; j++) {
      const T *__restrict__ x = p.x[j];
      const T *__restrict__ uin = p.uin[j];
      const T *__restrict__ Kj = p.K[j];
      T s = T(0);
      k.each([&](int m) {
        T v = x[m];
        if (MODE == FUSE_EULER)
          v = rk_euler_point(v, dt, uin[m], a, p.y[j], b, a2, p.y2[j], b2, (int64_t)m);
        if (MODE == FUSE_ACCUM_BEFORE) v = rk_accum_point(v, Kj[m], ch);
        s = __fadd_rn_t(s, v);
      });
      acc[j] = s / (T)k.count();
    }
#pragma unroll
    for (int j = 0; j < NC; j++) {
      T *__restrict__ x = p.x[j];
      T *__restrict__ ao = p.acc[j];
      k.each([&](int m) {
        x[m] = acc[j];
        if (MODE == FUSE_ACCUM_AFTER) ao[m] = rk_accum_point(ao[m], acc[j], ch);
      });
    }
  }
}

// k_dss_box Smooth on every state component in one pass
template <typename T, int NC>
__global__ void __launch_bounds__(256) k_dss_smooth_box_n(RKComps<T> p, BoxWalk w) {
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w.nL;
       c = (c < w.nL - stride) ? c + stride : w.nL) {
    const BoxCopies k = w.copies(c);
    T acc[NC];
#pragma unroll
    for (int j = 0; j < NC; j++) acc[j] = box_fold<T, GF_DSS_SMOOTH>(p.x[j], k);
#pragma unroll
    for (int j = 0; j < NC; j++) {
      T *__restrict__ x = p.x[j];
      k.each([&](int m) { x[m] = acc[j]; });
    }
  }
}

}  // namespace gfk

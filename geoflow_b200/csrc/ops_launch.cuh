// ops_launch.cuh -- host launchers for the per-order kernel templates,
// selected at run time by dispatch_n over the GLL point count.
#pragma once
#include <type_traits>
#include <unordered_map>

#include "gf_common.cuh"
#include "k_def.cuh"
#include "k_dudt.cuh"
#include "k_helm_k1.cuh"
#include "k_helm_tf32.cuh"
#include "k_tensor.cuh"

namespace gfk {

// Library-wide choice of the FP32 3-d affine apply at p = 7 (gf_set_fp32_apply).
extern int g_fp32_apply_mode;

// Raises a kernel's dynamic shared-memory limit once per kernel (several
// kernels share one function type, so the record is keyed by address).
template <typename K>
inline void set_smem(K kern, size_t bytes) {
  static std::unordered_map<const void *, size_t> done;
  size_t &have = done[(const void *)kern];
  if (bytes > have) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    have = bytes;
  }
}

// Deformed / embedded elements (k_def.cuh): one element per block.
template <typename T, class LD>
struct DefLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, int mode, T p, const T *pvec, T q, const T *qvec,
                   int use_mass, LD ld, int nv, const T *const *c, int idir, T *uo,
                   cudaStream_t st, const double *stop) {
      const Basis<T, N> B = make_basis<T, N>(prob);
      const DefGeom<T> g = def_of<T>(prob);
      const T *cc[3] = {nullptr, nullptr, nullptr};
      for (int k = 0; k < nv; k++) cc[k] = c[k];
      const int NE = prob->dim == 3 ? N * N * N : N * N;
      const size_t smem = sizeof(T) * (1 + 2 * prob->dim) * NE;
      const int threads = NE < 256 ? ((NE + 31) / 32) * 32 : 256;
      prob->launches++;
      if (prob->dim == 3) {
        auto kern = k_def<T, N, 3, LD, T>;
        set_smem(kern, smem);
        kern<<<(unsigned)prob->ne, threads, smem, st>>>(B, g, prob->ne, mode, p, pvec, q, qvec,
                                                        use_mass, ld, nv, cc[0], cc[1], cc[2], idir,
                                                        imass_of<T>(prob), uo, stop);
      } else {
        auto kern = k_def<T, N, 2, LD, T>;
        set_smem(kern, smem);
        kern<<<(unsigned)prob->ne, threads, smem, st>>>(B, g, prob->ne, mode, p, pvec, q, qvec,
                                                        use_mass, ld, nv, cc[0], cc[1], cc[2], idir,
                                                        imass_of<T>(prob), uo, stop);
      }
      return GF_OK;
    }
  };
};

template <typename T, class LD, typename TO = T>
struct HelmLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, T p, const T *pvec, T q, const T *qvec, int use_mass,
                   LD ld, TO *uo, cudaStream_t st, const double *stop) {
      if (prob->geom >= GF_GEOM_DEFORMED) {  // full per-node metric
        if constexpr (!std::is_same<T, TO>::value) {
          return GF_ERR_UNSUPPORTED;
        } else {
          return DefLaunch<T, LD>::template F<N>::run(prob, DEF_HELM, p, pvec, q, qvec, use_mass,
                                                      ld, 0, nullptr, 0, uo, st, stop);
        }
      }
      const Geom<T> g = geom_of<T>(prob);
      constexpr int P = Pad<N>::P;
      if constexpr (std::is_same<T, float>::value && N == 8) {
        if (prob->dim == 3 && g.egeom && !pvec && g_fp32_apply_mode == GF_FP32_APPLY_TF32) {
          // affine elements, scalar p, p = 7: the K1 contractions as 3xTF32
          // tensor-core products (k_helm_tf32.cuh)
          constexpr int EPB = 4;
          const Tf32Basis TB = make_tf32basis(prob);
          const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
          prob->launches++;
          k_helm3d_tf32<EPB, LD, TO><<<grid, dim3(64, EPB), 0, st>>>(TB, g.egeom, prob->ne, p, q,
                                                                    qvec, use_mass, ld, uo, stop);
          return GF_OK;
        }
      }
      if (prob->dim == 3 && g.egeom && !pvec) {
        // affine elements, scalar p: one K1 contraction per direction
        constexpr int EPB = epb_k1<N>();
        const K1Basis<T, N> KB = make_k1basis<T, N>(prob);
        const size_t smem = sizeof(T) * 2 * N * N * P * EPB;
        auto kern = k_helm3d_k1<T, N, EPB, LD, TO>;
        set_smem(kern, smem);
        const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
        prob->launches++;
        kern<<<grid, dim3(N * N, EPB), smem, st>>>(KB, g.egeom, prob->ne, p, q, qvec, use_mass, ld,
                                                    uo, stop);
        return GF_OK;
      }
      const Basis<T, N> B = make_basis<T, N>(prob);
      if (prob->dim == 3) {
        constexpr int EPB = epb3<N>();
        const size_t smem = sizeof(T) * 3 * N * N * P * EPB;
        auto kern = k_helm3d<T, N, EPB, LD, TO>;
        set_smem(kern, smem);
        const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
        prob->launches++;
        kern<<<grid, dim3(N * N, EPB), smem, st>>>(B, g, prob->ne, p, pvec, q, qvec, use_mass, ld,
                                                    uo, stop);
      } else if constexpr (!std::is_same<T, TO>::value) {
        return GF_ERR_UNSUPPORTED;  // mixed storage/arithmetic is 3-d only
      } else {
        constexpr int EPB = epb2<N>();
        const size_t smem = sizeof(T) * 3 * N * P * EPB;
        auto kern = k_helm2d<T, N, EPB, LD>;
        set_smem(kern, smem);
        const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
        prob->launches++;
        kern<<<grid, dim3(N * N, EPB), smem, st>>>(B, g, prob->ne, p, pvec, q, qvec, use_mass, ld,
                                                    uo, stop);
      }
      return GF_OK;
    }
  };
};

template <typename T>
struct DerivLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, const T *u, int idir, int dotrans, int phys, int accum, T *du,
                   cudaStream_t st) {
      const Basis<T, N> B = make_basis<T, N>(prob);
      const Geom<T> g = geom_of<T>(prob);
      if (prob->dim == 3) {
        const size_t smem = sizeof(T) * N * N * N;
        auto kern = k_grefderiv<T, N, 3, 1>;
        set_smem(kern, smem);
        prob->launches++;
        kern<<<(unsigned)prob->ne, dim3(N * N, 1), smem, st>>>(B, g, prob->ne, u, idir, dotrans,
                                                                phys, accum, du);
      } else {
        constexpr int EPB = epb2<N>();
        const size_t smem = sizeof(T) * N * N * EPB;
        auto kern = k_grefderiv<T, N, 2, EPB>;
        set_smem(kern, smem);
        const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
        prob->launches++;
        kern<<<grid, dim3(N * N, EPB), smem, st>>>(B, g, prob->ne, u, idir, dotrans, phys, accum, du);
      }
      return GF_OK;
    }
  };
};

template <typename T, int N, int EQN, int MODE>
inline void launch_dudt_kernel(gf_problem *prob, T nu, const T *const *f, T *const *o,
                               const T *imass, cudaStream_t st, const RKEpi<T> &epi) {
  const Basis<T, N> B = make_basis<T, N>(prob);
  const Geom<T> g = geom_of<T>(prob);
  constexpr int P = Pad<N>::P;
  if (prob->dim == 3) {
    constexpr int NF = EQN == GF_EQN_ADVECT ? 4 : (EQN == GF_EQN_BURGERS ? 3 : 1);
    constexpr int EPB = epb_dudt3<N, NF>();
    const size_t smem = sizeof(T) * dudt_slot<T, N, NF>() * EPB;
    auto kern = g.egeom ? k_dudt3d<T, N, EPB, EQN, MODE, true> : k_dudt3d<T, N, EPB, EQN, MODE, false>;
    set_smem(kern, smem);
    const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
    prob->launches++;
    kern<<<grid, dim3(N * N, EPB), smem, st>>>(B, g, prob->ne, nu, f[0], f[1], f[2], f[3], imass,
                                                o[0], o[1], o[2], epi);
  } else {
    constexpr int NF = EQN == GF_EQN_ADVECT ? 3 : (EQN == GF_EQN_BURGERS ? 2 : 1);
    constexpr int EPB = epb2<N>();
    const size_t smem = sizeof(T) * (NF + 2) * N * P * EPB;
    auto kern = k_dudt2d<T, N, EPB, EQN, MODE>;
    set_smem(kern, smem);
    const unsigned grid = (unsigned)((prob->ne + EPB - 1) / EPB);
    prob->launches++;
    kern<<<grid, dim3(N * N, EPB), smem, st>>>(B, g, prob->ne, nu, f[0], f[1], f[2], f[3], imass,
                                                o[0], o[1], o[2], epi);
  }
}

template <typename T>
struct DudtLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, int eqn, int mode, T nu, const T *const *f, T *const *o,
                   cudaStream_t st, const RKEpi<T> &epi) {
      const T *im = imass_of<T>(prob);
      if (mode == MODE_EULER) {
        if (prob->dim != 3) return GF_ERR_UNSUPPORTED;
        if (eqn == GF_EQN_ADVECT)
          launch_dudt_kernel<T, N, GF_EQN_ADVECT, MODE_EULER>(prob, nu, f, o, im, st, epi);
        else if (eqn == GF_EQN_BURGERS)
          launch_dudt_kernel<T, N, GF_EQN_BURGERS, MODE_EULER>(prob, nu, f, o, im, st, epi);
        else
          launch_dudt_kernel<T, N, GF_EQN_HEAT, MODE_EULER>(prob, nu, f, o, im, st, epi);
      } else if (eqn == GF_EQN_ADVECT && mode == MODE_ADVECT)
        launch_dudt_kernel<T, N, GF_EQN_ADVECT, MODE_ADVECT>(prob, nu, f, o, im, st, epi);
      else if (eqn == GF_EQN_ADVECT)
        launch_dudt_kernel<T, N, GF_EQN_ADVECT, MODE_DUDT>(prob, nu, f, o, im, st, epi);
      else if (eqn == GF_EQN_BURGERS)
        launch_dudt_kernel<T, N, GF_EQN_BURGERS, MODE_DUDT>(prob, nu, f, o, im, st, epi);
      else
        launch_dudt_kernel<T, N, GF_EQN_HEAT, MODE_DUDT>(prob, nu, f, o, im, st, epi);
      return GF_OK;
    }
  };
};

}  // namespace gfk

// launchers shared across translation units
template <typename T>
int launch_helm(gf_problem *prob, T p, const T *pvec, T q, const T *qvec, int use_mass,
                const T *u, T *uo, cudaStream_t st, const double *stop = nullptr);
// same operator on a unique-node input wL (gathered per element), writing
// the element-local result uo
template <typename T>
int launch_helm_L(gf_problem *prob, T p, T q, int use_mass, const T *wL, T *uo, cudaStream_t st,
                  const double *stop = nullptr);
// FP32-stored input and output, FP64 arithmetic (3-d)
int launch_helm_L_f32io(gf_problem *prob, double p, double q, int use_mass, const float *wL,
                        float *uo, cudaStream_t st, const double *stop);
template <typename T>
int launch_dss(gf_problem *prob, int op, T *u, cudaStream_t st);
template <typename T>
int launch_dudt(gf_problem *prob, int eqn, int mode, T nu, const T *const *f, T *const *o,
                cudaStream_t st, const gfk::RKEpi<T> *epi = nullptr);

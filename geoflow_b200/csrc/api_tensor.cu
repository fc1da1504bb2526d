// api_tensor.cu -- full tensor products of per-direction matrices,
//   out = (A3 (x) A2 (x) A1) u   in every element (2-d: (A2 (x) A1) u),
// the GMTK forms D2_X_D1 (blas/gmtk.ipp:1570-1619) and D3_X_D2_X_D1
// (1930-1996), their weighted variants (Dg2_X_D1, D2_X_Dg1,
// Dg3_X_Dg2_X_D1, ... 1639-1911, 2311-2519: the weights are folded into
// the matrices by the caller), and the spectral filter application of
// GBoydFilter / GProjectionFilter::apply_impl (sem/gboyd_filter.ipp), which
// is D3_X_D2_X_D1(F, F^T, F^T) with the basis' filter matrix F.
// A_d(i,m) = A_d[i + m*n] (column-major like the GLL D); A_d acts along
// direction d: out(i,j,k) = sum A1(i,i') A2(j,j') A3(k,k') u(i',j',k').
// Per element one thread per (i,j) column: x-, y- and z-lines are
// contracted in turn through shared memory (the z-line in registers).
#include "gf_common.cuh"
#include "k_tensor.cuh"

using namespace gfk;

namespace {

template <typename T, int N>
struct TMats {
  T A[3][N * N];
};

template <typename T, int N>
__device__ __forceinline__ void line_apply(const T *__restrict__ A, const T (&a)[N], T (&y)[N]) {
#pragma unroll
  for (int i = 0; i < N; i++) {
    T s = A[i] * a[0];
#pragma unroll
    for (int m = 1; m < N; m++) s = fma(A[i + m * N], a[m], s);
    y[i] = s;
  }
}

template <typename T, int N, int DIM, int EPB>
__global__ void __launch_bounds__(N *N *EPB)
    k_tensor_apply(const __grid_constant__ TMats<T, N> M, int64_t ne, const T *__restrict__ u,
                   T *__restrict__ out) {
  constexpr int P = Pad<N>::P, PLANE = N * P, NN = N * N;
  constexpr int VOL = DIM == 3 ? N * PLANE : PLANE, NE = DIM == 3 ? NN * N : NN;
  extern __shared__ __align__(16) unsigned char smem_t[];
  T *s = reinterpret_cast<T *>(smem_t) + threadIdx.y * VOL;
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int a0 = t % N, a1 = t / N;
  const int64_t base = e * NE;
  if (DIM == 2) {
    // thread (i=a0, j=a1): x-lines by row j, then y-lines by column i
    s[a1 * P + a0] = active ? u[base + a1 * N + a0] : T(0);
    __syncthreads();
    T a[N], y[N];
    if (a1 == 0) {  // N threads own the N x-lines
#pragma unroll
      for (int m = 0; m < N; m++) a[m] = s[a0 * P + m];
      line_apply<T, N>(M.A[0], a, y);
#pragma unroll
      for (int i = 0; i < N; i++) s[a0 * P + i] = y[i];
    }
    __syncthreads();
    if (a1 == 0) {
#pragma unroll
      for (int m = 0; m < N; m++) a[m] = s[m * P + a0];
      line_apply<T, N>(M.A[1], a, y);
      if (active) {
#pragma unroll
        for (int j = 0; j < N; j++) out[base + j * N + a0] = y[j];
      }
    }
    return;
  }
  T rz[N];
#pragma unroll
  for (int k = 0; k < N; k++) rz[k] = active ? u[base + k * NN + a1 * N + a0] : T(0);
#pragma unroll
  for (int k = 0; k < N; k++) s[k * PLANE + a1 * P + a0] = rz[k];
  __syncthreads();
  {  // x-line (j=a0, k=a1), in place
    T a[N], y[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = s[a1 * PLANE + a0 * P + m];
    line_apply<T, N>(M.A[0], a, y);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < N; i++) s[a1 * PLANE + a0 * P + i] = y[i];
  }
  __syncthreads();
  {  // y-line (i=a0, k=a1), in place
    T a[N], y[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = s[a1 * PLANE + m * P + a0];
    line_apply<T, N>(M.A[1], a, y);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < N; j++) s[a1 * PLANE + j * P + a0] = y[j];
  }
  __syncthreads();
  {  // z-line (i=a0, j=a1) to the output
    T a[N], y[N];
#pragma unroll
    for (int m = 0; m < N; m++) a[m] = s[m * PLANE + a1 * P + a0];
    line_apply<T, N>(M.A[2], a, y);
    if (active) {
#pragma unroll
      for (int k = 0; k < N; k++) out[base + k * NN + a1 * N + a0] = y[k];
    }
  }
}

template <typename T>
struct TensorLaunch {
  template <int N>
  struct F {
    static int run(gf_problem *prob, const double *const *A, const T *u, T *out, cudaStream_t st) {
      TMats<T, N> M;
      for (int d = 0; d < 3; d++)
        for (int i = 0; i < N * N; i++) M.A[d][i] = (d < prob->dim) ? (T)A[d][i] : T(0);
      constexpr int P = Pad<N>::P;
      prob->launches++;
      if (prob->dim == 3) {
        constexpr int EPB = epb3<N>();
        const size_t smem = sizeof(T) * N * N * P * EPB;
        auto kern = k_tensor_apply<T, N, 3, EPB>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<(unsigned)((prob->ne + EPB - 1) / EPB), dim3(N * N, EPB), smem, st>>>(M, prob->ne,
                                                                                     u, out);
      } else {
        constexpr int EPB = epb2<N>();
        const size_t smem = sizeof(T) * N * P * EPB;
        auto kern = k_tensor_apply<T, N, 2, EPB>;
        kern<<<(unsigned)((prob->ne + EPB - 1) / EPB), dim3(N * N, EPB), smem, st>>>(M, prob->ne,
                                                                                     u, out);
      }
      return cudaPeekAtLastError() == cudaSuccess ? GF_OK : GF_ERR_CUDA;
    }
  };
};

}  // namespace

extern "C" int gf_tensor_apply(gf_problem_t prob, int dtype, const double *A1, const double *A2,
                               const double *A3, const void *u, void *out) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, A1 && A2 && (prob->dim == 2 || A3) && u && out, "bad arguments");
  GF_REQUIRE(ctx, u != out, "out must not alias u");
  const double *A[3] = {A1, A2, prob->dim == 3 ? A3 : A1};
  int rc = dtype == GF_F64
               ? dispatch_n<TensorLaunch<double>::template F>(prob->n, prob, A, (const double *)u,
                                                             (double *)out, ctx->stream)
           : dtype == GF_F32
               ? dispatch_n<TensorLaunch<float>::template F>(prob->n, prob, A, (const float *)u,
                                                            (float *)out, ctx->stream)
               : GF_ERR_ARG;
  if (rc) return gf_fail(ctx, rc, "tensor apply failed");
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

// Spectral filter in place: the tensor kernel reads each element's values
// before writing any of them, and no other block reads the element.
extern "C" int gf_filter_apply(gf_problem_t prob, int dtype, const double *F1, const double *F2,
                               const double *F3, int ncomp, void *const *u) {
  if (!prob) return GF_ERR_ARG;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, F1 && F2 && (prob->dim == 2 || F3) && u && ncomp >= 1, "bad arguments");
  const double *A[3] = {F1, F2, prob->dim == 3 ? F3 : F1};
  for (int k = 0; k < ncomp; k++) {
    GF_REQUIRE(ctx, u[k], "component %d missing", k);
    int rc = dtype == GF_F64
                 ? dispatch_n<TensorLaunch<double>::template F>(prob->n, prob, A, (const double *)u[k],
                                                               (double *)u[k], ctx->stream)
             : dtype == GF_F32
                 ? dispatch_n<TensorLaunch<float>::template F>(prob->n, prob, A, (const float *)u[k],
                                                              (float *)u[k], ctx->stream)
                 : GF_ERR_ARG;
    if (rc) return gf_fail(ctx, rc, "filter apply failed");
  }
  GF_CHECK_LAUNCH(ctx);
  return GF_OK;
}

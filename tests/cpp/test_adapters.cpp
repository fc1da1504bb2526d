// C++ host-side check of the gfgpu.hpp adapters: the known answer of the
// reference's cdg_cg test (test/actions/cdg/cdg_cg.cpp:113-341,
// data/cg_input.jsn) -- 2-d box, 4x4 elements, p = 6, -lap u = f with
// u = y(1-y)x^3, Dirichlet data, CG tol 1e-7, INF norm, maxit 256; pass
// when the integral of (u - ua)^2 over the volume is below 1e-12.
// Also applies GGFX Smooth to a continuous field (cdg_ggfx.cpp:158-235:
// values must come back bit-identical).  Exit status 0 on success.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/gfgpu.hpp"

int main() {
  using namespace gfgpu;
  Context ctx(0);
  BoxGrid g(2, {4, 4}, 6, {0.0, 0.0}, {1.0, 1.0}, {0, 0});
  Problem prob(ctx, g);
  const int64_t N = g.ndof();
  std::vector<double> f(N), ua(N), ub(N, 0.0), mass(N), one(N, 1.0);
  const double eps = 100 * 2.220446049250313e-16;
  for (int64_t i = 0; i < N; i++) {
    const double x = g.xyz[0][i], y = g.xyz[1][i];
    f[i] = 6.0 * x * y * (1.0 - y) - 2.0 * x * x * x;
    ua[i] = y * (1.0 - y) * x * x * x;
    if (std::fabs(x - 1.0) <= eps) ub[i] = y * (1.0 - y);
  }
  double *d_f, *d_b, *d_ub, *d_u, *d_m, *d_one;
  cudaMalloc(&d_f, N * 8);
  cudaMalloc(&d_b, N * 8);
  cudaMalloc(&d_ub, N * 8);
  cudaMalloc(&d_u, N * 8);
  cudaMalloc(&d_m, N * 8);
  cudaMalloc(&d_one, N * 8);
  cudaMemcpy(d_f, f.data(), N * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_ub, ub.data(), N * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_one, one.data(), N * 8, cudaMemcpyHostToDevice);
  cudaMemset(d_u, 0, N * 8);
  // b = -M_L f
  check(ctx.get(), gf_mass_apply(prob.get(), GF_F64, 0, d_one, d_m), "mass");
  cudaDeviceSynchronize();
  cudaMemcpy(mass.data(), d_m, N * 8, cudaMemcpyDeviceToHost);
  std::vector<double> b(N);
  for (int64_t i = 0; i < N; i++) b[i] = -(f[i] * mass[i]);
  cudaMemcpy(d_b, b.data(), N * 8, cudaMemcpyHostToDevice);

  Helmholtz L(prob);
  gf_cg_traits tr{};
  tr.maxit = 256;
  tr.normtype = GF_NORM_INF;
  tr.tol = 1e-7;
  tr.precond = GF_PRECOND_NONE;
  tr.precision = GF_CG_FP64;
  tr.check_every = 8;
  CG cg(tr, prob);
  int rc = cg.solve(L, d_b, d_ub, d_u);
  std::vector<double> u(N);
  cudaMemcpy(u.data(), d_u, N * 8, cudaMemcpyDeviceToHost);
  double num = 0.0, vol = 0.0;
  for (int64_t i = 0; i < N; i++) {
    num += mass[i] * (u[i] - ua[i]) * (u[i] - ua[i]);
    vol += mass[i];
  }
  const double err = num / vol;
  std::printf("cdg_cg: rc=%d iterations=%d err=%.3e\n", rc, cg.iterations(), err);
  if (rc != CG::GCGERR_NONE || !(err < 1e-12)) return 1;

  // the reference's three-argument opVec_prod(in, utmp, out) gives the
  // two-argument result bit for bit
  {
    std::vector<double> utmp;  // stands in for the reference's State utmp
    double *d_o1 = nullptr, *d_o2 = nullptr;
    cudaMalloc(&d_o1, N * 8);
    cudaMalloc(&d_o2, N * 8);
    L.opVec_prod(d_u, d_o1);
    L.opVec_prod(d_u, utmp, d_o2);
    cudaDeviceSynchronize();
    std::vector<double> o1(N), o2(N);
    cudaMemcpy(o1.data(), d_o1, N * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(o2.data(), d_o2, N * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_o1);
    cudaFree(d_o2);
    if (std::memcmp(o1.data(), o2.data(), N * 8) != 0) return 3;
  }

  // GGFX Smooth of a continuous field leaves it bit-identical
  std::vector<double> h(N);
  for (int64_t i = 0; i < N; i++) {
    const int32_t first = g.members[g.class_ptr[g.node_class[i]]];
    h[i] = 1.0 + 2.0 * g.xyz[0][first] + 3.0 * g.xyz[1][first];
  }
  cudaMemcpy(d_f, h.data(), N * 8, cudaMemcpyHostToDevice);
  GGFX ggfx(prob);
  ggfx.doOp(d_f, GGFX::Smooth);
  std::vector<double> h2(N);
  cudaDeviceSynchronize();
  cudaMemcpy(h2.data(), d_f, N * 8, cudaMemcpyDeviceToHost);
  if (std::memcmp(h.data(), h2.data(), N * 8) != 0) {
    std::printf("GGFX Smooth changed a continuous field\n");
    return 2;
  }
  std::printf("adapters ok\n");
  cudaFree(d_f);
  cudaFree(d_b);
  cudaFree(d_ub);
  cudaFree(d_u);
  cudaFree(d_m);
  cudaFree(d_one);
  return 0;
}

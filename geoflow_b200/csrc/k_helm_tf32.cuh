// k_helm_tf32.cuh -- FP32 3-d Helmholtz apply for affine elements at
// p = 7 (N = 8) with the line contractions on the tensor cores.
//
// The arithmetic is that of k_helm3d_k1 (k_helm_k1.cuh): per direction d
// the chain D_d^T diag(W) D_d along a line is the symmetric 1-d matrix
// K1 = D^T diag(W) D times a per-line constant, so the x-, y- and z-
// contractions of an element are three 64 x 8 by 8 x 8 matrix products
//     Y_d = diag(c_d) U_d K1,   U_d = the element's 64 d-lines as rows,
// which map onto mma.sync m16n8k8 with TF32 operands: 4 tiles of 16 lines
// per direction and element.  TF32 keeps 10 mantissa bits, so each operand
// is split into a TF32 head and a TF32 tail (x = hi + lo, hi = x with the
// low 13 mantissa bits cleared, lo = x - hi) and a product is accumulated in FP32 as lo*Bhi + hi*Blo + hi*Bhi
// ("3xTF32"): the lost lo*lo term is ~2^-22 relative, the accuracy of an
// FP32 contraction.  Directions accumulate in FP32 through the mma's C
// operand: the x-pass writes diag(c_x) U_x K1 + q M u into a result plane,
// the y-pass adds into it, and the z-pass adds its part and stores the
// node values.
//
// Thread layout: 64 threads (two warps) per element, EPB elements per
// block; warp w of an element takes tiles 2w and 2w+1 of every direction.
// Shared memory per element: u and the result R, each [k][j][i] with planes
// of 72 words and rows of 8 whose halves swap for j >= 4 (column i stored
// at i ^ (j & 4)): the A-fragment loads of all three directions and the
// z-line stores are then free of bank conflicts.  The two warps of an
// element meet at a named barrier of 64 threads (ids 1..EPB).
//
// mma.m16n8k8 fragments (PTX ISA, TF32 A/B, FP32 C/D), lane = 4 g + t:
//   A (16 x 8, row): a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4)
//   B (8 x 8, col):  b0 (t, g), b1 (t+4, g)
//   C/D (16 x 8):    c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1)
#pragma once
#include "k_helm_k1.cuh"

namespace gfk {

struct Tf32Basis {
  float K1[64];  // K1(l, m) at l + 8 m (symmetric)
  float W[8];
};

inline Tf32Basis make_tf32basis(const gf_problem *p) {
  Tf32Basis b{};
  for (int i = 0; i < 64; i++) b.K1[i] = (float)p->K1[i];
  for (int i = 0; i < 8; i++) b.W[i] = (float)p->W[i];
  return b;
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo in TF32 (hi the nearest TF32, lo the nearest TF32 of the rest)
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

// The same split by truncation, in two integer/float instructions: hi = x
// with its 13 low mantissa bits cleared (a TF32 value), lo = x - hi (exact
// in FP32); the mma reads the TF32 part of lo, an error of at most 2^-11
// |lo| <= 2^-21 |x|.
__device__ __forceinline__ void tf32_split_fast(float x, uint32_t &hi, uint32_t &lo) {
  hi = __float_as_uint(x) & 0xffffe000u;
  lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += diag(rows) A K1 in 3xTF32, A given in FP32 (a0..a3 of the fragment),
// the row scales already applied.
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const float (&a)[4], uint32_t bh0,
                                           uint32_t bh1, uint32_t bl0, uint32_t bl1) {
  uint32_t ah[4], al[4];
#pragma unroll
  for (int r = 0; r < 4; r++) tf32_split_fast(a[r], ah[r], al[r]);
  mma_tf32(d, al, bh0, bh1);
  mma_tf32(d, ah, bl0, bl1);
  mma_tf32(d, ah, bh0, bh1);
}

__device__ __forceinline__ void elem_barrier(int id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

template <int EPB> constexpr int epb_tf32() { return EPB; }

// uo = p sum_d D_d^T (M G_d D_d u) + q M u   (qvec: per-node q), N = 8.
template <int EPB, class LD, typename TO = float>
__global__ void __launch_bounds__(64 * EPB)
    k_helm3d_tf32(const __grid_constant__ Tf32Basis B, const float *__restrict__ egeom, int64_t ne,
                  float p, float q, const float *__restrict__ qvec, int use_mass, const LD ld,
                  TO *__restrict__ uo, const double *__restrict__ stop) {
  if (stop && stop[0] != 0.0) return;
  constexpr int PL = 72, VOL = 8 * PL;
  __shared__ __align__(16) float smem[EPB * 2 * VOL];
  float *su = smem + threadIdx.y * 2 * VOL;
  float *sr = su + VOL;
  auto at = [](int k, int j, int i) { return k * PL + j * 8 + (i ^ (j & 4)); };
  const int t = threadIdx.x;
  const int64_t e = (int64_t)blockIdx.x * EPB + threadIdx.y;
  const bool active = e < ne;
  const int64_t base = e * 512;
  const int bar = threadIdx.y + 1;

  // 1. z-line of thread (i, j) = (t % 8, t / 8) into shared memory
  {
    const int i = t & 7, j = t >> 3;
    float ru[8];
    if (active) {
      typename LD::value_type lv[8];
      ld.template zline<8>(e, i, j, lv);
#pragma unroll
      for (int k = 0; k < 8; k++) ru[k] = (float)lv[k];
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) ru[k] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) su[at(k, j, i)] = ru[k];
  }

  // per-element constants and this lane's fragment coordinates
  const int lane = t & 31, w = t >> 5, g = lane >> 2, tg = lane & 3;
  float J = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
  if (active) {
    const float *ge = egeom + e * 4;
    gx = ge[0];
    gy = ge[1];
    gz = ge[2];
    J = ge[3];
  }
  const float pj = p * J;
  const float cxs = pj * gx * gx, cys = pj * gy * gy, czs = pj * gz * gz;
  const float cm = (qvec ? 1.0f : q) * J;
  // B = K1 (symmetric): b0 = K1(t, g), b1 = K1(t+4, g), split once
  uint32_t bh0, bl0, bh1, bl1;
  tf32_split(B.K1[tg + 8 * g], bh0, bl0);
  tf32_split(B.K1[tg + 4 + 8 * g], bh1, bl1);
  const float Wg = B.W[g];
  elem_barrier(bar);

  // 2. x-lines: line (j, k) = row, i = column; R = c_x U_x K1 + q M u
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int tile = 2 * w + h, k0 = 2 * tile;  // rows g -> (j=g, k=k0), g+8 -> (g, k0+1)
    const float c0 = cxs * Wg * B.W[k0], c1 = cxs * Wg * B.W[k0 + 1];
    float a[4];
    a[0] = c0 * su[at(k0, g, tg)];
    a[1] = c1 * su[at(k0 + 1, g, tg)];
    a[2] = c0 * su[at(k0, g, tg + 4)];
    a[3] = c1 * su[at(k0 + 1, g, tg + 4)];
    // mass term at the output positions (i = 2tg, 2tg+1; j = g; k0, k0+1)
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (use_mass) {
#pragma unroll
      for (int r = 0; r < 2; r++) {
        const int k = k0 + r;
        const float2 uu = *reinterpret_cast<const float2 *>(&su[at(k, g, 2 * tg)]);
        float m0 = cm * Wg * B.W[k] * B.W[2 * tg], m1 = cm * Wg * B.W[k] * B.W[2 * tg + 1];
        if (qvec) {
          const int64_t n0 = base + k * 64 + g * 8 + 2 * tg;
          m0 *= qvec[n0];
          m1 *= qvec[n0 + 1];
        }
        d[2 * r] = m0 * uu.x;
        d[2 * r + 1] = m1 * uu.y;
      }
    }
    mma_3xtf32(d, a, bh0, bh1, bl0, bl1);
    *reinterpret_cast<float2 *>(&sr[at(k0, g, 2 * tg)]) = make_float2(d[0], d[1]);
    *reinterpret_cast<float2 *>(&sr[at(k0 + 1, g, 2 * tg)]) = make_float2(d[2], d[3]);
  }
  elem_barrier(bar);

  // 3. y-lines: line (i, k) = row, j = column; R += c_y U_y K1
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int tile = 2 * w + h, k0 = 2 * tile;  // rows g -> (i=g, k=k0), g+8 -> (g, k0+1)
    const float c0 = cys * Wg * B.W[k0], c1 = cys * Wg * B.W[k0 + 1];
    float a[4];
    a[0] = c0 * su[at(k0, tg, g)];
    a[1] = c1 * su[at(k0 + 1, tg, g)];
    a[2] = c0 * su[at(k0, tg + 4, g)];
    a[3] = c1 * su[at(k0 + 1, tg + 4, g)];
    float d[4];
    d[0] = sr[at(k0, 2 * tg, g)];
    d[1] = sr[at(k0, 2 * tg + 1, g)];
    d[2] = sr[at(k0 + 1, 2 * tg, g)];
    d[3] = sr[at(k0 + 1, 2 * tg + 1, g)];
    mma_3xtf32(d, a, bh0, bh1, bl0, bl1);
    sr[at(k0, 2 * tg, g)] = d[0];
    sr[at(k0, 2 * tg + 1, g)] = d[1];
    sr[at(k0 + 1, 2 * tg, g)] = d[2];
    sr[at(k0 + 1, 2 * tg + 1, g)] = d[3];
  }
  elem_barrier(bar);

  // 4. z-lines: line (i, j) = row, k = column; out = R + c_z U_z K1
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int tile = 2 * w + h, j0 = 2 * tile;  // rows g -> (i=g, j=j0), g+8 -> (g, j0+1)
    const float c0 = czs * Wg * B.W[j0], c1 = czs * Wg * B.W[j0 + 1];
    float a[4];
    a[0] = c0 * su[at(tg, j0, g)];
    a[1] = c1 * su[at(tg, j0 + 1, g)];
    a[2] = c0 * su[at(tg + 4, j0, g)];
    a[3] = c1 * su[at(tg + 4, j0 + 1, g)];
    float d[4];
    d[0] = sr[at(2 * tg, j0, g)];
    d[1] = sr[at(2 * tg + 1, j0, g)];
    d[2] = sr[at(2 * tg, j0 + 1, g)];
    d[3] = sr[at(2 * tg + 1, j0 + 1, g)];
    mma_3xtf32(d, a, bh0, bh1, bl0, bl1);
    if (active) {
      TO *o = uo + base + g;
      o[(2 * tg) * 64 + j0 * 8] = (TO)d[0];
      o[(2 * tg + 1) * 64 + j0 * 8] = (TO)d[1];
      o[(2 * tg) * 64 + (j0 + 1) * 8] = (TO)d[2];
      o[(2 * tg + 1) * 64 + (j0 + 1) * 8] = (TO)d[3];
    }
  }
}

}  // namespace gfk

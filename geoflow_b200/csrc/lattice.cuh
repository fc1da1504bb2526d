// lattice.cuh -- the unique-node lattice of a regular box grid (GGridBox,
// grid/ggrid_box.ipp).  The unique nodes of a box are the points of the
// global GLL lattice, M_d = ne_d p (+1 when direction d is not periodic);
// GGFX::init (comm/ggfx.hpp:169-342) finds exactly these classes by
// coordinate matching after the periodize step.  The class of node
// (e; i,j,k) and the members of a lattice point follow from the element
// coordinates alone, so no index array is read.
#pragma once
#include <cstdint>

namespace gfk {

struct BoxLattice {
  int dim;
  int ne[3];
  int per[3];
  int p;            // polynomial order (n = p+1 points per direction)
  int64_t M[3];     // lattice points per direction
  __host__ __device__ void elem_coords(int64_t e, int (&c)[3]) const {
    c[0] = (int)(e % ne[0]);
    int64_t r = e / ne[0];
    c[1] = (int)(r % ne[1]);
    c[2] = dim > 2 ? (int)(r / ne[1]) : 0;
  }
  // lattice coordinate of local index l in element coordinate ec (dir d)
  __host__ __device__ int64_t g1(int d, int ec, int l) const {
    int64_t gi = (int64_t)ec * p + l;
    if (per[d] && gi == M[d]) gi = 0;
    return gi;
  }
  __host__ __device__ int64_t size() const { return M[0] * M[1] * (dim > 2 ? M[2] : 1); }
  // (element coordinate, local index) pairs of lattice coordinate g in
  // direction d; returns the count (1 or 2).  The caller orders the members.
  __device__ int cands(int d, int64_t g, int (&ec)[2], int (&l)[2]) const {
    const int64_t r = g % p, q = g / p;
    if (r != 0) {
      ec[0] = (int)q;
      l[0] = (int)r;
      return 1;
    }
    int k = 0;
    if (per[d]) {  // (q-1 mod ne, p) and (q, 0); one element when ne == 1
      ec[0] = (int)((q + ne[d] - 1) % ne[d]);
      l[0] = p;
      ec[1] = (int)q;
      l[1] = 0;
      return 2;
    }
    if (q - 1 >= 0) {
      ec[k] = (int)(q - 1);
      l[k] = p;
      k++;
    }
    if (q < ne[d]) {
      ec[k] = (int)q;
      l[k] = 0;
      k++;
    }
    return k;
  }
  __device__ void lattice_coords(int64_t c, int64_t (&g)[3]) const {
    g[0] = c % M[0];
    int64_t r = c / M[0];
    g[1] = r % M[1];
    g[2] = dim > 2 ? r / M[1] : 0;
  }
  __device__ bool dirichlet(int64_t c) const {
    int64_t g[3];
    lattice_coords(c, g);
    for (int d = 0; d < dim; d++)
      if (!per[d] && (g[d] == 0 || g[d] == M[d] - 1)) return true;
    return false;
  }
  __device__ int mult(int64_t c) const {
    int64_t g[3];
    lattice_coords(c, g);
    int m = 1;
    for (int d = 0; d < dim; d++) {
      int ec[2], l[2];
      m *= cands(d, g[d], ec, l);
    }
    return m;
  }
  // members (E indices) of lattice point c in ascending order; returns count
  __device__ int members(int64_t c, int64_t (&out)[8]) const {
    int64_t g[3];
    lattice_coords(c, g);
    int ec[3][2], l[3][2], cnt[3] = {1, 1, 1};
    for (int d = 0; d < 3; d++) {
      if (d < dim) cnt[d] = cands(d, g[d], ec[d], l[d]);
      else { ec[d][0] = 0; l[d][0] = 0; }
    }
    const int n = p + 1;
    const int64_t nn = dim > 2 ? (int64_t)n * n * n : (int64_t)n * n;
    int m = 0;
    for (int a = 0; a < cnt[2]; a++)
      for (int b = 0; b < cnt[1]; b++)
        for (int k = 0; k < cnt[0]; k++) {
          const int64_t e = ec[0][k] + (int64_t)ne[0] * (ec[1][b] + (int64_t)ne[1] * ec[2][a]);
          const int64_t loc = l[0][k] + (int64_t)n * (l[1][b] + (int64_t)n * l[2][a]);
          out[m++] = e * nn + loc;
        }
    // ascending local id (insertion sort, at most 8 entries)
    for (int i = 1; i < m; i++) {
      const int64_t v = out[i];
      int j = i - 1;
      while (j >= 0 && out[j] > v) {
        out[j + 1] = out[j];
        j--;
      }
      out[j + 1] = v;
    }
    return m;
  }
};

// n / d for 0 <= n < 2^31 by a multiply and a shift (Granlund & Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, sec. 4):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// q = (mulhi(m, n) + n) >> l  (the add cannot overflow for n < 2^31).
struct FastDiv {
  uint32_t m;
  int l;
  static FastDiv make(int d) {
    FastDiv f;
    f.l = 0;
    while ((int64_t(1) << f.l) < d) f.l++;
    f.m = (uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << f.l) - (uint64_t)d)) / (uint64_t)d + 1);
    return f;
  }
  __host__ __device__ __forceinline__ int div(int n) const {
#ifdef __CUDA_ARCH__
    const uint32_t hi = __umulhi((uint32_t)n, m);
#else
    const uint32_t hi = (uint32_t)(((uint64_t)(uint32_t)n * m) >> 32);
#endif
    return (int)((hi + (uint32_t)n) >> l);
  }
};

// The element copies of the lattice coordinate g = q P + r along one
// direction, as offsets into the E-vector (es = the element stride, ls = the
// local index stride), in ascending element coordinate; returns their
// count.  Off an element face (r != 0, most points) the one copy is
// (q, r); on a face the copies are (q - 1, P) and (q, 0), the first
// wrapping to (ne - 1, P) and coming second when periodic and q = 0, and
// only one of them on a non-periodic boundary.  (A branch-free form with
// selects executed 5-10 % more instructions per point on B200.)
__host__ __device__ __forceinline__ int lattice_offsets_qr(int q, int r, int P, int ne, int per, int es,
                                                  int ls, int &o0, int &o1) {
  if (r != 0) {
    o0 = o1 = q * es + r * ls;
    return 1;
  }
  if (per) {
    if (q == 0) {
      o0 = 0;
      o1 = (ne - 1) * es + P * ls;
    } else {
      o0 = (q - 1) * es + P * ls;
      o1 = q * es;
    }
    return 2;
  }
  if (q == 0) {
    o0 = o1 = 0;
    return 1;
  }
  o0 = (q - 1) * es + P * ls;
  o1 = q == ne ? o0 : q * es;
  return q == ne ? 1 : 2;
}
template <int P>
__device__ __forceinline__ int lattice_offsets(int g, int ne, int per, int es, int ls, int &o0,
                                               int &o1) {
  const int q = g / P;
  return lattice_offsets_qr(q, g - q * P, P, ne, per, es, ls, o0, o1);
}

// The copies of one lattice point: per direction one or two offsets.
// each() visits them in the (z, y, x) nesting, which is ascending local id
// when no periodic direction has a single element.
struct BoxCopies {
  int ox0, ox1, oy0, oy1, oz0, oz1, nx, ny, nz;
  __host__ __device__ __forceinline__ int count() const { return nx * ny * nz; }
  template <class F>
  __device__ __forceinline__ void each(F f) const {
#pragma unroll
    for (int az = 0; az < 2; az++) {
      if (az >= nz) break;
      const int oz = az ? oz1 : oz0;
#pragma unroll
      for (int ay = 0; ay < 2; ay++) {
        if (ay >= ny) break;
        const int o = oz + (ay ? oy1 : oy0);
        f(o + ox0);
        if (nx > 1) f(o + ox1);
      }
    }
  }
};

// Flat walk of a box lattice with the order a run-time value: the copies of
// lattice point c from three multiply-shift divisions, no index arrays.
// Lattice and element-local sizes below 2^31.
struct BoxWalk {
  int dim, P, ne[3], per[3], M[3], nL, es[3];
  bool sorted;  // no periodic direction with a single element
  FastDiv f0, f1, fP;
  static BoxWalk make(const BoxLattice &L) {
    BoxWalk w;
    w.dim = L.dim;
    w.P = L.p;
    const int n = L.p + 1, nn = L.dim > 2 ? n * n * n : n * n;
    w.sorted = true;
    for (int d = 0; d < 3; d++) {
      w.ne[d] = d < L.dim ? L.ne[d] : 1;
      w.per[d] = d < L.dim ? L.per[d] : 0;
      w.M[d] = d < L.dim ? (int)L.M[d] : 1;
      if (d < L.dim && L.per[d] && L.ne[d] == 1) w.sorted = false;
    }
    w.nL = w.M[0] * w.M[1] * w.M[2];
    w.es[0] = nn;
    w.es[1] = w.ne[0] * nn;
    w.es[2] = w.ne[0] * w.ne[1] * nn;
    w.f0 = FastDiv::make(w.M[0]);
    w.f1 = FastDiv::make(w.M[1]);
    w.fP = FastDiv::make(w.P);
    return w;
  }
  __host__ __device__ __forceinline__ BoxCopies copies(int c) const {
    const int row = f0.div(c), g0 = c - row * M[0];
    const int g2 = f1.div(row), g1 = row - g2 * M[1];
    BoxCopies k;
    int q = fP.div(g0);
    k.nx = lattice_offsets_qr(q, g0 - q * P, P, ne[0], per[0], es[0], 1, k.ox0, k.ox1);
    q = fP.div(g1);
    k.ny = lattice_offsets_qr(q, g1 - q * P, P, ne[1], per[1], es[1], P + 1, k.oy0, k.oy1);
    if (dim > 2) {
      q = fP.div(g2);
      k.nz = lattice_offsets_qr(q, g2 - q * P, P, ne[2], per[2], es[2], (P + 1) * (P + 1), k.oz0,
                                k.oz1);
    } else {
      k.oz0 = k.oz1 = 0;
      k.nz = 1;
    }
    return k;
  }
};

}  // namespace gfk

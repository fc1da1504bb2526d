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

}  // namespace gfk

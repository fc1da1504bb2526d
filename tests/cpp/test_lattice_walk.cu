// Host check of the box-lattice index arithmetic that the lattice-order
// kernels share (geoflow_b200/csrc/lattice.cuh):
//  * FastDiv (multiply-shift division) against integer division;
//  * BoxWalk::copies against the element-to-lattice map BoxLattice::g1: over
//    all lattice points every element-local node is visited exactly once, at
//    the lattice point its own coordinates give, and a point's copies come in
//    ascending local id whenever no periodic direction has a single element.
// Compiled by nvcc as host code only and run on the CPU (no GPU needed).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../geoflow_b200/csrc/lattice.cuh"

using namespace gfk;

static int fails = 0;
#define CHECK(cond, ...)                 \
  do {                                   \
    if (!(cond)) {                       \
      if (fails++ < 10) {                \
        std::printf("FAIL: " __VA_ARGS__); \
        std::printf("\n");               \
      }                                  \
    }                                    \
  } while (0)

static void check_fastdiv() {
  uint64_t state = 12345;
  auto rnd = [&]() {  // 31-bit values from a 64-bit LCG
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return (int)(state >> 33);
  };
  std::vector<int> ds;
  for (int d = 1; d <= 4096; d++) ds.push_back(d);
  for (int i = 0; i < 2000; i++) ds.push_back(1 + rnd() % 0x7fffffff);
  ds.push_back(0x7fffffff);
  ds.push_back(1 << 30);
  ds.push_back((1 << 30) + 1);
  for (int d : ds) {
    const FastDiv f = FastDiv::make(d);
    auto one = [&](int n) { CHECK(f.div(n) == n / d, "FastDiv %d / %d", n, d); };
    for (int n = 0; n < 3 * d + 3 && n < 20000; n++) one(n);
    for (int k = 1; k < 40; k++) {
      const int64_t a = (int64_t)k * d;
      if (a - 1 < 0x7fffffff) one((int)(a - 1));
      if (a < 0x7fffffff) one((int)a);
    }
    for (int i = 0; i < 200; i++) one(rnd());
    one(0x7fffffff);
  }
}

static void check_walk(int dim, const int (&ne)[3], const int (&per)[3], int p) {
  BoxLattice L{};
  L.dim = dim;
  L.p = p;
  int64_t nel = 1;
  for (int d = 0; d < 3; d++) {
    L.ne[d] = d < dim ? ne[d] : 1;
    L.per[d] = d < dim ? per[d] : 0;
    L.M[d] = d < dim ? (int64_t)L.ne[d] * p + (L.per[d] ? 0 : 1) : 1;
    nel *= L.ne[d];
  }
  const int n = p + 1, nn = dim > 2 ? n * n * n : n * n;
  const int64_t nE = nel * nn;
  // lattice point of every element-local node, by the element coordinates
  std::vector<int64_t> lat(nE);
  for (int64_t m = 0; m < nE; m++) {
    const int64_t e = m / nn;
    const int a = (int)(m % nn);
    int ec[3];
    L.elem_coords(e, ec);
    int64_t g = L.g1(0, ec[0], a % n) + L.M[0] * L.g1(1, ec[1], (a / n) % n);
    if (dim > 2) g += L.M[0] * L.M[1] * L.g1(2, ec[2], a / (n * n));
    lat[m] = g;
  }
  const BoxWalk w = BoxWalk::make(L);
  CHECK(w.nL == L.size(), "nL %d vs %lld", w.nL, (long long)L.size());
  std::vector<int> seen(nE, 0);
  for (int c = 0; c < w.nL; c++) {
    const BoxCopies k = w.copies(c);
    std::vector<int64_t> ms;
    for (int az = 0; az < k.nz; az++)
      for (int ay = 0; ay < k.ny; ay++)
        for (int ax = 0; ax < k.nx; ax++)
          ms.push_back((int64_t)(az ? k.oz1 : k.oz0) + (ay ? k.oy1 : k.oy0) +
                       (ax ? k.ox1 : k.ox0));
    CHECK((int)ms.size() == k.count(), "count at %d", c);
    for (size_t i = 0; i < ms.size(); i++) {
      const int64_t m = ms[i];
      CHECK(m >= 0 && m < nE, "copy %lld out of range at point %d", (long long)m, c);
      if (m < 0 || m >= nE) continue;
      CHECK(lat[m] == c, "copy %lld of point %d belongs to point %lld (dim %d p %d)",
            (long long)m, c, (long long)lat[m], dim, p);
      seen[m]++;
      if (w.sorted && i > 0)
        CHECK(ms[i - 1] < m, "copies of point %d not ascending (dim %d p %d)", c, dim, p);
    }
  }
  for (int64_t m = 0; m < nE; m++)
    CHECK(seen[m] == 1, "node %lld visited %d times (dim %d p %d)", (long long)m, seen[m],
          dim, p);
}

int main() {
  check_fastdiv();
  int shapes = 0;
  for (int dim = 2; dim <= 3; dim++)
    for (int p = 1; p <= 8; p++)
      for (int pm = 0; pm < (1 << dim); pm++) {
        const int per[3] = {pm & 1, (pm >> 1) & 1, (pm >> 2) & 1};
        const int ne_a[3] = {3, 2, 4}, ne_b[3] = {1, 3, 2}, ne_c[3] = {2, 1, 1};
        check_walk(dim, ne_a, per, p);
        check_walk(dim, ne_b, per, p);
        check_walk(dim, ne_c, per, p);
        shapes += 3;
      }
  const int wide[3] = {70, 2, 1}, none[3] = {0, 1, 0};
  check_walk(3, wide, none, 5);  // rows longer than a block: 351 points
  shapes++;
  if (fails) {
    std::printf("%d failures\n", fails);
    return 1;
  }
  std::printf("lattice walk ok: %d shapes\n", shapes);
  return 0;
}

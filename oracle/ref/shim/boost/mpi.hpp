// Test infrastructure: a single-rank stand-in for the Boost.MPI subset the
// reference's GGFX (src/cdg/comm/ggfx.hpp) and tbox use, so that the
// reference's own gather-scatter, solver and stepper sources compile into
// oracle/_ref without MPI.  One rank: rank() = 0, size() = 1; point-to-point
// requests are complete when made (GGFX on one rank sends to nobody).
#ifndef GFREF_SHIM_BOOST_MPI_HPP
#define GFREF_SHIM_BOOST_MPI_HPP
#include <cstdlib>
#include <vector>

namespace boost {
namespace mpi {

class environment {
 public:
  environment() {}
  environment(int &, char **&, bool = true) {}
};

class request {
 public:
  void wait() {}
  bool test() { return true; }
};

class communicator {
 public:
  int rank() const { return 0; }
  int size() const { return 1; }
  void barrier() const {}
  // No peer exists on one rank; a message to or from one is a caller bug.
  template <typename T>
  request isend(int dest, int, const T &) const {
    if (dest != 0) std::abort();
    return request();
  }
  template <typename T>
  request irecv(int src, int, T &) const {
    if (src != 0) std::abort();
    return request();
  }
  // GGFX::getComm converts the communicator to GC_COMM, an int handle when
  // the reference is built without MPI.
  operator int() const { return 1; }
};

template <typename It>
void wait_all(It, It) {}

template <typename T>
void all_gather(const communicator &, const T &in, std::vector<T> &out) {
  out.assign(1, in);
}

}  // namespace mpi
}  // namespace boost
#endif

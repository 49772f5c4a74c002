/* TEST INFRASTRUCTURE ONLY: single-rank stand-in for Boost.MPI, enough to
 * compile the reference with HAVE_MPI for one process.  Point-to-point calls
 * exist only so mpiBC.hxx compiles; with one rank parallelCom::internal()
 * never selects an mpiBC, so they are never reached. */
#ifndef ORC_SHIM_BOOST_MPI_HPP
#define ORC_SHIM_BOOST_MPI_HPP
#include <algorithm>
#include <cstring>
#include <cmath>
#include <iostream>
#include <sstream>
#include <array>
#include <map>
#include <string>
#include <vector>
#include <cstdlib>
#include "mpi.h"

namespace boost {
namespace serialization { class access {}; }
namespace mpi {
enum comm_create_kind { comm_duplicate, comm_take_ownership, comm_attach };
class request {
public:
    void wait() {}
};
class environment {
public:
    environment() {}
    environment(int &, char **&) {}
};
class communicator {
public:
    communicator() {}
    communicator(MPI_Comm, comm_create_kind) {}
    int rank() const { return 0; }
    int size() const { return 1; }
    operator MPI_Comm() const { return 0; }
    template <class T> request isend(int, int, const T *, int) const { std::abort(); }
    template <class T> request irecv(int, int, T *, int) const { std::abort(); }
};
template <class It> void wait_all(It, It) {}
template <class T, class Op> void reduce(const communicator &, const T &in, T &out, Op, int) { out = in; }
template <class T, class Op> void reduce(const communicator &, const T *in, int n, T *out, Op, int)
{
    std::copy(in, in + n, out);
}
template <class T, class Op> void all_reduce(const communicator &, const T &in, T &out, Op) { out = in; }
template <class T, class Op> void all_reduce(const communicator &, const T *in, int n, T *out, Op)
{
    std::copy(in, in + n, out);
}
template <class T> void broadcast(const communicator &, T &, int) {}
} // namespace mpi
} // namespace boost
#define BOOST_IS_MPI_DATATYPE(T)
#endif

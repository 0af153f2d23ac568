// Test stand-in for green::utils::shared_object (node-shared arrays: object(), fence()) and the
// MPI context (context().node_rank), single process.  Test infrastructure only.
#pragma once
#include <utility>

namespace green::utils {

struct mpi_context {
  int node_rank = 0;
  static mpi_context& context() {
    static mpi_context c;
    return c;
  }
};
inline mpi_context& context() { return mpi_context::context(); }

template <typename T>
class shared_object {
 public:
  explicit shared_object(T obj) : obj_(std::move(obj)) {}
  T& object() { return obj_; }
  const T& object() const { return obj_; }
  void fence() {}

 private:
  T obj_;
};

}  // namespace green::utils

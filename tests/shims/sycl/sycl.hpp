// Declarations of the SYCL names the reference's include/core headers use, for
// a syntax-only compile of the adapters in practice_b200/adapters/ against
// them (tests/test_visitor_dropin.py).  Nothing here is defined or linked.
#pragma once
#include <cstddef>
#include <cstdint>

namespace sycl {
struct event {
  void wait() {}
};
class queue {
 public:
  event memset(void*, int, std::size_t);
  event memcpy(void*, const void*, std::size_t);
  event fill(void*, int, std::size_t);
  template <typename T>
  event copy(const T*, T*, std::size_t);
  void wait();
};
template <typename T>
T* malloc_device(std::size_t, const queue&);
void free(void*, const queue&);
}  // namespace sycl

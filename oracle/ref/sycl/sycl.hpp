// Minimal host stand-in for the two SYCL facilities the reference's crystal
// primitives use (include/crystal/join.h, include/core/inline_math.h):
// sycl::atomic_ref with relaxed ordering, and the enum tags it is spelled with.
// Test infrastructure for oracle/_ref only.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>

namespace sycl {
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, generic_space };
}

template <typename T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::generic_space>
class atomic_ref {
 public:
  explicit atomic_ref(T& t) : ref_(t) {}
  bool compare_exchange_strong(T& expected, T desired) const {
    return ref_.compare_exchange_strong(expected, desired, std::memory_order_relaxed);
  }
  bool compare_exchange_weak(T& expected, T desired) const {
    return ref_.compare_exchange_weak(expected, desired, std::memory_order_relaxed);
  }
  T fetch_add(T v) const { return ref_.fetch_add(v, std::memory_order_relaxed); }
  T fetch_or(T v) const { return ref_.fetch_or(v, std::memory_order_relaxed); }
  T load() const { return ref_.load(std::memory_order_relaxed); }

 private:
  std::atomic_ref<T> ref_;
};
}  // namespace sycl

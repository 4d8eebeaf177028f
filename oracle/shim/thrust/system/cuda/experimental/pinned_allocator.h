// Stand-in for the pinned_allocator header that CCCL 2.x removed; the
// reference's Buffer<T> (src/utils/buffer.h) only names the type (test
// infrastructure for compiling the reference into oracle/_ref).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>

namespace thrust {
namespace cuda {
namespace experimental {
template <typename T>
struct pinned_allocator {
  using value_type = T;
  pinned_allocator() = default;
  template <class U>
  pinned_allocator(const pinned_allocator<U> &) {}
  template <class U>
  struct rebind {
    using other = pinned_allocator<U>;
  };
  T *allocate(std::size_t n) {
    void *p = nullptr;
    if (cudaMallocHost(&p, n * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
    return static_cast<T *>(p);
  }
  void deallocate(T *p, std::size_t) { cudaFreeHost(p); }
  bool operator==(const pinned_allocator &) const { return true; }
  bool operator!=(const pinned_allocator &) const { return false; }
};
}  // namespace experimental
}  // namespace cuda
}  // namespace thrust

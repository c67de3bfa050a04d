// The one Boost.Align name the reference's dtl/adept.hpp names
// (boost::alignment::aligned_allocator<T, A>), for building the adapter where
// Boost is not installed.  It is on the include path after every other
// directory (-idirafter), so an installed Boost takes precedence.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <new>
namespace boost {
namespace alignment {
template <class T, std::size_t Align = alignof(T)>
class aligned_allocator {
 public:
  using value_type = T;
  template <class U>
  struct rebind {
    using other = aligned_allocator<U, Align>;
  };
  aligned_allocator() noexcept = default;
  template <class U>
  aligned_allocator(const aligned_allocator<U, Align>&) noexcept {}
  T* allocate(std::size_t n) {
    const std::size_t a = Align < alignof(void*) ? alignof(void*) : Align;
    void* p = nullptr;
    if (posix_memalign(&p, a, n * sizeof(T) ? n * sizeof(T) : a) != 0) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, std::size_t) noexcept { std::free(p); }
  template <class U>
  bool operator==(const aligned_allocator<U, Align>&) const noexcept { return true; }
  template <class U>
  bool operator!=(const aligned_allocator<U, Align>&) const noexcept { return false; }
};
}  // namespace alignment
}  // namespace boost

// Project-written stand-in for the one Boost.Align name the reference headers
// use (adept.hpp: boost::alignment::aligned_allocator<T, A>).  Boost is not in
// this image; this shim is only for compiling the reference as a test oracle.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <new>
namespace boost { namespace alignment {
template <class T, std::size_t Align = alignof(T)>
class aligned_allocator {
 public:
  using value_type = T;
  template <class U> struct rebind { using other = aligned_allocator<U, Align>; };
  aligned_allocator() noexcept = default;
  template <class U> aligned_allocator(const aligned_allocator<U, Align>&) noexcept {}
  T* allocate(std::size_t n) {
    std::size_t a = Align < alignof(void*) ? alignof(void*) : Align;
    void* p = nullptr;
    if (posix_memalign(&p, a, n * sizeof(T) ? n * sizeof(T) : a)) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, std::size_t) noexcept { std::free(p); }
  template <class U> bool operator==(const aligned_allocator<U, Align>&) const noexcept { return true; }
  template <class U> bool operator!=(const aligned_allocator<U, Align>&) const noexcept { return false; }
};
}}

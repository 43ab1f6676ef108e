// An allocator whose resize leaves new elements uninitialised: for large host arrays
// that are filled in parallel right after they are sized, where zero-filling them first
// would be a wasted serial pass over the memory.
#pragma once

#include <memory>
#include <utility>
#include <vector>

namespace fftsvd {

template <typename T>
struct FillLater : std::allocator<T> {
   template <typename U>
   struct rebind {
      using other = FillLater<U>;
   };
   FillLater() = default;
   template <typename U>
   FillLater(const FillLater<U>&) noexcept {}
   template <typename U>
   void construct(U* p) noexcept {
      ::new ((void*)p) U;
   }
   template <typename U, typename... A>
   void construct(U* p, A&&... a) {
      ::new ((void*)p) U(std::forward<A>(a)...);
   }
};

}  // namespace fftsvd

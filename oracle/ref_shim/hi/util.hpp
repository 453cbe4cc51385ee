// Stand-in for <hi/util.hpp>: the functors the reference uses to free its
// scene containers (libhi/hi/util.hpp:9-21 restated).
#pragma once
#include <hi/lang.hpp>
namespace hi {
template <typename T>
struct delete_ptr {
  void operator()(T *p) const { delete p; }
  void operator()(T const *p) const { delete p; }
};
template <typename T>
struct delete_ary {
  void operator()(T *p) const { delete[] p; }
  void operator()(T const *p) const { delete[] p; }
};
}  // namespace hi

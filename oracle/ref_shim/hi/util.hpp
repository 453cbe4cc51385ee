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
// hi::trim (libhi/hi/util/string.hpp:22-34): strips " \t\r\n" at both ends
// (the MQO loader uses it; string.hpp itself pulls in Win32 headers).
inline void trim(std::tstring &s) {
  std::size_t const b = s.find_first_not_of(" \t\r\n");
  if (b == std::tstring::npos) {
    s.clear();
    return;
  }
  s = s.substr(b, s.find_last_not_of(" \t\r\n") - b + 1);
}
}  // namespace hi

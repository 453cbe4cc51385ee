// Stand-in for <hi/math.hpp>: the reference's own scalar maths and 2-/3-vectors.
//  * libhi/hi/math/math.hpp:236,261 call hi::dot / hi::sum from templates defined
//    before the vector headers declare them (MSVC resolves this late, g++ does
//    not), so those two functions are declared first, with the signatures of
//    libhi/hi/math/vector{2,3}.hpp.
//  * libhi/hi/math/vector4.hpp does not build with g++; only the OpenGL preview
//    uses 4-vectors, so a minimal value type stands in for it.
#pragma once
#include <hi/lang.hpp>
#include <hi/math/promote_traits.hpp>
namespace hi {
template <typename T>
class basic_vector2;
template <typename T>
class basic_vector3;
template <typename T, typename S>
inline typename promote_traits<T, S>::type dot(basic_vector2<T> const &a,
                                               basic_vector2<S> const &b);
template <typename T, typename S>
inline typename promote_traits<T, S>::type dot(basic_vector3<T> const &a,
                                               basic_vector3<S> const &b);
template <typename T>
inline T sum(basic_vector2<T> const &a);
template <typename T>
inline T sum(basic_vector3<T> const &a);
}  // namespace hi
#include <hi/math/math.hpp>
#include <hi/math/vector2.hpp>
#include <hi/math/vector3.hpp>
namespace hi {
template <typename T>
class basic_vector4 {
 public:
  typedef T value_type;
  explicit basic_vector4(T a = T()) : v_{a, a, a, a} {}
  basic_vector4(T a, T b, T c, T d) : v_{a, b, c, d} {}
  basic_vector4 &operator=(T a) {  // `dst = 0` of imagefilm_hdr.cpp:20
    v_[0] = v_[1] = v_[2] = v_[3] = a;
    return *this;
  }
  T *data() { return v_; }
  T const *data() const { return v_; }
  T &operator[](std::size_t i) { return v_[i]; }
  T const &operator[](std::size_t i) const { return v_[i]; }

 private:
  T v_[4];
};
}  // namespace hi

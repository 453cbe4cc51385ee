// Stand-in for <hi/image.hpp>: the spectrum and colour-space parts only
// (memory_image.hpp needs GDI and is not on the path-tracing path).
#pragma once
#include <hi/math.hpp>
#include <hi/image/spectrum.hpp>
#include <hi/image/color_space.hpp>
namespace hi {
// renderer/core/config.hpp:91 passes a double XYZ vector to the float
// overload of spd2xyz (MSVC binds a temporary there); this overload lets the
// spectral renderer compile.  Its path tracer does not use the result.
inline void spd2xyz(basic_spectrum const &spd, basic_vector3<double> &xyz) {
  basic_vector3<float> f;
  spd2xyz(spd, f);
  xyz = f;
}
}  // namespace hi

// Stand-in for <hi/image.hpp>: the spectrum and colour-space parts only
// (memory_image.hpp needs GDI and is not on the path-tracing path).
#pragma once
#include <hi/math.hpp>
#include <hi/image/spectrum.hpp>
#include <hi/image/color_space.hpp>

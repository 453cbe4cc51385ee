// Command-line harness around the reference's Radiance writer,
// ImageFilm::SaveAsHdr (xyz/core/imagefilm_hdr.cpp, compiled where it lies by
// oracle/Makefile into the program oracle/_ref/xyzref_hdr).  TEST
// INFRASTRUCTURE: only tests/ run it.  A separate process, because the
// writer's iostreams and locale must not share a process with another C++
// runtime (loaded into Python next to numpy's, it crashes).
//   xyzref_hdr <film.f32> <width> <height> <spp> <out.hdr>
// film.f32: W * H * 3 float32 XYZ sums, row 0 at the bottom.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <core/imagefilm.hpp>

namespace {
// SaveAsHdr is private (ImageFilm::Save picks it by extension, but Save is not
// compiled here: it lives in imagefilm.cpp with the GL-era pieces).  An
// explicit instantiation may name a private member, which hands its pointer out.
struct HdrTag {
  typedef bool (xyz::ImageFilm::*type)(std::tchar_t const *, xyz::float_t) const;
  friend type member(HdrTag);
};
template <typename Tag, typename Tag::type M>
struct Expose {
  friend typename Tag::type member(Tag) { return M; }
};
template struct Expose<HdrTag, &xyz::ImageFilm::SaveAsHdr>;
}  // namespace

int main(int argc, char **argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: xyzref_hdr <film.f32> <width> <height> <spp> <out.hdr>\n");
    return 2;
  }
  int const width = std::atoi(argv[2]), height = std::atoi(argv[3]);
  float const spp = static_cast<float>(std::atof(argv[4]));
  std::vector<float> film(3 * static_cast<std::size_t>(width) * height);
  std::FILE *in = std::fopen(argv[1], "rb");
  if (!in || std::fread(film.data(), sizeof(float), film.size(), in) != film.size()) return 3;
  std::fclose(in);
  xyz::ImageFilm f(static_cast<std::size_t>(width), static_cast<std::size_t>(height));
  for (std::size_t p = 0; p < f.count(); ++p)
    f[p] = xyz::ImageFilm::color_t(film[3 * p], film[3 * p + 1], film[3 * p + 2]);
  return (f.*member(HdrTag()))(argv[5], spp) ? 0 : 1;
}

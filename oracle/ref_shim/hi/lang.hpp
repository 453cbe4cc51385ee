// Compatibility stand-in for the reference's <hi/lang.hpp> (libhi/hi/lang/lang.hpp),
// which pulls in <windows.h>/<tchar.h>.  Test infrastructure only: it lets the
// reference's own path-tracing sources compile with g++ on Linux as an oracle.
#pragma once
#ifndef _USE_MATH_DEFINES
#define _USE_MATH_DEFINES
#endif
#include <cassert>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <algorithm>
#include <atomic>
#include <thread>
#include <unordered_map>
#include <mutex>
#include <array>
#include <deque>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <stack>
#include <string>
#include <vector>

// MSVC SAL annotations and keywords used throughout the reference.  Every
// standard header the oracle needs is included above: libstdc++ uses `__out`
// and `__in` as parameter names, which these empty macros would break.
#define __in
#define __out
#define __inout
#define sealed
#ifndef INOUT
#define INOUT
#endif
#define UNREFERENCED_PARAMETER(p) ((void)(p))
#ifndef MAX_PATH
#define MAX_PATH 260
#endif
// TCHAR mapping to narrow characters.
#define _TEXT(x) x
#define _T(x) x
#define _ftprintf_s fprintf
#define _stprintf_s snprintf
#define _tcscpy_s(d, n, s) std::strncpy((d), (s), (n))
// MSVC CRT's _finite (xyz/core/imagefilm_hdr.cpp:165)
inline int _finite(double x) { return std::isfinite(x) ? 1 : 0; }

#define HI_TO_STRING(x) #x
#define HI_ARRAYS_LENGTH(ary) (sizeof(ary) / sizeof(ary[0]))
#define HI_RANGE_CHECK(a, i)
#define HI_DISALLOW_COPY_AND_ASSIGN(TypeName) \
 private:                                     \
  TypeName(TypeName const &);                 \
  TypeName &operator=(TypeName const &)

namespace hi {
typedef std::uint16_t word;
typedef std::uint32_t dword;
typedef std::uint64_t qword;
typedef std::uint8_t ubyte;
typedef std::uint16_t ushort;
typedef std::uint32_t uint;
typedef std::uint64_t ulong;
typedef std::int8_t sbyte;
typedef std::int16_t sshort;
typedef std::int32_t sint;
typedef std::int64_t slong;
}  // namespace hi

namespace std {
typedef char tchar_t;
typedef std::string tstring;
typedef std::istream tistream;
typedef std::ostream tostream;
typedef std::ifstream tifstream;
typedef std::ofstream tofstream;
typedef std::stringstream tstringstream;
typedef std::istringstream tistringstream;
typedef std::ostringstream tostringstream;
static std::ostream &tcerr = std::cerr;
static std::ostream &tcout = std::cout;
}  // namespace std

// <hi/util/mt19937.hpp> is included by the reference but absent from its tree.
// The sources call `std::mt19937_64::next<T>()`, a uniform draw in [0,1).
// Only off-path estimators (photon maps, importance) use it; the oracle's
// path tracer draws its numbers through IPrimarySample instead.
namespace std {
struct xyzref_mt19937_64 : public std::mersenne_twister_engine<
                               std::uint_fast64_t, 64, 312, 156, 31,
                               0xb5026f5aa96619e9ULL, 29, 0x5555555555555555ULL,
                               17, 0x71d67fffeda60000ULL, 37,
                               0xfff7eee000000000ULL, 43, 6364136223846793005ULL> {
  using std::mersenne_twister_engine<std::uint_fast64_t, 64, 312, 156, 31, 0xb5026f5aa96619e9ULL,
                                     29, 0x5555555555555555ULL, 17, 0x71d67fffeda60000ULL, 37,
                                     0xfff7eee000000000ULL, 43,
                                     6364136223846793005ULL>::mersenne_twister_engine;
  template <typename T>
  T next() {
    return T((*this)() >> 11) * T(1.0 / 9007199254740992.0);
  }
};
}  // namespace std
#define mt19937_64 xyzref_mt19937_64

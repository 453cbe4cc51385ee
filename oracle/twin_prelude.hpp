// Force-included ahead of every source of the reference's spectral renderer
// (renderer/, namespace tgir) that the oracle compiles.  Test infrastructure.
//  * renderer/stdafx.hpp is that project's precompiled header.
//  * renderer/bsdf/Bsdf.cpp:8 defines a std::mt19937 overload that its header
//    declares with std::mt19937_64 (MSVC accepted the mismatch); the two names
//    are made one.
//  * The depth cap and Russian-roulette threshold macros
//    (renderer/core/config.hpp:34 and its CONFIG_TERMINATE_THRESHOLD) are
//    re-pointed at run-time variables.
//  * renderer/geom/Path.hpp names `enum EMutationType` before it is declared;
//    Path.hpp is pre-included with that name mapped to a forward-declared enum.
#pragma once
#include <cstddef>
extern std::size_t xyztwin_kmax;
extern double xyztwin_rr_threshold;
#include <stdafx.hpp>
#define mt19937 mt19937_64
#include <core/config.hpp>
#undef TGIR_CONFIG_kMaxRandomWalkDepth
#define TGIR_CONFIG_kMaxRandomWalkDepth (::xyztwin_kmax)
#undef CONFIG_TERMINATE_THRESHOLD
#define CONFIG_TERMINATE_THRESHOLD (::xyztwin_rr_threshold)
namespace tgir {
enum EMutationTypeForwarded : int;
}
#define EMutationType EMutationTypeForwarded
#include <geom/Path.hpp>
#undef EMutationType

// Force-included (g++ -include) ahead of every reference source the oracle
// compiles.  Test infrastructure only.
//  * xyz/stdafx.hpp is the reference's precompiled header (MSVC /FI).
//  * The depth cap and the Russian-roulette threshold are compile-time macros in
//    xyz/core/config.hpp:30,60; they are re-pointed at run-time variables so one
//    build serves every configuration (same meaning, same comparisons).
//  * xyz/geom/path.hpp:23 names `enum EMutationType` before xyz/core/scene.hpp:30
//    declares it (accepted by MSVC, rejected by g++); path.hpp is pre-included
//    here with that name mapped to a forward-declared enum.  Path is not used by
//    the path tracer.
#pragma once
#include <cstddef>
extern std::size_t xyzref_kmax;
extern float xyzref_rr_threshold;
#include <stdafx.hpp>
#include <core/config.hpp>
#undef XYZ_CONFIG_kMaxRandomWalkDepth
#define XYZ_CONFIG_kMaxRandomWalkDepth (::xyzref_kmax)
#undef CONFIG_TERMINATE_THRESHOLD
#define CONFIG_TERMINATE_THRESHOLD (::xyzref_rr_threshold)
namespace xyz {
enum EMutationTypeForwarded : int;
}
#define EMutationType EMutationTypeForwarded
#include <geom/path.hpp>
#undef EMutationType

// <hi/sds.hpp>: the reference's array kd-tree (photon maps, off the path-tracing
// path).  Its .inl lacks one `typename` that g++ requires, so the oracle recipe
// builds from a copy with that single token added (see oracle/Makefile).
#pragma once
#include <hi/lang.hpp>
#include "patched/hi/sds/array_kdtree.hpp"

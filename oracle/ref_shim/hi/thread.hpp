// Stand-in for <hi/thread.hpp> (Win32 thread wrappers).  The oracle drives the
// reference's estimator from its own harness threads, so nothing is needed here.
#pragma once
#include <hi/lang.hpp>

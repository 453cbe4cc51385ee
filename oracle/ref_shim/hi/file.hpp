// Stand-in for <hi/file.hpp> (Win32 directory helpers, unused by the path tracer).
#pragma once
#include <hi/lang.hpp>

/* Stand-in for the Win32 <tchar.h> that ply2mqo's stdafx.hpp includes: the
 * tool uses no TCHAR names.  Test infrastructure only. */
#pragma once

/* Empty stand-in for MSVC's <crtdbg.h>; the reference only includes it (std_incl.h:4). Test infrastructure only. */
#pragma once

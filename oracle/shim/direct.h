/* Stand-in for MSVC's <direct.h> (_mkdir). Test infrastructure only. */
#pragma once
#include <sys/stat.h>
static inline int _mkdir(const char *p) { return mkdir(p, 0755); }

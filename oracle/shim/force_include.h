/*
 * Forced include (-include) for compiling the reference CPU tracker with g++ on Linux.
 * MSVC pulls these in transitively; g++ needs them explicitly. `using std::fabs` lets
 * std::max(0.0f, fabs(float)) at cpu_tracker.cpp:714 resolve to the float overload, as
 * MSVC does. Test infrastructure only.
 */
#pragma once
#include <cstring>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <list>
using std::fabs;

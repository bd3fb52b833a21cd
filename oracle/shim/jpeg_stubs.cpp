/*
 * The reference's JPEG helpers (fastjpg.cpp) need libjpeg, which it does not vendor.
 * The oracle never writes or reads JPEGs, so these stand-ins satisfy the linker.
 * Test infrastructure only.
 */
#include "std_incl.h"
#include "utils.h"
void FloatToJPEGFile(const char *, const float *, int, int) {}
void WriteJPEGFile(uchar *, int, int, const char *, int) {}
int ReadJPEGFile(uchar *, int, uchar **, int *, int *) { throw std::runtime_error("JPEG support is not built into the oracle"); }

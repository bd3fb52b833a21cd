/*
 * A stand-in for the two LabVIEW run-time functions the LabVIEW binding calls
 * (NumericArrayResize, MoveBlock), for the tests: handles are a malloc'd master pointer to a
 * block {int32 dims[N]; (padding to the element alignment); elements}, as LabVIEW lays out
 * numeric arrays. fake_lv_new / fake_lv_free let the tests create and release handles.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int32_t MgErr;
typedef void **UHandle;

static size_t elem_size(int32_t code)
{
    switch (code) {
    case 1: case 5: return 1;             /* int8, uint8 */
    case 2: case 6: return 2;             /* int16, uint16 */
    case 3: case 7: case 9: return 4;     /* int32, uint32, float */
    case 4: case 8: case 10: case 0xc: return 8; /* int64, uint64, double, complex float */
    case 0xd: return 16;                  /* complex double */
    default: return 0;
    }
}

static size_t elem_align(int32_t code)
{
    size_t s = elem_size(code);
    if (code == 0xc) return 4;
    if (code == 0xd) return 8;
    return s > 8 ? 8 : s;
}

MgErr NumericArrayResize(int32_t code, int32_t ndims, UHandle *hp, size_t n)
{
    size_t es = elem_size(code), al = elem_align(code);
    if (!es || ndims < 1 || !hp) return 1;
    size_t hdr = 4 * (size_t)ndims;
    hdr = (hdr + al - 1) / al * al;
    size_t bytes = hdr + (n ? n : 1) * es;
    if (!*hp) {
        *hp = (UHandle)malloc(sizeof(void *));
        if (!*hp) return 2;
        **hp = calloc(1, bytes);
        return **hp ? 0 : 2;
    }
    void *p = realloc(**hp, bytes);
    if (!p) return 2;
    **hp = p;
    return 0;
}

MgErr MoveBlock(const void *src, void *dst, size_t n)
{
    memmove(dst, src, n);
    return 0;
}

UHandle fake_lv_new(int32_t code, int32_t ndims, const int32_t *dims)
{
    UHandle h = NULL;
    size_t n = 1;
    for (int i = 0; i < ndims; i++) n *= (size_t)dims[i];
    if (NumericArrayResize(code, ndims, &h, n)) return NULL;
    memcpy(*h, dims, 4 * (size_t)ndims);
    return h;
}

void fake_lv_free(UHandle h)
{
    if (!h) return;
    free(*h);
    free(h);
}

/* Test infrastructure, not product code.
 *
 * The one translation unit that compiles the reference codec (yhbsh/fdv,
 * include/fdv.h) from its own header, so the oracle build can link it into a
 * shared library and the tests can call its public entry points
 * (fdv_video_encode, fdv_vtile_encode, fdv_video_decode, fdv_vtile_decode and
 * the per-kernel functions of sections 6-9) through ctypes.  Nothing of the
 * reference is copied here: the header is read from the reference tree at
 * build time by oracle/build.py. */
#define FDV_IMPLEMENTATION
#include "fdv.h"

/* The reference keeps its 8x8 tables private (fdv.h:2585-2612).  This accessor
 * exposes them so the oracle tests can confirm that the tables the product
 * computes on the host are the same integers. */
void fdvref_c8_tables(int32_t c8_out[64], int32_t qstep_out[52]) {
    int16_t x[64] = {0};
    int32_t y[64];
    fdv_fdct8x8(x, y);              /* forces the one-time table build */
    for (int u = 0; u < 8; ++u)
        for (int v = 0; v < 8; ++v) c8_out[u * 8 + v] = C8[u][v];
    for (int q = 0; q < 52; ++q) qstep_out[q] = QSTEP8[q];
}

// Host-computed constants of the analysis loop.
#include <cmath>

#include "fdvb_internal.h"

// fdv.h:5804 and :4870.  Evaluated left to right in double precision with the
// host libm, exactly as the reference's expression, and handed to the device
// as a double so every RD comparison on the GPU uses the identical lambda.
double fdvb_lambda(int qp, double lscale) {
    return lscale * 0.425 * pow(2.0, (qp - 12) / 3.0);
}

// fdv.h:2597-2612: the fixed-point 8x8 DCT-II basis (x512, AC rows forced to
// sum to zero) and the per-QP quantiser step (x262144).  The reference builds
// these with libm cos/pow/lround; they are built here the same way on the host
// and uploaded, never recomputed on the device.
void fdvb_c8_tables(int32_t c8[64], int32_t qstep8[52]) {
    const double pi = 3.14159265358979323846;
    int32_t m[8][8];
    for (int u = 0; u < 8; ++u) {
        double a = (u == 0) ? sqrt(1.0 / 8.0) : sqrt(2.0 / 8.0);
        for (int x = 0; x < 8; ++x)
            m[u][x] = (int32_t)lround(a * cos((2 * x + 1) * u * pi / 16.0) * 512.0);
    }
    for (int u = 1; u < 8; ++u) {
        int s = 0;
        for (int x = 0; x < 8; ++x) s += m[u][x];
        m[u][0] -= s;
    }
    for (int u = 0; u < 8; ++u)
        for (int x = 0; x < 8; ++x) c8[u * 8 + x] = m[u][x];
    for (int qp = 0; qp < 52; ++qp) qstep8[qp] = (int32_t)lround(262144.0 * (0.625 * pow(2.0, qp / 6.0)));
}

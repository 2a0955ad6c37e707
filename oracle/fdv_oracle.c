/* ORACLE -- test infrastructure, not product code.
 *
 * A CPU restatement, in plain C, of the reference encoder's analysis loop
 * (yhbsh/fdv, include/fdv.h): motion search, motion compensation, the 4x4 and
 * 8x8 transforms with quantisation and RDOQ, the P-frame mode decision, the
 * key-frame intra quadtree, reconstruction and deblocking.  It emits the
 * symbol streams in the exact order and partition the reference's entropy
 * tail consumes (9 structure streams + 7 coefficient streams per P-frame, 12
 * streams per intra plane), plus the reconstruction, so the tests can check
 * the GPU analysis against it stream by stream and macroblock by macroblock.
 *
 * It is pinned against the reference itself: the tests compose these streams
 * with the host entropy tail and require the resulting .fdv bytes to equal the
 * reference encoder's output (oracle/_ref, built from the reference sources),
 * and they check the per-kernel functions below against the reference's
 * exported kernels on seeded inputs.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library.  Every function cites the reference lines it restates.
 *
 * Reads beyond a plane's edge are evaluated by clamping the coordinate.  The
 * reference instead reads a border of replicated edge samples (fdv.h:1603-1624)
 * that its static assert (fdv.h:5178) proves is never overrun, so the two are
 * the same function of the picture. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Stream indices (fdv.h:4170, :4273-4289). */
enum { PS_REF_ = 4, PS_MVX_ = 5, PS_MVY_ = 6, PS_SUB_ = 7, PS_MERGE_ = 8 };
enum { IS_SPLIT0_ = 0, IS_MODEB_ = 4, IS_MODE0_ = 5, IS_MODE1_ = 6 };

/* ----------------------------------------------------------- op count -- */
/* With -DORACLE_OPCOUNT (a separate build, oracle/opcount.py) every primitive
 * adds its integer-op cost to a category: the algorithmic op count of a frame
 * for the integer-pipe roofline.  Costs per call (byte-lane ops count once
 * per lane): SAD 2 per pixel (absolute difference, accumulate); luma MC per
 * sample by phase (copy 1, a half-pel 6-tap sample 12, the centre j 66, a
 * quarter-pel mean 2 plus its sources); chroma MC 10 per sample; 4x4
 * transform 64 each way; 4x4 quantisation 64, dequantisation 32; an RDOQ
 * truncation trial 48 (plus its dequantisation and inverse transform); 8x8
 * transform 2048 each way (two 8x8x8 multiply-accumulate passes); 8x8
 * quantisation 256, dequantisation 128; 4x4 SATD 112; intra prediction 3 per
 * sample; residual, reconstruction and SSD 5 per pixel; a deblocking edge
 * sample 20.  The normal build compiles all of it away. */
#ifdef ORACLE_OPCOUNT
enum { OPC_SAD, OPC_MC, OPC_SATD, OPC_TR4, OPC_Q4, OPC_RDOQ, OPC_TR8, OPC_Q8, OPC_PIX, OPC_INTRA, OPC_DBK, OPC_N };
static unsigned long long g_opc[OPC_N];
#define OPC(k, n) (g_opc[k] += (unsigned long long)(n))
int oracle_opcount(unsigned long long *out, int reset) {
    for (int k = 0; k < OPC_N; ++k) {
        if (out) out[k] = g_opc[k];
        if (reset) g_opc[k] = 0;
    }
    return OPC_N;
}
#else
#define OPC(k, n) ((void)0)
#endif

/* ------------------------------------------------------------ helpers -- */
static int clipb(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
static int iabs(int v) { return v < 0 ? -v : v; }

/* Growable byte array. */
typedef struct { uint8_t *b; size_t n, cap; } buf_t;
static void bput(buf_t *x, uint8_t v) {
    if (x->n == x->cap) { x->cap = x->cap ? x->cap * 2 : 256; x->b = realloc(x->b, x->cap); }
    x->b[x->n++] = v;
}
static void bcat(buf_t *x, const buf_t *y) { for (size_t i = 0; i < y->n; ++i) bput(x, y->b[i]); }
static void bfree(buf_t *x) { free(x->b); x->b = NULL; x->n = x->cap = 0; }

static const int ZZ4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15}; /* fdv.h:1699 */
static const int ZZ8[64] = {                                                      /* fdv.h:2153 */
     0,  1,  8, 16,  9,  2,  3, 10, 17, 24, 32, 25, 18, 11,  4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13,  6,  7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
static uint32_t zz_enc(int v) { return ((uint32_t)v << 1) ^ (uint32_t)(v >> 31); } /* fdv.h:1701 */
static int leb_size(uint32_t u) { int n = 1; while (u >= 0x80) { u >>= 7; ++n; } return n; } /* :1709 */
static void leb_put(buf_t *x, uint32_t u) {                                     /* fdv.h:1704 */
    while (u >= 0x80) { bput(x, (uint8_t)(u | 0x80)); u >>= 7; }
    bput(x, (uint8_t)u);
}
static int bits_val(uint32_t v) {                                               /* fdv.h:2487 */
    int n = 0;
    for (uint32_t x = v + 1; x > 1; x >>= 1) ++n;
    return 2 * n + 1;
}

/* --------------------------------------------------------- transforms -- */
/* fdv.h:2233-2292 */
static void fwd_1d(const int *in, int *out) {
    int a0 = in[0] + in[3], a3 = in[0] - in[3], a1 = in[1] + in[2], a2 = in[1] - in[2];
    out[0] = a0 + a1; out[1] = a3 * 2 + a2; out[2] = a0 - a1; out[3] = a3 - a2 * 2;
}
static void inv_1d(const int *in, int *out) {
    int z0 = in[0] + in[2], z1 = in[0] - in[2];
    int z2 = (in[1] >> 1) - in[3], z3 = in[1] + (in[3] >> 1);
    out[0] = z0 + z3; out[1] = z1 + z2; out[2] = z1 - z2; out[3] = z0 - z3;
}
void oracle_fdct4x4(const int16_t r[16], int32_t c[16]) {
    OPC(OPC_TR4, 64);
    int t[16], a[4], b[4];
    for (int i = 0; i < 4; ++i) { for (int j = 0; j < 4; ++j) a[j] = r[i * 4 + j]; fwd_1d(a, b); for (int j = 0; j < 4; ++j) t[i * 4 + j] = b[j]; }
    for (int j = 0; j < 4; ++j) { for (int i = 0; i < 4; ++i) a[i] = t[i * 4 + j]; fwd_1d(a, b); for (int i = 0; i < 4; ++i) c[i * 4 + j] = b[i]; }
}
void oracle_idct4x4(const int32_t d[16], int16_t r[16]) {
    OPC(OPC_TR4, 64);
    int t[16], a[4], b[4];
    for (int i = 0; i < 4; ++i) { for (int j = 0; j < 4; ++j) a[j] = d[i * 4 + j]; inv_1d(a, b); for (int j = 0; j < 4; ++j) t[i * 4 + j] = b[j]; }
    for (int j = 0; j < 4; ++j) { for (int i = 0; i < 4; ++i) a[i] = t[i * 4 + j]; inv_1d(a, b); for (int i = 0; i < 4; ++i) r[i * 4 + j] = (int16_t)((b[i] + 32) >> 6); }
}
/* fdv.h:2405-2428 */
static const int MF[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                             {9362, 3647, 5825}, {8192, 3355, 5243}, {7282, 2893, 4559}};
static const int DQV[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16},
                              {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
static int pos_class(int idx) {
    int i = idx >> 2, j = idx & 3;
    if (!(i & 1) && !(j & 1)) return 0;
    if ((i & 1) && (j & 1)) return 1;
    return 2;
}
void oracle_quant4x4(const int32_t c[16], int16_t l[16], int qp) {              /* fdv.h:2430 */
    OPC(OPC_Q4, 64);
    int m = qp % 6, qbits = 15 + qp / 6, f = (1 << qbits) / 3;
    for (int i = 0; i < 16; ++i) {
        int w = c[i], sign = w < 0 ? -1 : 1;
        long aw = (long)(w < 0 ? -w : w);
        l[i] = (int16_t)(sign * (int)((aw * MF[m][pos_class(i)] + f) >> qbits));
    }
}
void oracle_dequant4x4(const int16_t l[16], int32_t d[16], int qp) {            /* fdv.h:2546 */
    OPC(OPC_Q4, 32);
    int m = qp % 6, sh = qp / 6;
    for (int i = 0; i < 16; ++i) d[i] = (int32_t)(l[i] * DQV[m][pos_class(i)]) * (int32_t)(1 << sh);
}
void oracle_rdoq4x4(int16_t level[16], const int16_t res[16], int qp, double lambda) { /* fdv.h:2493 */
    int last = -1;
    for (int k = 0; k < 16; ++k) if (level[ZZ4[k]] != 0) last = k;
    if (last < 0) return;
    int16_t trial[16];
    memcpy(trial, level, sizeof trial);
    int bits = bits_val((uint32_t)(last + 1));
    for (int k = 0; k <= last; ++k) bits += bits_val(zz_enc(level[ZZ4[k]]));
    double bestJ = -1.0;
    int bestL = last;
    for (int L = last; L >= -1; --L) {
        if (L < 0 || level[ZZ4[L]] != 0) {
            int32_t dc[16]; int16_t rr[16];
            oracle_dequant4x4(trial, dc, qp);
            oracle_idct4x4(dc, rr);
            int64_t D = 0;
            OPC(OPC_RDOQ, 48);
            for (int i = 0; i < 16; ++i) { int d = res[i] - rr[i]; D += (int64_t)d * d; }
            double J = (double)D + lambda * bits;
            if (bestJ < 0.0 || J < bestJ) { bestJ = J; bestL = L; }
        }
        if (L >= 0) { bits -= 8 * leb_size(zz_enc(level[ZZ4[L]])); trial[ZZ4[L]] = 0; }
    }
    for (int k = bestL + 1; k < 16; ++k) level[ZZ4[k]] = 0;
}
/* fdv.h:2585-2685 -- tables from the same libm calls. */
static int32_t C8[8][8], QSTEP8[52];
static int c8_ready = 0;
static void c8_init(void) {
    if (c8_ready) return;
    for (int u = 0; u < 8; ++u) {
        double a = (u == 0) ? sqrt(1.0 / 8.0) : sqrt(2.0 / 8.0);
        for (int x = 0; x < 8; ++x)
            C8[u][x] = (int32_t)lround(a * cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0) * 512.0);
    }
    for (int u = 1; u < 8; ++u) { int s = 0; for (int x = 0; x < 8; ++x) s += C8[u][x]; C8[u][0] -= s; }
    for (int qp = 0; qp < 52; ++qp) QSTEP8[qp] = (int32_t)lround(262144.0 * (0.625 * pow(2.0, qp / 6.0)));
    c8_ready = 1;
}
void oracle_c8_tables(int32_t c8[64], int32_t q[52]) {
    c8_init();
    for (int i = 0; i < 64; ++i) c8[i] = C8[i / 8][i % 8];
    for (int i = 0; i < 52; ++i) q[i] = QSTEP8[i];
}
void oracle_fdct8x8(const int16_t X[64], int32_t Y[64]) {
    OPC(OPC_TR8, 2048);
    c8_init();
    int32_t A[64];
    for (int u = 0; u < 8; ++u) for (int x = 0; x < 8; ++x) { int32_t s = 0; for (int y = 0; y < 8; ++y) s += C8[u][y] * (int32_t)X[y * 8 + x]; A[u * 8 + x] = s; }
    for (int u = 0; u < 8; ++u) for (int v = 0; v < 8; ++v) { int32_t s = 0; for (int x = 0; x < 8; ++x) s += A[u * 8 + x] * C8[v][x]; Y[u * 8 + v] = s; }
}
void oracle_idct8x8(const int32_t Y[64], int16_t X[64]) {
    OPC(OPC_TR8, 2048);
    c8_init();
    int64_t B[64];
    for (int y = 0; y < 8; ++y) for (int v = 0; v < 8; ++v) { int64_t s = 0; for (int u = 0; u < 8; ++u) s += (int64_t)C8[u][y] * Y[u * 8 + v]; B[y * 8 + v] = s; }
    for (int y = 0; y < 8; ++y) for (int x = 0; x < 8; ++x) { int64_t s = 0; for (int v = 0; v < 8; ++v) s += B[y * 8 + v] * C8[v][x]; X[y * 8 + x] = (int16_t)((s + ((int64_t)1 << 35)) >> 36); }
}
void oracle_quant8x8(const int32_t Y[64], int16_t l[64], int qp) {
    OPC(OPC_Q8, 256);
    c8_init();
    int32_t q = QSTEP8[qp], f = q / 3;
    for (int i = 0; i < 64; ++i) { int32_t c = Y[i]; int sign = c < 0 ? -1 : 1; int32_t a = c < 0 ? -c : c; l[i] = (int16_t)(sign * ((a + f) / q)); }
}
void oracle_dequant8x8(const int16_t l[64], int32_t Y[64], int qp) {
    OPC(OPC_Q8, 128);
    c8_init();
    int32_t q = QSTEP8[qp];
    for (int i = 0; i < 64; ++i) { int64_t v = (int64_t)l[i] * q; Y[i] = v < INT32_MIN ? INT32_MIN : (v > INT32_MAX ? INT32_MAX : (int32_t)v); }
}
int oracle_satd4x4(const uint8_t *src, int ss, const uint8_t *pred) {         /* fdv.h:3803 */
    OPC(OPC_SATD, 112);
    int d[16];
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) d[i * 4 + j] = src[i * ss + j] - pred[i * 4 + j];
    for (int i = 0; i < 4; ++i) {
        int a0 = d[i*4+0] + d[i*4+1], a1 = d[i*4+0] - d[i*4+1], a2 = d[i*4+2] + d[i*4+3], a3 = d[i*4+2] - d[i*4+3];
        d[i*4+0] = a0 + a2; d[i*4+1] = a1 + a3; d[i*4+2] = a0 - a2; d[i*4+3] = a1 - a3;
    }
    int sum = 0;
    for (int j = 0; j < 4; ++j) {
        int a0 = d[j] + d[4+j], a1 = d[j] - d[4+j], a2 = d[8+j] + d[12+j], a3 = d[8+j] - d[12+j];
        sum += iabs(a0 + a2) + iabs(a1 + a3) + iabs(a0 - a2) + iabs(a1 - a3);
    }
    return sum;
}

/* -------------------------------------------------------------- intra -- */
void oracle_intra4x4(int mode, const uint8_t top[8], const uint8_t left[4], uint8_t tl,
                     int ht, int hl, uint8_t pred[16]) {                        /* fdv.h:2698 */
    OPC(OPC_INTRA, 48);
    int Tn[9], Ln[5];
    Tn[0] = tl; for (int i = 0; i < 8; ++i) Tn[i + 1] = top[i];
    Ln[0] = tl; for (int i = 0; i < 4; ++i) Ln[i + 1] = left[i];
#define T(i) Tn[(i) + 1]
#define L(i) Ln[(i) + 1]
    for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x) {
            int v;
            switch (mode) {
            case 1: v = T(x); break;
            case 2: v = L(y); break;
            case 3: v = (x == 3 && y == 3) ? (T(6) + 3 * T(7) + 2) >> 2 : (T(x + y) + 2 * T(x + y + 1) + T(x + y + 2) + 2) >> 2; break;
            case 4: if (x > y) v = (T(x - y - 2) + 2 * T(x - y - 1) + T(x - y) + 2) >> 2;
                    else if (x < y) v = (L(y - x - 2) + 2 * L(y - x - 1) + L(y - x) + 2) >> 2;
                    else v = (T(0) + 2 * T(-1) + L(0) + 2) >> 2; break;
            case 5: { int z = 2 * x - y;
                    if (z >= 0 && !(z & 1)) v = (T(x - (y >> 1) - 1) + T(x - (y >> 1)) + 1) >> 1;
                    else if (z >= 0) v = (T(x - (y >> 1) - 2) + 2 * T(x - (y >> 1) - 1) + T(x - (y >> 1)) + 2) >> 2;
                    else if (z == -1) v = (L(0) + 2 * T(-1) + T(0) + 2) >> 2;
                    else v = (L(y - 1) + 2 * L(y - 2) + L(y - 3) + 2) >> 2; break; }
            case 6: { int z = 2 * y - x;
                    if (z >= 0 && !(z & 1)) v = (L(y - (x >> 1) - 1) + L(y - (x >> 1)) + 1) >> 1;
                    else if (z >= 0) v = (L(y - (x >> 1) - 2) + 2 * L(y - (x >> 1) - 1) + L(y - (x >> 1)) + 2) >> 2;
                    else if (z == -1) v = (T(0) + 2 * T(-1) + L(0) + 2) >> 2;
                    else v = (T(x - 1) + 2 * T(x - 2) + T(x - 3) + 2) >> 2; break; }
            case 7: v = !(y & 1) ? (T(x + (y >> 1)) + T(x + (y >> 1) + 1) + 1) >> 1
                                 : (T(x + (y >> 1)) + 2 * T(x + (y >> 1) + 1) + T(x + (y >> 1) + 2) + 2) >> 2; break;
            case 8: { int z = x + 2 * y;
                    if (z < 5 && !(z & 1)) v = (L(y + (x >> 1)) + L(y + (x >> 1) + 1) + 1) >> 1;
                    else if (z < 5) v = (L(y + (x >> 1)) + 2 * L(y + (x >> 1) + 1) + L(y + (x >> 1) + 2) + 2) >> 2;
                    else if (z == 5) v = (L(2) + 3 * L(3) + 2) >> 2;
                    else v = L(3); break; }
            default: {
                int s = 0;
                if (ht && hl) { for (int k = 0; k < 4; ++k) s += top[k] + left[k]; v = (s + 4) >> 3; }
                else if (ht) { for (int k = 0; k < 4; ++k) s += top[k]; v = (s + 2) >> 2; }
                else if (hl) { for (int k = 0; k < 4; ++k) s += left[k]; v = (s + 2) >> 2; }
                else v = 128;
            }
            }
            pred[y * 4 + x] = (uint8_t)v;
        }
#undef T
#undef L
}
static int nn_mode_ok(int m, int n, int ht, int hl) {                           /* fdv.h:2827 */
    switch (m) {
    case 0: return 1;
    case 1: return ht;
    case 2: return hl;
    case 3: return ht && hl && (n == 8 || n == 16 || n == 32);
    }
    return 0;
}
void oracle_intra_nxn(int mode, const uint8_t *top, const uint8_t *left, uint8_t tl,
                      int n, int ht, int hl, uint8_t *pred) {                   /* fdv.h:2851-2910 */
    OPC(OPC_INTRA, 3 * n * n);
    if (mode == 3 && nn_mode_ok(3, n, ht, hl)) {
        int half = n / 2, H = 0, V = 0;
        for (int k = 1; k <= half; ++k) {
            int t0 = (half - 1 - k) < 0 ? tl : top[half - 1 - k];
            int l0 = (half - 1 - k) < 0 ? tl : left[half - 1 - k];
            H += k * (top[half - 1 + k] - t0);
            V += k * (left[half - 1 + k] - l0);
        }
        int a = 16 * (left[n - 1] + top[n - 1]), b, c;
        if (n == 32) { b = (11 * H + 512) >> 10; c = (11 * V + 512) >> 10; }
        else if (n == 16) { b = (5 * H + 32) >> 6; c = (5 * V + 32) >> 6; }
        else { b = (17 * H + 16) >> 5; c = (17 * V + 16) >> 5; }
        int c0 = half - 1;
        for (int y = 0; y < n; ++y) { int base = a + c * (y - c0) + 16; for (int x = 0; x < n; ++x) pred[y * n + x] = (uint8_t)clipb((base + b * (x - c0)) >> 5); }
    } else if (mode == 1 && ht) {
        for (int y = 0; y < n; ++y) for (int x = 0; x < n; ++x) pred[y * n + x] = top[x];
    } else if (mode == 2 && hl) {
        for (int y = 0; y < n; ++y) for (int x = 0; x < n; ++x) pred[y * n + x] = left[y];
    } else {
        int dc, s = 0;
        if (ht && hl) { for (int k = 0; k < n; ++k) s += top[k] + left[k]; dc = (s + n) / (2 * n); }
        else if (ht) { for (int k = 0; k < n; ++k) s += top[k]; dc = (s + n / 2) / n; }
        else if (hl) { for (int k = 0; k < n; ++k) s += left[k]; dc = (s + n / 2) / n; }
        else dc = 128;
        memset(pred, dc, (size_t)n * n);
    }
}

/* -------------------------------------------------------------- inter -- */
/* A plane read with edge clamping (see the header comment). */
typedef struct { const uint8_t *p; int w, h, stride; } cplane;
static int PX(const cplane *r, int x, int y) {
    x = x < 0 ? 0 : (x >= r->w ? r->w - 1 : x);
    y = y < 0 ? 0 : (y >= r->h ? r->h - 1 : y);
    return r->p[(size_t)y * r->stride + x];
}
static int tap6(int a, int b, int c, int d, int e, int f) { return a - 5 * b + 20 * c + 20 * d - 5 * e + f; }
static int hf(const cplane *r, int x, int y) { return tap6(PX(r,x-2,y), PX(r,x-1,y), PX(r,x,y), PX(r,x+1,y), PX(r,x+2,y), PX(r,x+3,y)); }
static int vf(const cplane *r, int x, int y) { return tap6(PX(r,x,y-2), PX(r,x,y-1), PX(r,x,y), PX(r,x,y+1), PX(r,x,y+2), PX(r,x,y+3)); }
static int half_b(const cplane *r, int x, int y) { return clipb((hf(r, x, y) + 16) >> 5); }
static int half_h(const cplane *r, int x, int y) { return clipb((vf(r, x, y) + 16) >> 5); }
static int half_j(const cplane *r, int x, int y) {
    int jj = tap6(hf(r, x, y - 2), hf(r, x, y - 1), hf(r, x, y), hf(r, x, y + 1), hf(r, x, y + 2), hf(r, x, y + 3));
    return clipb((jj + 512) >> 10);
}
/* fdv.h:2970-2990 (the block form at :3082-3230 is proven bit-identical to it). */
static int interp(const cplane *r, int x, int y, int fx, int fy) {
    switch (fy * 4 + fx) {
    case 0: return PX(r, x, y);
    case 1: return (PX(r, x, y) + half_b(r, x, y) + 1) >> 1;
    case 2: return half_b(r, x, y);
    case 3: return (half_b(r, x, y) + PX(r, x + 1, y) + 1) >> 1;
    case 4: return (PX(r, x, y) + half_h(r, x, y) + 1) >> 1;
    case 5: return (half_b(r, x, y) + half_h(r, x, y) + 1) >> 1;
    case 6: return (half_b(r, x, y) + half_j(r, x, y) + 1) >> 1;
    case 7: return (half_b(r, x, y) + half_h(r, x + 1, y) + 1) >> 1;
    case 8: return half_h(r, x, y);
    case 9: return (half_h(r, x, y) + half_j(r, x, y) + 1) >> 1;
    case 10: return half_j(r, x, y);
    case 11: return (half_j(r, x, y) + half_h(r, x + 1, y) + 1) >> 1;
    case 12: return (half_h(r, x, y) + PX(r, x, y + 1) + 1) >> 1;
    case 13: return (half_h(r, x, y) + half_b(r, x, y + 1) + 1) >> 1;
    case 14: return (half_j(r, x, y) + half_b(r, x, y + 1) + 1) >> 1;
    default: return (half_h(r, x + 1, y) + half_b(r, x, y + 1) + 1) >> 1;
    }
}
static void mc_luma(const cplane *r, int bx, int by, int bw, int bh, int mvx, int mvy, uint8_t *dst, int ds) {
    int fx = mvx & 3, fy = mvy & 3, ix = bx + (mvx >> 2), iy = by + (mvy >> 2);
#ifdef ORACLE_OPCOUNT
    static const int kPhaseOps[16] = {1, 15, 12, 15, 15, 26, 80, 26, 12, 80, 66, 80, 15, 26, 80, 26};
    OPC(OPC_MC, kPhaseOps[fy * 4 + fx] * bw * bh);
#endif
    for (int i = 0; i < bh; ++i) for (int j = 0; j < bw; ++j) dst[i * ds + j] = (uint8_t)interp(r, ix + j, iy + i, fx, fy);
}
static void mc_chroma(const cplane *r, int bx, int by, int bw, int bh, int mvx, int mvy, uint8_t *dst, int ds) { /* :3260 */
    int fx = mvx & 3, fy = mvy & 3, ix = bx + (mvx >> 2), iy = by + (mvy >> 2);
    OPC(OPC_MC, 10 * bw * bh);
    for (int i = 0; i < bh; ++i) for (int j = 0; j < bw; ++j) {
        int a = PX(r, ix + j, iy + i), b = PX(r, ix + j + 1, iy + i), c = PX(r, ix + j, iy + i + 1), d = PX(r, ix + j + 1, iy + i + 1);
        int top = a * (4 - fx) + b * fx, bot = c * (4 - fx) + d * fx;
        dst[i * ds + j] = (uint8_t)((top * (4 - fy) + bot * fy + 8) >> 4);
    }
}
void oracle_mc_luma(const uint8_t *plane, int w, int h, int stride, int bx, int by, int bw, int bh,
                    int mvx, int mvy, uint8_t *dst, int ds) {
    cplane r = {plane, w, h, stride};
    mc_luma(&r, bx, by, bw, bh, mvx, mvy, dst, ds);
}
void oracle_mc_chroma(const uint8_t *plane, int w, int h, int stride, int bx, int by, int bw, int bh,
                      int mvx, int mvy, uint8_t *dst, int ds) {
    cplane r = {plane, w, h, stride};
    mc_chroma(&r, bx, by, bw, bh, mvx, mvy, dst, ds);
}
static int block_sad(const uint8_t *cur, int cs, const cplane *r, int bx, int by, int bw, int bh, int mvx, int mvy) { /* :3321 */
    uint8_t pred[256];
    mc_luma(r, bx, by, bw, bh, mvx, mvy, pred, bw);
    OPC(OPC_SAD, 2 * bw * bh);
    int sad = 0;
    for (int i = 0; i < bh; ++i) for (int j = 0; j < bw; ++j) sad += iabs(cur[(size_t)(by + i) * cs + bx + j] - pred[i * bw + j]);
    return sad;
}
static int me_search(const uint8_t *cur, int cs, const cplane *r, int bx, int by, int bw, int bh, int range,
                     int pmx, int pmy, int *mvx, int *mvy) {                    /* fdv.h:3375-3466 */
    static const int LD[8][2] = {{0, 8}, {0, -8}, {8, 0}, {-8, 0}, {4, 4}, {4, -4}, {-4, 4}, {-4, -4}};
    static const int SD[4][2] = {{0, 4}, {0, -4}, {4, 0}, {-4, 0}};
    static const int SP[4][2] = {{0, -1}, {0, 1}, {-1, 0}, {1, 0}};
    int lim = range * 4, bx_ = 0, by_ = 0;
    int best = block_sad(cur, cs, r, bx, by, bw, bh, 0, 0);
    int px = (pmx >> 2) * 4, py = (pmy >> 2) * 4;
    if (px < -lim) px = -lim; else if (px > lim) px = lim;
    if (py < -lim) py = -lim; else if (py > lim) py = lim;
    if (px != 0 || py != 0) { int s = block_sad(cur, cs, r, bx, by, bw, bh, px, py); if (s < best) { best = s; bx_ = px; by_ = py; } }
    for (int it = 0; it < 64; ++it) {
        int cx = bx_, cy = by_, moved = 0;
        for (int k = 0; k < 8; ++k) {
            int nx = cx + LD[k][0], ny = cy + LD[k][1];
            if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
            int s = block_sad(cur, cs, r, bx, by, bw, bh, nx, ny);
            if (s < best) { best = s; bx_ = nx; by_ = ny; moved = 1; }
        }
        if (!moved) break;
    }
    { int cx = bx_, cy = by_;
      for (int k = 0; k < 4; ++k) {
          int nx = cx + SD[k][0], ny = cy + SD[k][1];
          if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
          int s = block_sad(cur, cs, r, bx, by, bw, bh, nx, ny);
          if (s < best) { best = s; bx_ = nx; by_ = ny; }
      } }
    for (int step = 2; step >= 1 && best > 0; step >>= 1) {
        int cx = bx_, cy = by_;
        for (int k = 0; k < 4; ++k) {
            int s = block_sad(cur, cs, r, bx, by, bw, bh, cx + SP[k][0] * step, cy + SP[k][1] * step);
            if (s < best) { best = s; bx_ = cx + SP[k][0] * step; by_ = cy + SP[k][1] * step; }
        }
    }
    *mvx = bx_; *mvy = by_;
    return best;
}
int oracle_me_search(const uint8_t *cur, int cs, const uint8_t *ref, int w, int h, int rs,
                     int bx, int by, int bw, int bh, int range, int pmx, int pmy, int *mvx, int *mvy) {
    cplane r = {ref, w, h, rs};
    return me_search(cur, cs, &r, bx, by, bw, bh, range, pmx, pmy, mvx, mvy);
}

/* ------------------------------------------------------------ deblock -- */
static void filter_edge(uint8_t *a, int step, int alpha, int beta, int tc) {    /* fdv.h:3491 */
    OPC(OPC_DBK, 20);
    int p1 = a[-2 * step], p0 = a[-step], q0 = a[0], q1 = a[step];
    if (iabs(p0 - q0) < alpha && iabs(p1 - p0) < beta && iabs(q1 - q0) < beta) {
        int d = ((q0 - p0) * 4 + (p1 - q1) + 4) >> 3;
        d = d < -tc ? -tc : (d > tc ? tc : d);
        a[-step] = (uint8_t)clipb(p0 + d);
        a[0] = (uint8_t)clipb(q0 - d);
    }
}
void oracle_deblock(uint8_t *pl, int w, int h, int stride, int qp) {            /* fdv.h:3617-3625 */
    int alpha = 6 + qp, beta = 2 + qp / 4, tc = 1 + qp / 10;
    for (int y = 0; y < h; ++y) for (int x = 8; x < w; x += 8) filter_edge(&pl[y * stride + x], 1, alpha, beta, tc);
    for (int y = 8; y < h; y += 8) for (int x = 0; x < w; ++x) filter_edge(&pl[y * stride + x], stride, alpha, beta, tc);
}

/* ---------------------------------------------------- coefficient sink -- */
/* The seven coefficient streams of fdv_cw (fdv.h:618-627). */
typedef struct { buf_t n, l, n8, l8, fl, nc, lc; int chroma; } cw_t;
static void cw_free(cw_t *w) { bfree(&w->n); bfree(&w->l); bfree(&w->n8); bfree(&w->l8); bfree(&w->fl); bfree(&w->nc); bfree(&w->lc); }
static void cw_cat(cw_t *d, const cw_t *s) {
    bcat(&d->n, &s->n); bcat(&d->l, &s->l); bcat(&d->n8, &s->n8); bcat(&d->l8, &s->l8);
    bcat(&d->fl, &s->fl); bcat(&d->nc, &s->nc); bcat(&d->lc, &s->lc);
}
static void cw_count(cw_t *w, unsigned v) { bput(w->chroma ? &w->nc : &w->n, (uint8_t)v); }
static void cw_level(cw_t *w, uint32_t z) { leb_put(w->chroma ? &w->lc : &w->l, z); }

/* fdv.h:5214-5278 */
static void code_block4(const uint8_t *cur, int cs, int cx, int cy, const uint8_t *pred, int ps, int px, int py,
                        uint8_t *rec, int rs, int rx, int ry, int qp, double lambda, cw_t *w, double *D, int *bits) {
    int16_t res[16], level[16], rr[16]; int32_t co[16], dc[16];
    const uint8_t *cb = &cur[(size_t)cy * cs + cx], *pb = &pred[(size_t)py * ps + px];
    OPC(OPC_PIX, 5 * 16);
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) res[i * 4 + j] = (int16_t)(cb[i * cs + j] - pb[i * ps + j]);
    oracle_fdct4x4(res, co);
    oracle_quant4x4(co, level, qp);
    oracle_rdoq4x4(level, res, qp, lambda);
    oracle_dequant4x4(level, dc, qp);
    oracle_idct4x4(dc, rr);
    int32_t ssd = 0;
    uint8_t *rb = &rec[(size_t)ry * rs + rx];
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) {
        int r = clipb(pb[i * ps + j] + rr[i * 4 + j]);
        rb[i * rs + j] = (uint8_t)r;
        int d = cb[i * cs + j] - r;
        ssd += d * d;
    }
    *D += (double)ssd;
    int last = -1;
    for (int k = 0; k < 16; ++k) if (level[ZZ4[k]] != 0) last = k;
    cw_count(w, (unsigned)(last + 1));
    *bits += bits_val((uint32_t)(last + 1));
    for (int k = 0; k <= last; ++k) { uint32_t z = zz_enc(level[ZZ4[k]]); cw_level(w, z); *bits += bits_val(z); }
}

/* fdv.h:5300-5414 */
static void code_residual(const uint8_t *cur, int cs, int ox, int oy, const uint8_t *pred, int n, int qp,
                          double lambda, uint8_t *rec, cw_t *w, double *ssd, int *bits) {
    double e = 0.0; int b = 0;
    if (n == 4) {
        code_block4(cur, cs, ox, oy, pred, n, 0, 0, rec, n, 0, 0, qp, lambda, w, &e, &b);
        *ssd += e; *bits += b;
        return;
    }
    for (int ry = 0; ry < n; ry += 8)
        for (int rx = 0; rx < n; rx += 8) {
            cw_t wA; memset(&wA, 0, sizeof wA);
            uint8_t recA[64];
            double eA = 0.0; int bA = 2;
            for (int sy = 0; sy < 8; sy += 4)
                for (int sx = 0; sx < 8; sx += 4)
                    code_block4(cur, cs, ox + rx + sx, oy + ry + sy, pred, n, rx + sx, ry + sy, recA, 8, sx, sy, qp, lambda, &wA, &eA, &bA);
            int16_t res8[64], lev8[64], rr8[64]; int32_t co8[64], dc8[64];
            const uint8_t *cB = &cur[(size_t)(oy + ry) * cs + ox + rx], *pB = &pred[(size_t)ry * n + rx];
            OPC(OPC_PIX, 5 * 64);
            for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) res8[i * 8 + j] = (int16_t)(cB[i * cs + j] - pB[i * n + j]);
            oracle_fdct8x8(res8, co8);
            oracle_quant8x8(co8, lev8, qp);
            oracle_dequant8x8(lev8, dc8, qp);
            oracle_idct8x8(dc8, rr8);
            uint8_t recB[64]; int32_t eBi = 0;
            for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) {
                int r = clipb(pB[i * n + j] + rr8[i * 8 + j]);
                recB[i * 8 + j] = (uint8_t)r;
                int d = cB[i * cs + j] - r; eBi += d * d;
            }
            double eB = (double)eBi;
            int last8 = 0;
            for (int k = 0; k < 64; ++k) if (lev8[ZZ8[k]] != 0) last8 = k + 1;
            int bB = 2 + bits_val((uint32_t)last8);
            for (int k = 0; k < last8; ++k) bB += bits_val(zz_enc(lev8[ZZ8[k]]));
            int emptyA = (wA.l.n == 0), emptyB = (last8 == 0);
            if (emptyA) bA = 2;
            if (emptyB) bB = 2;
            if (eA + lambda * bA <= eB + lambda * bB) {
                if (emptyA) bput(&w->fl, 0);
                else {
                    bput(&w->fl, 1);
                    bcat(w->chroma ? &w->nc : &w->n, &wA.n);
                    bcat(w->chroma ? &w->lc : &w->l, &wA.l);
                }
                for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) rec[(ry + i) * n + rx + j] = recA[i * 8 + j];
                e += eA; b += bA;
            } else {
                if (emptyB) bput(&w->fl, 0);
                else {
                    bput(&w->fl, 2);
                    bput(&w->n8, (uint8_t)last8);
                    for (int k = 0; k < last8; ++k) leb_put(&w->l8, zz_enc(lev8[ZZ8[k]]));
                }
                for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) rec[(ry + i) * n + rx + j] = recB[i * 8 + j];
                e += eB; b += bB;
            }
            cw_free(&wA);
        }
    *ssd += e; *bits += b;
}

/* ========================================================== P-frames == */
/* fdv.h:5576-5637: one chroma 8x8 block, SKIP (prediction only) or INTER. */
static void chroma_block(const uint8_t *cur, uint8_t *rec, int cw, const cplane *ref, int cbx, int cby,
                         int cmvx, int cmvy, int qp, int skip, cw_t *w) {
    uint8_t pred[64];
    mc_chroma(ref, cbx, cby, 8, 8, cmvx, cmvy, pred, 8);
    if (skip) { for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) rec[(cby + i) * cw + cbx + j] = pred[i * 8 + j]; return; }
    int16_t lv[4][16]; int last[4], any = 0, bi = 0;
    for (int sy = 0; sy < 8; sy += 4)
        for (int sx = 0; sx < 8; sx += 4, ++bi) {
            int16_t res[16], rres[16]; int32_t co[16], dc[16];
            OPC(OPC_PIX, 3 * 16);   /* residual and reconstruction */
            for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j)
                res[i * 4 + j] = (int16_t)(cur[(cby + sy + i) * cw + cbx + sx + j] - pred[(sy + i) * 8 + sx + j]);
            oracle_fdct4x4(res, co);
            oracle_quant4x4(co, lv[bi], qp);
            oracle_dequant4x4(lv[bi], dc, qp);
            oracle_idct4x4(dc, rres);
            for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j)
                rec[(cby + sy + i) * cw + cbx + sx + j] = (uint8_t)clipb(pred[(sy + i) * 8 + sx + j] + rres[i * 4 + j]);
            last[bi] = -1;
            for (int k = 0; k < 16; ++k) if (lv[bi][ZZ4[k]] != 0) last[bi] = k;
            if (last[bi] >= 0) any = 1;
        }
    if (!any) { bput(&w->fl, 0); return; }
    bput(&w->fl, 1);
    for (int b2 = 0; b2 < 4; ++b2) {
        bput(&w->nc, (uint8_t)(last[b2] + 1));
        for (int k = 0; k <= last[b2]; ++k) leb_put(&w->lc, zz_enc(lv[b2][ZZ4[k]]));
    }
}

typedef struct { int16_t x, y; uint8_t ref, inter; } mbmv_t;                      /* fdv.h:5680 */

static int merge_cands(const mbmv_t *mv, int mmw, int mbx, int mby, int pmvx, int pmvy, mbmv_t *out) { /* :5711 */
    int n = 0;
    out[0].x = (int16_t)pmvx; out[0].y = (int16_t)pmvy; out[0].ref = 0; out[0].inter = 1; n = 1;
    const int src[2][2] = {{mbx, mby - 1}, {mbx + 1, mby - 1}};
    for (int k = 0; k < 2 && n < 3; ++k) {
        int cx = src[k][0], cy = src[k][1];
        if (cx < 0 || cy < 0 || cx >= mmw) continue;
        const mbmv_t *m = &mv[(size_t)cy * mmw + cx];
        if (!m->inter) continue;
        int dup = 0;
        for (int j = 0; j < n; ++j) if (out[j].x == m->x && out[j].y == m->y && out[j].ref == m->ref) dup = 1;
        if (!dup) out[n++] = *m;
    }
    return n;
}

static void gather_nb(const uint8_t *buf, int stride, int bx, int by, int n, int ytop,
                      uint8_t *top, uint8_t *left, uint8_t *tl, int *ht, int *hl) {  /* fdv.h:5201 */
    *ht = by > ytop; *hl = bx > 0;
    for (int k = 0; k < n; ++k) { top[k] = 0; left[k] = 0; }
    if (*ht) for (int k = 0; k < n; ++k) top[k] = buf[(by - 1) * stride + bx + k];
    if (*hl) for (int k = 0; k < n; ++k) left[k] = buf[(by + k) * stride + bx - 1];
    *tl = (*ht && *hl) ? buf[(by - 1) * stride + bx - 1] : 128;
}

static int mb_satd(const uint8_t *cur, int cs, const uint8_t *pred, int ps, int n) {  /* fdv.h:4411 */
    int sum = 0;
    for (int i = 0; i < n; i += 4) for (int j = 0; j < n; j += 4) {
        uint8_t pk[16];
        for (int k = 0; k < 4; ++k) memcpy(pk + k * 4, pred + (size_t)(i + k) * ps + j, 4);
        sum += oracle_satd4x4(cur + (size_t)i * cs + j, cs, pk);
    }
    return sum;
}

/* One encoder instance: a w x h video with its two-frame reference pool. */
typedef struct {
    int w, h, range;
    uint8_t *ref[2][3];      /* [near/far][plane], tight planes */
    int near_i, nref;
    uint8_t *rec[3];
    int tally[4];
    uint8_t *modes;          /* per MB: chosen mode of the last P-frame (diagnostics) */
    int16_t *mvs;            /* per MB: chosen MV (x, y) */
} ounit_t;

void *oracle_open(int w, int h, int range) {
    if (w <= 0 || h <= 0 || (w & 15) || (h & 15)) return NULL;
    ounit_t *u = calloc(1, sizeof *u);
    u->w = w; u->h = h; u->range = range;
    size_t ys = (size_t)w * h, cs = ys / 4;
    for (int r = 0; r < 2; ++r) { u->ref[r][0] = calloc(ys, 1); u->ref[r][1] = calloc(cs, 1); u->ref[r][2] = calloc(cs, 1); }
    u->rec[0] = calloc(ys, 1); u->rec[1] = calloc(cs, 1); u->rec[2] = calloc(cs, 1);
    u->modes = calloc(ys / 256, 1);
    u->mvs = calloc(ys / 256 * 2, sizeof(int16_t));
    return u;
}
void oracle_close(void *p) {
    ounit_t *u = p;
    if (!u) return;
    for (int r = 0; r < 2; ++r) for (int k = 0; k < 3; ++k) free(u->ref[r][k]);
    for (int k = 0; k < 3; ++k) free(u->rec[k]);
    free(u->modes); free(u->mvs); free(u);
}

/* Output: 16 streams (caller frees with oracle_free). */
typedef struct { uint8_t *s[16]; size_t n[16]; } ostreams_t;
static void give(ostreams_t *o, int k, buf_t *b) { o->s[k] = b->b; o->n[k] = b->n; b->b = NULL; b->n = b->cap = 0; }
void oracle_free(void *p) { free(p); }

/* fdv.h:5764-6170: the macroblock loop of one P-frame over the whole unit,
 * followed by the band-local deblock. */
static void pframe(ounit_t *u, const uint8_t *cy, const uint8_t *cu, const uint8_t *cv, int qp, double lscale,
                   int force_skip, ostreams_t *out) {
    int w = u->w, h = u->h, cw = w / 2, mmw = w / 16, mmh = h / 16;
    int navail = u->nref >= 2 ? 2 : 1;
    uint8_t **nearp = u->ref[u->near_i], **farp = u->ref[1 - u->near_i];
    uint8_t **refp[2] = {nearp, navail == 2 ? farp : nearp};
    cplane rY[2], rU[2], rV[2];
    for (int r = 0; r < 2; ++r) {
        rY[r] = (cplane){refp[r][0], w, h, w};
        rU[r] = (cplane){refp[r][1], cw, h / 2, cw};
        rV[r] = (cplane){refp[r][2], cw, h / 2, cw};
    }
    uint8_t *ry = u->rec[0], *ru = u->rec[1], *rv = u->rec[2];
    buf_t S[9]; memset(S, 0, sizeof S);
    cw_t W; memset(&W, 0, sizeof W);
    uint8_t *mmap = calloc((size_t)mmw * mmh, 1);
    mbmv_t *mvmap = calloc((size_t)mmw * mmh, sizeof *mvmap);
    double lambda = lscale * 0.425 * pow(2.0, (qp - 12) / 3.0);
    memset(u->tally, 0, sizeof u->tally);
    const int R = u->range;

    for (int by = 0; by < h; by += 16) {
        int mbrow = by / 16, pmvx = 0, pmvy = 0;
        for (int bx = 0; bx < w; bx += 16) {
            int mbx = bx / 16, cbx = bx / 2, cby = by / 2;
#define MODECTX() ((mbx > 0 && mmap[mbrow * mmw + mbx - 1] ? 2 : 0) + (mbrow > 0 && mmap[(mbrow - 1) * mmw + mbx] ? 1 : 0))
            if (force_skip) {
                uint8_t pf[256];
                mc_luma(&rY[0], bx, by, 16, 16, 0, 0, pf, 16);
                bput(&S[MODECTX()], 0);
                mmap[mbrow * mmw + mbx] = 0;
                mvmap[mbrow * mmw + mbx] = (mbmv_t){0, 0, 0, 1};
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) ry[(by + i) * w + bx + j] = pf[i * 16 + j];
                chroma_block(NULL, ru, cw, &rU[0], cbx, cby, 0, 0, qp, 1, &W);
                chroma_block(NULL, rv, cw, &rV[0], cbx, cby, 0, 0, qp, 1, &W);
                u->tally[0]++;
                u->modes[mbrow * mmw + mbx] = 0;
                u->mvs[2 * (mbrow * mmw + mbx)] = 0; u->mvs[2 * (mbrow * mmw + mbx) + 1] = 0;
                continue;
            }
            uint8_t ntop[16], nleft[16], ntl; int iht, ihl;
            gather_nb(ry, w, bx, by, 16, 0, ntop, nleft, &ntl, &iht, &ihl);

            /* SKIP (fdv.h:5843-5899) */
            mbmv_t cand[3];
            int ncand = merge_cands(mvmap, mmw, mbx, mbrow, pmvx, pmvy, cand);
            int midx_bits = ncand > 1 ? 3 : 0;
            uint8_t pred_s[256]; int best_mi = 0; int32_t Ds_i = 0;
            for (int mi = 0; mi < ncand; ++mi) {
                uint8_t tp[256];
                mc_luma(&rY[cand[mi].ref], bx, by, 16, 16, cand[mi].x, cand[mi].y, tp, 16);
                int32_t e = 0;
                OPC(OPC_PIX, 3 * 256);   /* SSD */
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) { int d = cy[(by + i) * w + bx + j] - tp[i * 16 + j]; e += d * d; }
                if (mi == 0 || e < Ds_i) { Ds_i = e; best_mi = mi; memcpy(pred_s, tp, 256); }
            }
            int smvx = cand[best_mi].x, smvy = cand[best_mi].y, sref = cand[best_mi].ref;
            double Js = (double)Ds_i + lambda * (3 + midx_bits);
            double Jbest = Js;
            int skip_wins = (Js <= lambda * 14);

            /* INTER16 (fdv.h:5901-5943) */
            int mvx = 0, mvy = 0, best_ref = 0, sad16 = 0;
            uint8_t rec_i[256];
            buf_t isS; memset(&isS, 0, sizeof isS);
            cw_t isw; memset(&isw, 0, sizeof isw);
            double Ji = 1e30;
            for (int r = 0; r < navail && !skip_wins; ++r) {
                if (r > 0 && Jbest <= lambda * 16) break;
                int rmx, rmy;
                int rsad = me_search(cy, w, &rY[r], bx, by, 16, 16, R, pmvx, pmvy, &rmx, &rmy);
                uint8_t pr[256], rr[256];
                mc_luma(&rY[r], bx, by, 16, 16, rmx, rmy, pr, 16);
                cw_t tw; memset(&tw, 0, sizeof tw);
                buf_t tS; memset(&tS, 0, sizeof tS);
                bput(&tS, (uint8_t)r);
                uint32_t zx = zz_enc(rmx - pmvx), zy = zz_enc(rmy - pmvy);
                leb_put(&tS, zx); leb_put(&tS, zy);
                double dd = 0.0;
                int bb = 3 + 3 + bits_val(zx) + bits_val(zy);
                code_residual(cy, w, bx, by, pr, 16, qp, lambda, rr, &tw, &dd, &bb);
                double J = dd + lambda * bb;
                if (J < Jbest) Jbest = J;
                if (J < Ji) {
                    Ji = J; best_ref = r; mvx = rmx; mvy = rmy; sad16 = rsad;
                    memcpy(rec_i, rr, 256);
                    bfree(&isS); isS = tS; memset(&tS, 0, sizeof tS);
                    cw_free(&isw); isw = tw; memset(&tw, 0, sizeof tw);
                }
                bfree(&tS); cw_free(&tw);
            }

            /* INTRA (fdv.h:5945-5988) */
            double Jintra = 1e30; int best_sub = 0;
            uint8_t rec_in[256];
            cw_t inw; memset(&inw, 0, sizeof inw);
            if (!skip_wins && Jbest > lambda * 14) {
                uint8_t predI[256]; int sel = -1, sbest = 0;
                for (int sub = 0; sub < 4; ++sub) {
                    if (!nn_mode_ok(sub, 16, iht, ihl)) continue;
                    oracle_intra_nxn(sub, ntop, nleft, ntl, 16, iht, ihl, predI);
                    int sa = mb_satd(cy + (size_t)by * w + bx, w, predI, 16, 16);
                    if (sel < 0 || sa < sbest) { sbest = sa; sel = sub; }
                }
                if (sel >= 0) {
                    oracle_intra_nxn(sel, ntop, nleft, ntl, 16, iht, ihl, predI);
                    double Dn = 0.0; int bn = 6;
                    code_residual(cy, w, bx, by, predI, 16, qp, lambda, rec_in, &inw, &Dn, &bn);
                    Jintra = Dn + lambda * bn;
                    best_sub = sel;
                    if (Jintra < Jbest) Jbest = Jintra;
                }
            }

            /* INTER8 (fdv.h:5990-6033) */
            buf_t p8S; memset(&p8S, 0, sizeof p8S);
            cw_t w8; memset(&w8, 0, sizeof w8);
            uint8_t rec8[256];
            double D8 = 0.0; int b8 = 3, qmv[4][2];
            int try8 = !skip_wins && (Jbest > lambda * 19);
            if (try8) {
                int ssad = 0, qpx = pmvx, qpy = pmvy;
                for (int q = 0; q < 4; ++q) {
                    int qx = (q & 1) * 8, qy = (q >> 1) * 8, mx, my;
                    ssad += me_search(cy, w, &rY[0], bx + qx, by + qy, 8, 8, R, qpx, qpy, &mx, &my);
                    qmv[q][0] = mx; qmv[q][1] = my; qpx = mx; qpy = my;
                }
                if (sad16 > 0 && ssad * 10 >= sad16 * 9) try8 = 0;
                qpx = pmvx; qpy = pmvy;
                for (int q = 0; q < 4 && try8; ++q) {
                    int qx = (q & 1) * 8, qy = (q >> 1) * 8, mx = qmv[q][0], my = qmv[q][1];
                    uint32_t zdx = zz_enc(mx - qpx), zdy = zz_enc(my - qpy);
                    leb_put(&p8S, zdx); leb_put(&p8S, zdy);
                    b8 += bits_val(zdx) + bits_val(zdy);
                    qpx = mx; qpy = my;
                    uint8_t pred8[64], r8[64];
                    mc_luma(&rY[0], bx + qx, by + qy, 8, 8, mx, my, pred8, 8);
                    code_residual(cy, w, bx + qx, by + qy, pred8, 8, qp, lambda, r8, &w8, &D8, &b8);
                    for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) rec8[(qy + i) * 16 + qx + j] = r8[i * 8 + j];
                }
            }
            double J8 = try8 ? D8 + lambda * b8 : 1e30;

            /* Commit (fdv.h:6035-6160) */
            double Jmin = Js; int chosen = 0;
            if (Ji < Jmin) { Jmin = Ji; chosen = 1; }
            if (Jintra < Jmin) { Jmin = Jintra; chosen = 2; }
            if (J8 < Jmin) { Jmin = J8; chosen = 3; }
            u->tally[chosen]++;
            bput(&S[MODECTX()], (uint8_t)chosen);
            mmap[mbrow * mmw + mbx] = (uint8_t)chosen;
            u->modes[mbrow * mmw + mbx] = (uint8_t)chosen;
            if (chosen == 0) {
                if (ncand > 1) bput(&S[PS_MERGE_], (uint8_t)best_mi);
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) ry[(by + i) * w + bx + j] = pred_s[i * 16 + j];
                chroma_block(cu, ru, cw, &rU[sref], cbx, cby, smvx / 2, smvy / 2, qp, 1, &W);
                chroma_block(cv, rv, cw, &rV[sref], cbx, cby, smvx / 2, smvy / 2, qp, 1, &W);
                mvmap[mbrow * mmw + mbx] = (mbmv_t){(int16_t)smvx, (int16_t)smvy, (uint8_t)sref, 1};
                pmvx = smvx; pmvy = smvy;
            } else if (chosen == 1) {
                bput(&S[PS_REF_], isS.b[0]);
                int part = 0;
                for (size_t q = 1; q < isS.n; ++q) {
                    bput(&S[part ? PS_MVY_ : PS_MVX_], isS.b[q]);
                    if (!(isS.b[q] & 0x80)) ++part;
                }
                cw_cat(&W, &isw);
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) ry[(by + i) * w + bx + j] = rec_i[i * 16 + j];
                pmvx = mvx; pmvy = mvy;
                mvmap[mbrow * mmw + mbx] = (mbmv_t){(int16_t)mvx, (int16_t)mvy, (uint8_t)best_ref, 1};
                chroma_block(cu, ru, cw, &rU[best_ref], cbx, cby, mvx / 2, mvy / 2, qp, 0, &W);
                chroma_block(cv, rv, cw, &rV[best_ref], cbx, cby, mvx / 2, mvy / 2, qp, 0, &W);
            } else if (chosen == 2) {
                bput(&S[PS_SUB_], (uint8_t)best_sub);
                cw_cat(&W, &inw);
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) ry[(by + i) * w + bx + j] = rec_in[i * 16 + j];
                const uint8_t *csrc[2] = {cu, cv};
                uint8_t *crec[2] = {ru, rv};
                for (int pl = 0; pl < 2; ++pl) {
                    uint8_t ct[8], cl[8], ctl; int cht, chl;
                    gather_nb(crec[pl], cw, cbx, cby, 8, 0, ct, cl, &ctl, &cht, &chl);
                    uint8_t cpred[64], crec8[64];
                    oracle_intra_nxn(best_sub, ct, cl, ctl, 8, cht, chl, cpred);
                    double dd = 0.0; int bb = 0;
                    W.chroma = 1;
                    code_residual(csrc[pl], cw, cbx, cby, cpred, 8, qp, lambda, crec8, &W, &dd, &bb);
                    W.chroma = 0;
                    for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) crec[pl][(cby + i) * cw + cbx + j] = crec8[i * 8 + j];
                }
                mvmap[mbrow * mmw + mbx] = (mbmv_t){0, 0, 0, 0};
            } else {
                int part = 0;
                for (size_t q = 0; q < p8S.n; ++q) {
                    bput(&S[(part & 1) ? PS_MVY_ : PS_MVX_], p8S.b[q]);
                    if (!(p8S.b[q] & 0x80)) ++part;
                }
                cw_cat(&W, &w8);
                for (int i = 0; i < 16; ++i) for (int j = 0; j < 16; ++j) ry[(by + i) * w + bx + j] = rec8[i * 16 + j];
                pmvx = qmv[3][0]; pmvy = qmv[3][1];
                mvmap[mbrow * mmw + mbx] = (mbmv_t){(int16_t)qmv[3][0], (int16_t)qmv[3][1], 0, 1};
                const uint8_t *csrc[2] = {cu, cv};
                uint8_t *crec[2] = {ru, rv};
                const cplane *cref[2] = {&rU[0], &rV[0]};
                for (int pl = 0; pl < 2; ++pl)
                    for (int q = 0; q < 4; ++q) {
                        int qcx = (q & 1) * 4, qcy = (q >> 1) * 4;
                        uint8_t cpred[16], crec4[16];
                        mc_chroma(cref[pl], cbx + qcx, cby + qcy, 4, 4, qmv[q][0] / 2, qmv[q][1] / 2, cpred, 4);
                        double dd = 0.0; int bb = 0;
                        W.chroma = 1;
                        code_residual(csrc[pl], cw, cbx + qcx, cby + qcy, cpred, 4, qp, lambda, crec4, &W, &dd, &bb);
                        W.chroma = 0;
                        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) crec[pl][(cby + qcy + i) * cw + cbx + qcx + j] = crec4[i * 4 + j];
                    }
            }
            u->mvs[2 * (mbrow * mmw + mbx)] = mvmap[mbrow * mmw + mbx].x;
            u->mvs[2 * (mbrow * mmw + mbx) + 1] = mvmap[mbrow * mmw + mbx].y;
            bfree(&isS); cw_free(&isw); cw_free(&inw); bfree(&p8S); cw_free(&w8);
#undef MODECTX
        }
    }
    oracle_deblock(ry, w, h, w, qp);
    oracle_deblock(ru, cw, h / 2, cw, qp);
    oracle_deblock(rv, cw, h / 2, cw, qp);
    for (int k = 0; k < 9; ++k) give(out, k, &S[k]);
    give(out, 9, &W.n); give(out, 10, &W.l); give(out, 11, &W.n8); give(out, 12, &W.l8);
    give(out, 13, &W.fl); give(out, 14, &W.nc); give(out, 15, &W.lc);
    free(mmap); free(mvmap);
}

/* ============================================================ I-frames == */
/* The intra quadtree of fdv_image_encode (fdv.h:3653-4583, :4746-4879). */
typedef struct { buf_t s[7]; cw_t c; } isink_t;   /* 7 structure streams + coefficient streams */
static void isink_free(isink_t *k) { for (int i = 0; i < 7; ++i) bfree(&k->s[i]); cw_free(&k->c); }
static void isink_cat(isink_t *d, const isink_t *s) { for (int i = 0; i < 7; ++i) bcat(&d->s[i], &s->s[i]); cw_cat(&d->c, &s->c); }

static int zidx4(int lx, int ly) {                                              /* fdv.h:3659 */
    int z = 0;
    for (int b = 8; b; b >>= 1) z = (z << 2) | ((ly & b) ? 2 : 0) | ((lx & b) ? 1 : 0);
    return z;
}
static int cell_done(int x, int y, int bx, int by) {                            /* fdv.h:3677 */
    int cx0 = bx & ~63, cy0 = by & ~63;
    if (y < cy0) return 1;
    if (x < cx0) return 1;
    if (x >= cx0 + 64) return 0;
    return zidx4((x - cx0) >> 2, (y - cy0) >> 2) < zidx4((bx - cx0) >> 2, (by - cy0) >> 2);
}
static int mode_ok4(int m, int ht, int htr, int hl, int htl) {                  /* fdv.h:3709 */
    switch (m) {
    case 0: return 1;
    case 1: return ht;
    case 2: case 8: return hl;
    case 3: case 7: return ht && htr;
    case 4: case 5: case 6: return ht && hl && htl;
    }
    return 0;
}

typedef struct { const uint8_t *src; int stride; uint8_t *rec; int w, h, qp; double lambda; uint8_t *mmap; int mmw; } ictx_t;

static double intra_leaf4(ictx_t *x, int bx, int by, int *mode_out, cw_t *cw) {  /* fdv.h:3907-4111 */
    const uint8_t *src = x->src; int stride = x->stride, w = x->w, qp = x->qp; double lambda = x->lambda;
    uint8_t *rec = x->rec;
    uint8_t top[8], left[4], tl;
    int ht = by > 0, hl = bx > 0, htl = ht && hl;
    int htr = ht && (bx + 4 < w) && cell_done(bx + 4, by - 1, bx, by);
    memset(top, 0, 8); memset(left, 0, 4); tl = 128;
    if (ht) {
        for (int j = 0; j < 4; ++j) top[j] = rec[(by - 1) * w + bx + j];
        for (int j = 4; j < 8; ++j) top[j] = htr ? rec[(by - 1) * w + bx + j] : top[3];
    }
    if (hl) for (int i = 0; i < 4; ++i) left[i] = rec[(by + i) * w + bx - 1];
    if (htl) tl = rec[(by - 1) * w + bx - 1];
    uint8_t cp[9][16]; int cs[9], cm[9], nc = 0;
    const uint8_t *sblk = &src[(size_t)by * stride + bx];
    for (int m = 0; m < 9; ++m) {
        if (!mode_ok4(m, ht, htr, hl, htl)) continue;
        oracle_intra4x4(m, top, left, tl, ht, hl, cp[nc]);
        cs[nc] = oracle_satd4x4(sblk, stride, cp[nc]);
        cm[nc] = m; ++nc;
    }
    int ntry = qp < 12 ? nc : (nc < 2 ? nc : 2);
    for (int a = 0; a < ntry; ++a) {
        int bst = a;
        for (int b2 = a + 1; b2 < nc; ++b2) if (cs[b2] < cs[bst]) bst = b2;
        if (bst != a) {
            int t = cs[a]; cs[a] = cs[bst]; cs[bst] = t;
            t = cm[a]; cm[a] = cm[bst]; cm[bst] = t;
            uint8_t tp[16]; memcpy(tp, cp[a], 16); memcpy(cp[a], cp[bst], 16); memcpy(cp[bst], tp, 16);
        }
    }
    double best_cost = -1.0; int best_mode = 0, best_c = 0;
    for (int c = 0; c < ntry; ++c) {
        if (c > 0 && qp >= 12 && (int64_t)cs[c] * 4 > (int64_t)cs[0] * 5) break;
        const uint8_t *pred = cp[c];
        int16_t res[16], level[16], rres[16]; int32_t co[16], dc[16];
        OPC(OPC_PIX, 5 * 16);
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) res[i * 4 + j] = (int16_t)(sblk[i * stride + j] - pred[i * 4 + j]);
        oracle_fdct4x4(res, co);
        oracle_quant4x4(co, level, qp);
        oracle_dequant4x4(level, dc, qp);
        oracle_idct4x4(dc, rres);
        int32_t ssd = 0; int bits = 3;
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) { int r = clipb(pred[i * 4 + j] + rres[i * 4 + j]); int d = sblk[i * stride + j] - r; ssd += d * d; }
        int blast = -1;
        for (int k = 0; k < 16; ++k) if (level[ZZ4[k]] != 0) blast = k;
        bits += bits_val((uint32_t)(blast + 1));
        for (int k = 0; k <= blast; ++k) bits += bits_val(zz_enc(level[ZZ4[k]]));
        double J = (double)ssd + lambda * bits;
        if (best_cost < 0.0 || J < best_cost) { best_cost = J; best_mode = cm[c]; best_c = c; }
    }
    int16_t res[16], level[16], rres[16]; int32_t co[16], dc[16];
    const uint8_t *pred = cp[best_c];
    OPC(OPC_PIX, 5 * 16);
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) res[i * 4 + j] = (int16_t)(sblk[i * stride + j] - pred[i * 4 + j]);
    oracle_fdct4x4(res, co);
    oracle_quant4x4(co, level, qp);
    oracle_rdoq4x4(level, res, qp, lambda);
    oracle_dequant4x4(level, dc, qp);
    oracle_idct4x4(dc, rres);
    int32_t fssd = 0;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) {
        int r = clipb(pred[i * 4 + j] + rres[i * 4 + j]);
        rec[(by + i) * w + bx + j] = (uint8_t)r;
        int d = sblk[i * stride + j] - r; fssd += d * d;
    }
    *mode_out = best_mode;
    int last = -1;
    for (int k = 0; k < 16; ++k) if (level[ZZ4[k]] != 0) last = k;
    int fbits = 3 + bits_val((uint32_t)(last + 1));
    bput(&cw->n, (uint8_t)(last + 1));
    for (int k = 0; k <= last; ++k) { uint32_t z = zz_enc(level[ZZ4[k]]); leb_put(&cw->l, z); fbits += bits_val(z); }
    return (double)fssd + lambda * fbits;
}

static double intra_leafn(ictx_t *x, int bx, int by, int n, int *mode_out, cw_t *cw) {  /* fdv.h:4442-4484 */
    uint8_t top[64], left[64], tl; int ht, hl;
    gather_nb(x->rec, x->w, bx, by, n, 0, top, left, &tl, &ht, &hl);
    double best = -1.0; int best_mode = 0;
    uint8_t *pred = malloc((size_t)n * n), *trec = malloc((size_t)n * n), *brec = malloc((size_t)n * n);
    cw_t bw; memset(&bw, 0, sizeof bw);
    for (int m = 0; m < 4; ++m) {
        if (!nn_mode_ok(m, n, ht, hl)) continue;
        cw_t tw; memset(&tw, 0, sizeof tw);
        oracle_intra_nxn(m, top, left, tl, n, ht, hl, pred);
        double D = 0.0; int bits = 3;
        code_residual(x->src, x->stride, bx, by, pred, n, x->qp, x->lambda, trec, &tw, &D, &bits);
        double J = D + x->lambda * bits;
        if (best < 0.0 || J < best) {
            best = J; best_mode = m;
            memcpy(brec, trec, (size_t)n * n);
            cw_free(&bw); bw = tw; memset(&tw, 0, sizeof tw);
        }
        cw_free(&tw);
    }
    for (int i = 0; i < n; ++i) memcpy(&x->rec[(size_t)(by + i) * x->w + bx], brec + (size_t)i * n, (size_t)n);
    cw_cat(cw, &bw);
    cw_free(&bw);
    free(pred); free(trec); free(brec);
    *mode_out = best_mode;
    return best;
}

static int nn_to_4x4(int m) { return m == 1 ? 1 : (m == 2 ? 2 : 0); }           /* fdv.h:4400 */

static double intra_node(ictx_t *x, int bx, int by, int n, isink_t *sink, int depth) {  /* fdv.h:4494-4582 */
    int hn = n / 2;
    if (bx + n > x->w || by + n > x->h) {
        double J = 0.0;
        for (int k = 0; k < 4; ++k) {
            int cx = bx + (k & 1) * hn, cy = by + (k >> 1) * hn;
            if (cx >= x->w || cy >= x->h) continue;
            J += intra_node(x, cx, cy, hn, sink, depth + 1);
        }
        return J;
    }
    if (n == 4) {
        int mode = 0;
        double J = intra_leaf4(x, bx, by, &mode, &sink->c);
        int cx = bx / 4, cy = by / 4;
        int Lm = cx > 0 ? x->mmap[cy * x->mmw + cx - 1] : 0;
        int Am = cy > 0 ? x->mmap[(cy - 1) * x->mmw + cx] : 0;
        bput(&sink->s[Lm == Am ? IS_MODE0_ : IS_MODE1_], (uint8_t)mode);
        x->mmap[cy * x->mmw + cx] = (uint8_t)mode;
        return J;
    }
    isink_t sw; memset(&sw, 0, sizeof sw);
    double Jsplit = 0.0;
    for (int k = 0; k < 4; ++k) Jsplit += intra_node(x, bx + (k & 1) * hn, by + (k >> 1) * hn, hn, &sw, depth + 1);
    int cells = n / 4, mx0 = bx / 4, my0 = by / 4;
    uint8_t *rs = malloc((size_t)n * n), *ms = malloc((size_t)cells * cells);
    for (int i = 0; i < n; ++i) memcpy(rs + (size_t)i * n, &x->rec[(size_t)(by + i) * x->w + bx], (size_t)n);
    for (int i = 0; i < cells; ++i) memcpy(ms + (size_t)i * cells, &x->mmap[(size_t)(my0 + i) * x->mmw + mx0], (size_t)cells);
    cw_t lcw; memset(&lcw, 0, sizeof lcw);
    int mode = 0;
    double Jleaf = intra_leafn(x, bx, by, n, &mode, &lcw);
    int split = Jsplit < Jleaf;
    bput(&sink->s[IS_SPLIT0_ + depth], (uint8_t)split);
    double J;
    if (split) {
        for (int i = 0; i < n; ++i) memcpy(&x->rec[(size_t)(by + i) * x->w + bx], rs + (size_t)i * n, (size_t)n);
        for (int i = 0; i < cells; ++i) memcpy(&x->mmap[(size_t)(my0 + i) * x->mmw + mx0], ms + (size_t)i * cells, (size_t)cells);
        isink_cat(sink, &sw);
        J = Jsplit;
    } else {
        bput(&sink->s[IS_MODEB_], (uint8_t)mode);
        for (int i = 0; i < cells; ++i) memset(&x->mmap[(size_t)(my0 + i) * x->mmw + mx0], nn_to_4x4(mode), (size_t)cells);
        cw_cat(&sink->c, &lcw);
        J = Jleaf;
    }
    isink_free(&sw); cw_free(&lcw); free(rs); free(ms);
    return J;
}

/* One plane through the intra image codec's analysis (fdv.h:4845-4879). */
static void image_plane(const uint8_t *src, int w, int h, int qp, uint8_t *rec, ostreams_t *out) {
    ictx_t x = {src, w, rec, w, h, qp, 0.425 * pow(2.0, (qp - 12) / 3.0), calloc((size_t)(w / 4) * (h / 4), 1), w / 4};
    isink_t sink; memset(&sink, 0, sizeof sink);
    for (int r = 0; r < (h + 63) / 64; ++r)
        for (int c = 0; c < (w + 63) / 64; ++c)
            intra_node(&x, c * 64, r * 64, 64, &sink, 0);
    free(x.mmap);
    oracle_deblock(rec, w, h, w, qp);
    for (int k = 0; k < 7; ++k) give(out, k, &sink.s[k]);
    give(out, 7, &sink.c.n); give(out, 8, &sink.c.l); give(out, 9, &sink.c.n8); give(out, 10, &sink.c.l8);
    give(out, 11, &sink.c.fl);
    bfree(&sink.c.nc); bfree(&sink.c.lc);
}

/* ============================================================ driver == */
/* Encode one frame of the unit.  is_intra selects the path; the reference
 * pool rotates exactly as fdv_video_encode does (fdv.h:6842-6846).
 * For a P-frame `out` receives 16 streams in out[0]; for a key frame out[0..2]
 * receive the Y, U and V planes' 12 streams each.  Free each stream with
 * oracle_free. */
int oracle_frame(void *p, const uint8_t *i420, int is_intra, int qp, double lscale, int force_skip,
                 ostreams_t *out, int tally[4]) {
    ounit_t *u = p;
    int w = u->w, h = u->h, cw = w / 2, ch = h / 2;
    const uint8_t *cy = i420, *cu = i420 ? i420 + (size_t)w * h : NULL, *cv = cu ? cu + (size_t)cw * ch : NULL;
    if (is_intra) {
        image_plane(cy, w, h, qp, u->rec[0], &out[0]);
        image_plane(cu, cw, ch, qp, u->rec[1], &out[1]);
        image_plane(cv, cw, ch, qp, u->rec[2], &out[2]);
    } else {
        pframe(u, cy, cu, cv, qp, lscale, force_skip, &out[0]);
        if (tally) memcpy(tally, u->tally, sizeof u->tally);
    }
    int far_i = 1 - u->near_i;
    memcpy(u->ref[far_i][0], u->rec[0], (size_t)w * h);
    memcpy(u->ref[far_i][1], u->rec[1], (size_t)cw * ch);
    memcpy(u->ref[far_i][2], u->rec[2], (size_t)cw * ch);
    u->near_i = far_i;
    u->nref = is_intra ? 1 : (u->nref < 2 ? u->nref + 1 : 2);
    return 0;
}

/* The reconstruction of the last frame (tight I420). */
void oracle_recon(void *p, uint8_t *i420) {
    ounit_t *u = p;
    size_t ys = (size_t)u->w * u->h, cs = ys / 4;
    memcpy(i420, u->rec[0], ys); memcpy(i420 + ys, u->rec[1], cs); memcpy(i420 + ys + cs, u->rec[2], cs);
}

/* Per-macroblock mode and MV of the last P-frame, for localising a mismatch. */
void oracle_mb_info(void *p, uint8_t *modes, int16_t *mvs) {
    ounit_t *u = p;
    size_t nmb = (size_t)(u->w / 16) * (u->h / 16);
    memcpy(modes, u->modes, nmb);
    memcpy(mvs, u->mvs, nmb * 2 * sizeof(int16_t));
}

/* Seed the reference pool: nearest and (optionally) second reference, tight I420. */
void oracle_set_refs(void *p, const uint8_t *near_i420, const uint8_t *far_i420) {
    ounit_t *u = p;
    size_t ys = (size_t)u->w * u->h, cs = ys / 4;
    u->near_i = 0;
    memcpy(u->ref[0][0], near_i420, ys);
    memcpy(u->ref[0][1], near_i420 + ys, cs);
    memcpy(u->ref[0][2], near_i420 + ys + cs, cs);
    if (far_i420) {
        memcpy(u->ref[1][0], far_i420, ys);
        memcpy(u->ref[1][1], far_i420 + ys, cs);
        memcpy(u->ref[1][2], far_i420 + ys + cs, cs);
    }
    u->nref = far_i420 ? 2 : 1;
}

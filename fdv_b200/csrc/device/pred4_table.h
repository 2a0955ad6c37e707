// The nine 4x4 intra prediction modes (fdv_intra_predict_4x4, fdv.h:3720-3800)
// as one table.  Every predicted sample is one of four forms over a vector of
// neighbours
//     N = L(3) L(2) L(1) L(0) T(-1) T(0) .. T(7) DC
// (T(-1) = L(-1) = the corner; T(4..7) already replaced by T(3) when the
// above-right samples are unavailable; DC the mode-0 value):
//     copy     N[i0]
//     mean2    (N[i0] + N[i1] + 1) >> 1
//     tap121   (N[i0] + 2 N[i1] + N[i2] + 2) >> 2
//     tap13    (N[i0] + 3 N[i1] + 2) >> 2
// so that lanes predicting different modes run the same instructions.  The
// table is built at compile time from the same case analysis as pred4_px
// (intra.cuh), which it must equal sample for sample.
#pragma once
#include <cstdint>

namespace fdvb {

enum { P4_COPY = 0, P4_MEAN2 = 1, P4_TAP121 = 2, P4_TAP13 = 3 };

// Packed entry: i0 | i1 << 4 | i2 << 8 | form << 12.
struct P4Tab {
    uint16_t op[9 * 16];
};

__host__ __device__ constexpr int p4_t(int i) { return 5 + i; }   // T(i), i = -1..7
__host__ __device__ constexpr int p4_l(int i) { return 3 - i; }   // L(i), i = -1..3
__host__ __device__ constexpr uint16_t p4_pack(int form, int i0, int i1 = 0, int i2 = 0) {
    return (uint16_t)(i0 | (i1 << 4) | (i2 << 8) | (form << 12));
}

__host__ __device__ constexpr uint16_t p4_entry(int m, int x, int y) {
    switch (m) {
    case 1: return p4_pack(P4_COPY, p4_t(x));
    case 2: return p4_pack(P4_COPY, p4_l(y));
    case 3:
        if (x == 3 && y == 3) return p4_pack(P4_TAP13, p4_t(6), p4_t(7));
        return p4_pack(P4_TAP121, p4_t(x + y), p4_t(x + y + 1), p4_t(x + y + 2));
    case 4:
        if (x > y) return p4_pack(P4_TAP121, p4_t(x - y - 2), p4_t(x - y - 1), p4_t(x - y));
        if (x < y) return p4_pack(P4_TAP121, p4_l(y - x - 2), p4_l(y - x - 1), p4_l(y - x));
        return p4_pack(P4_TAP121, p4_t(0), p4_t(-1), p4_l(0));
    case 5: {
        const int z = 2 * x - y, k = x - (y >> 1);
        if (z >= 0 && !(z & 1)) return p4_pack(P4_MEAN2, p4_t(k - 1), p4_t(k));
        if (z >= 0) return p4_pack(P4_TAP121, p4_t(k - 2), p4_t(k - 1), p4_t(k));
        if (z == -1) return p4_pack(P4_TAP121, p4_l(0), p4_t(-1), p4_t(0));
        return p4_pack(P4_TAP121, p4_l(y - 1), p4_l(y - 2), p4_l(y - 3));
    }
    case 6: {
        const int z = 2 * y - x, k = y - (x >> 1);
        if (z >= 0 && !(z & 1)) return p4_pack(P4_MEAN2, p4_l(k - 1), p4_l(k));
        if (z >= 0) return p4_pack(P4_TAP121, p4_l(k - 2), p4_l(k - 1), p4_l(k));
        if (z == -1) return p4_pack(P4_TAP121, p4_t(0), p4_t(-1), p4_l(0));
        return p4_pack(P4_TAP121, p4_t(x - 1), p4_t(x - 2), p4_t(x - 3));
    }
    case 7: {
        const int k = x + (y >> 1);
        if (!(y & 1)) return p4_pack(P4_MEAN2, p4_t(k), p4_t(k + 1));
        return p4_pack(P4_TAP121, p4_t(k), p4_t(k + 1), p4_t(k + 2));
    }
    case 8: {
        const int z = x + 2 * y, k = y + (x >> 1);
        if (z < 5 && !(z & 1)) return p4_pack(P4_MEAN2, p4_l(k), p4_l(k + 1));
        if (z < 5) return p4_pack(P4_TAP121, p4_l(k), p4_l(k + 1), p4_l(k + 2));
        if (z == 5) return p4_pack(P4_TAP13, p4_l(2), p4_l(3));
        return p4_pack(P4_COPY, p4_l(3));
    }
    default: return p4_pack(P4_COPY, 13);   // DC
    }
}

__host__ __device__ constexpr P4Tab make_p4tab() {
    P4Tab t{};
    for (int m = 0; m < 9; ++m)
        for (int y = 0; y < 4; ++y)
            for (int x = 0; x < 4; ++x) t.op[m * 16 + y * 4 + x] = p4_entry(m, x, y);
    return t;
}

// One predicted sample from its packed entry: (a + f b + wc c + s) >> s with
// the form's weights copy (f 0, wc 0, s 0), mean2 (1, 0, 1), tap121 (2, 1, 2),
// tap13 (3, 0, 2) -- arithmetic in the form f, so that lanes evaluating
// different forms take no divergent branch.
__host__ __device__ __forceinline__ int p4_eval(unsigned op, const int *N) {
    const int f = (int)(op >> 12);
    const int a = N[op & 15], b = N[(op >> 4) & 15], c = N[(op >> 8) & 15];
    const int wc = (f >> 1) & ~f & 1, s = f - ((f >> 1) & f & 1);
    return (a + f * b + wc * c + s) >> s;
}

// The DC value (pred4_px's default case) from Tn = T(-1..7), Ln = L(-1..3).
__host__ __device__ __forceinline__ int p4_dc(const int *Tn, const int *Ln, int ht, int hl) {
    int s = 0;
    if (ht && hl) {
        for (int k = 0; k < 4; ++k) s += Tn[k + 1] + Ln[k + 1];
        return (s + 4) >> 3;
    }
    if (ht) {
        for (int k = 0; k < 4; ++k) s += Tn[k + 1];
        return (s + 2) >> 2;
    }
    if (hl) {
        for (int k = 0; k < 4; ++k) s += Ln[k + 1];
        return (s + 2) >> 2;
    }
    return 128;
}

}  // namespace fdvb

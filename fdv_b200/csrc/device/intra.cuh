// Intra prediction on the GPU: the n x n DC / V / H / PLANE predictors
// (fdv.h:2827-2910), the nine 4x4 directions (fdv.h:2698-2825) and the 4x4
// Hadamard SATD used to screen them (fdv.h:3803-3823).
#pragma once
#include "common.cuh"

namespace fdvb {

__device__ __forceinline__ bool nn_mode_ok(int m, int n, int ht, int hl) {
    switch (m) {
    case 0: return true;
    case 1: return ht;
    case 2: return hl;
    case 3: return ht && hl && (n == 8 || n == 16 || n == 32);
    }
    return false;
}

// Parameters of one n x n prediction, set up by one thread.
struct NNPred {
    int kind;     // 0 = flat (dc), 1 = vertical, 2 = horizontal, 3 = plane
    int dc, a, b, c, c0;
};
__device__ inline NNPred nn_setup(int mode, const uint8_t *top, const uint8_t *left, int tl, int n, int ht, int hl) {
    NNPred P = {0, 0, 0, 0, 0, 0};
    if (mode == 3 && nn_mode_ok(3, n, ht, hl)) {
        int half = n / 2, H = 0, V = 0;
        for (int k = 1; k <= half; ++k) {
            int t0 = (half - 1 - k) < 0 ? tl : top[half - 1 - k];
            int l0 = (half - 1 - k) < 0 ? tl : left[half - 1 - k];
            H += k * (top[half - 1 + k] - t0);
            V += k * (left[half - 1 + k] - l0);
        }
        P.kind = 3;
        P.a = 16 * (left[n - 1] + top[n - 1]);
        if (n == 32) { P.b = (11 * H + 512) >> 10; P.c = (11 * V + 512) >> 10; }
        else if (n == 16) { P.b = (5 * H + 32) >> 6; P.c = (5 * V + 32) >> 6; }
        else { P.b = (17 * H + 16) >> 5; P.c = (17 * V + 16) >> 5; }
        P.c0 = half - 1;
    } else if (mode == 1 && ht) {
        P.kind = 1;
    } else if (mode == 2 && hl) {
        P.kind = 2;
    } else {
        int s = 0;
        if (ht && hl) { for (int k = 0; k < n; ++k) s += top[k] + left[k]; P.dc = (s + n) / (2 * n); }
        else if (ht) { for (int k = 0; k < n; ++k) s += top[k]; P.dc = (s + n / 2) / n; }
        else if (hl) { for (int k = 0; k < n; ++k) s += left[k]; P.dc = (s + n / 2) / n; }
        else P.dc = 128;
    }
    return P;
}
// Sample (x, y) of the prediction.  Lanes of a warp may hold different kinds
// (one mode per half-warp in the screens), so the kinds' values are all
// formed and one is selected arithmetically: a switch on the kind would
// branch divergently on every sample.
__device__ __forceinline__ int nn_px(const NNPred &P, const uint8_t *top, const uint8_t *left, int x, int y) {
    const int k = P.kind;
    const int pl = clipb((P.a + P.c * (y - P.c0) + 16 + P.b * (x - P.c0)) >> 5);
    int v = P.dc;
    v += ((int)top[x] - v) & -(int)(k == 1);
    v += ((int)left[y] - v) & -(int)(k == 2);
    v += (pl - v) & -(int)(k == 3);
    return v;
}

// 4x4 directional prediction of pixel (x, y) from Tn = T(-1..7) and
// Ln = L(-1..3), T(-1) = L(-1) = the corner.
__device__ inline int pred4_px(int mode, const int *Tn, const int *Ln, int ht, int hl, int x, int y) {
#define T(i) Tn[(i) + 1]
#define L(i) Ln[(i) + 1]
    switch (mode) {
    case 1: return T(x);
    case 2: return L(y);
    case 3: return (x == 3 && y == 3) ? (T(6) + 3 * T(7) + 2) >> 2 : (T(x + y) + 2 * T(x + y + 1) + T(x + y + 2) + 2) >> 2;
    case 4:
        if (x > y) return (T(x - y - 2) + 2 * T(x - y - 1) + T(x - y) + 2) >> 2;
        if (x < y) return (L(y - x - 2) + 2 * L(y - x - 1) + L(y - x) + 2) >> 2;
        return (T(0) + 2 * T(-1) + L(0) + 2) >> 2;
    case 5: {
        int z = 2 * x - y;
        if (z >= 0 && !(z & 1)) return (T(x - (y >> 1) - 1) + T(x - (y >> 1)) + 1) >> 1;
        if (z >= 0) return (T(x - (y >> 1) - 2) + 2 * T(x - (y >> 1) - 1) + T(x - (y >> 1)) + 2) >> 2;
        if (z == -1) return (L(0) + 2 * T(-1) + T(0) + 2) >> 2;
        return (L(y - 1) + 2 * L(y - 2) + L(y - 3) + 2) >> 2;
    }
    case 6: {
        int z = 2 * y - x;
        if (z >= 0 && !(z & 1)) return (L(y - (x >> 1) - 1) + L(y - (x >> 1)) + 1) >> 1;
        if (z >= 0) return (L(y - (x >> 1) - 2) + 2 * L(y - (x >> 1) - 1) + L(y - (x >> 1)) + 2) >> 2;
        if (z == -1) return (T(0) + 2 * T(-1) + L(0) + 2) >> 2;
        return (T(x - 1) + 2 * T(x - 2) + T(x - 3) + 2) >> 2;
    }
    case 7:
        return !(y & 1) ? (T(x + (y >> 1)) + T(x + (y >> 1) + 1) + 1) >> 1
                        : (T(x + (y >> 1)) + 2 * T(x + (y >> 1) + 1) + T(x + (y >> 1) + 2) + 2) >> 2;
    case 8: {
        int z = x + 2 * y;
        if (z < 5 && !(z & 1)) return (L(y + (x >> 1)) + L(y + (x >> 1) + 1) + 1) >> 1;
        if (z < 5) return (L(y + (x >> 1)) + 2 * L(y + (x >> 1) + 1) + L(y + (x >> 1) + 2) + 2) >> 2;
        if (z == 5) return (L(2) + 3 * L(3) + 2) >> 2;
        return L(3);
    }
    default: {
        int s = 0;
        if (ht && hl) { for (int k = 0; k < 4; ++k) s += T(k) + L(k); return (s + 4) >> 3; }
        if (ht) { for (int k = 0; k < 4; ++k) s += T(k); return (s + 2) >> 2; }
        if (hl) { for (int k = 0; k < 4; ++k) s += L(k); return (s + 2) >> 2; }
        return 128;
    }
    }
#undef T
#undef L
}

// SATD of one 4x4 block on one thread: cur stride cs, pred stride ps.
__device__ inline int satd4(const uint8_t *cur, int cs, const uint8_t *pred, int ps) {
    int d[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) d[i * 4 + j] = (int)cur[i * cs + j] - (int)pred[i * ps + j];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int a0 = d[i * 4 + 0] + d[i * 4 + 1], a1 = d[i * 4 + 0] - d[i * 4 + 1];
        int a2 = d[i * 4 + 2] + d[i * 4 + 3], a3 = d[i * 4 + 2] - d[i * 4 + 3];
        d[i * 4 + 0] = a0 + a2; d[i * 4 + 1] = a1 + a3; d[i * 4 + 2] = a0 - a2; d[i * 4 + 3] = a1 - a3;
    }
    int sum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int a0 = d[j] + d[4 + j], a1 = d[j] - d[4 + j], a2 = d[8 + j] + d[12 + j], a3 = d[8 + j] - d[12 + j];
        sum += abs(a0 + a2) + abs(a1 + a3) + abs(a0 - a2) + abs(a1 - a3);
    }
    return sum;
}

}  // namespace fdvb

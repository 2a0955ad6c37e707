// Motion compensation and motion search on the GPU.
//
// Every reference frame is prepared once per frame (refprep.cu) into its
// integer plane G and the H.264 half-pel planes b, h, j, all border-padded.
// A quarter-pel sample is then one of those planes, or the rounded mean of
// two, exactly as the reference's per-phase blend table (fdv.h:3107-3229,
// equal by construction to interp_sample fdv.h:2970-2990).
#pragma once
#include "common.cuh"

namespace fdvb {

__device__ __forceinline__ int mc_px(const RefPlanes &R, int x, int y, int ph) {
    const long s = R.ys;
    const long o = (long)y * s + x;
    switch (ph) {
    case 0: return R.G[o];
    case 1: return (R.G[o] + R.B[o] + 1) >> 1;
    case 2: return R.B[o];
    case 3: return (R.B[o] + R.G[o + 1] + 1) >> 1;
    case 4: return (R.G[o] + R.H[o] + 1) >> 1;
    case 5: return (R.B[o] + R.H[o] + 1) >> 1;
    case 6: return (R.B[o] + R.J[o] + 1) >> 1;
    case 7: return (R.B[o] + R.H[o + 1] + 1) >> 1;
    case 8: return R.H[o];
    case 9: return (R.H[o] + R.J[o] + 1) >> 1;
    case 10: return R.J[o];
    case 11: return (R.J[o] + R.H[o + 1] + 1) >> 1;
    case 12: return (R.H[o] + R.G[o + s] + 1) >> 1;
    case 13: return (R.H[o] + R.B[o + s] + 1) >> 1;
    case 14: return (R.J[o] + R.B[o + s] + 1) >> 1;
    default: return (R.H[o + 1] + R.B[o + s] + 1) >> 1;
    }
}

// Bilinear chroma sample (fdv.h:3272-3282): quarter-pel chroma vector.
__device__ __forceinline__ int mc_cpx(const uint8_t *P, int s, int x, int y, int fx, int fy) {
    const uint8_t *p = P + (long)y * s + x;
    int a = p[0], b = p[1], c = p[s], d = p[s + 1];
    int top = a * (4 - fx) + b * fx, bot = c * (4 - fx) + d * fx;
    return (top * (4 - fy) + bot * fy + 8) >> 4;
}

// SAD of a bw x bh block of `cur` (stride cs) against the reference at
// quarter-pel vector (mvx, mvy), one warp, result in every lane.
__device__ __forceinline__ int warp_sad(const uint8_t *cur, int cs, const RefPlanes &R, int bx, int by,
                                        int bw, int bh, int mvx, int mvy, int lane) {
    const int ph = (mvy & 3) * 4 + (mvx & 3), ix = bx + (mvx >> 2), iy = by + (mvy >> 2);
    const int npx = bw * bh, sh = bw == 16 ? 4 : 3;
    int s = 0;
    if (ph == 0) {
        for (int p = lane; p < npx; p += 32) {
            int i = p >> sh, j = p & (bw - 1);
            s += abs((int)cur[i * cs + j] - (int)R.G[(long)(iy + i) * R.ys + ix + j]);
        }
    } else {
        for (int p = lane; p < npx; p += 32) {
            int i = p >> sh, j = p & (bw - 1);
            s += abs((int)cur[i * cs + j] - mc_px(R, ix + j, iy + i, ph));
        }
    }
    return __reduce_add_sync(FDVB_FULL, s);
}

// The reference's motion search (fdv.h:3375-3466) for one block, run by the
// whole thread block: zero vector, EPZS seed, large diamond (<= 64
// iterations, first strict improvement in pattern order), one small diamond,
// then half- and quarter-pel crosses.  The candidates of one step are scored
// in parallel, one warp each; the update is replayed in the reference's order
// by every thread on the shared scores, so all threads agree.
__device__ int me_search(const uint8_t *cur, int cs, const RefPlanes &R, int bx, int by, int bw, int bh,
                         int range, int pmx, int pmy, int *mvx, int *mvy, int *s_sad) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int LD[8][2] = {{0, 8}, {0, -8}, {8, 0}, {-8, 0}, {4, 4}, {4, -4}, {-4, 4}, {-4, -4}};
    const int SD[4][2] = {{0, 4}, {0, -4}, {4, 0}, {-4, 0}};
    const int SP[4][2] = {{0, -1}, {0, 1}, {-1, 0}, {1, 0}};
    const int lim = range * 4;
    int px = (pmx >> 2) * 4, py = (pmy >> 2) * 4;
    px = px < -lim ? -lim : (px > lim ? lim : px);
    py = py < -lim ? -lim : (py > lim ? lim : py);
    const bool seed = px != 0 || py != 0;
    if (warp == 0) { int v = warp_sad(cur, cs, R, bx, by, bw, bh, 0, 0, lane); if (lane == 0) s_sad[0] = v; }
    if (warp == 1 && seed) { int v = warp_sad(cur, cs, R, bx, by, bw, bh, px, py, lane); if (lane == 0) s_sad[1] = v; }
    __syncthreads();
    int best = s_sad[0], bx_ = 0, by_ = 0;
    if (seed && s_sad[1] < best) { best = s_sad[1]; bx_ = px; by_ = py; }
    __syncthreads();
    for (int it = 0; it < 64; ++it) {
        const int cx = bx_, cy = by_;
        {
            int nx = cx + LD[warp][0], ny = cy + LD[warp][1];
            bool in = !(nx < -lim || nx > lim || ny < -lim || ny > lim);
            if (in) { int v = warp_sad(cur, cs, R, bx, by, bw, bh, nx, ny, lane); if (lane == 0) s_sad[warp] = v; }
        }
        __syncthreads();
        bool moved = false;
        for (int k = 0; k < 8; ++k) {
            int nx = cx + LD[k][0], ny = cy + LD[k][1];
            if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
            int s = s_sad[k];
            if (s < best) { best = s; bx_ = nx; by_ = ny; moved = true; }
        }
        __syncthreads();
        if (!moved) break;
    }
    {
        const int cx = bx_, cy = by_;
        if (warp < 4) {
            int nx = cx + SD[warp][0], ny = cy + SD[warp][1];
            bool in = !(nx < -lim || nx > lim || ny < -lim || ny > lim);
            if (in) { int v = warp_sad(cur, cs, R, bx, by, bw, bh, nx, ny, lane); if (lane == 0) s_sad[warp] = v; }
        }
        __syncthreads();
        for (int k = 0; k < 4; ++k) {
            int nx = cx + SD[k][0], ny = cy + SD[k][1];
            if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
            int s = s_sad[k];
            if (s < best) { best = s; bx_ = nx; by_ = ny; }
        }
        __syncthreads();
    }
    for (int step = 2; step >= 1 && best > 0; step >>= 1) {
        const int cx = bx_, cy = by_;
        if (warp < 4) {
            int v = warp_sad(cur, cs, R, bx, by, bw, bh, cx + SP[warp][0] * step, cy + SP[warp][1] * step, lane);
            if (lane == 0) s_sad[warp] = v;
        }
        __syncthreads();
        for (int k = 0; k < 4; ++k) {
            int s = s_sad[k];
            if (s < best) { best = s; bx_ = cx + SP[k][0] * step; by_ = cy + SP[k][1] * step; }
        }
        __syncthreads();
    }
    *mvx = bx_;
    *mvy = by_;
    return best;
}

// ------------------------------------------------ packed-byte versions --
// Four consecutive plane bytes from any alignment: two aligned loads and a
// funnel shift (plane rows and the (0,0) origin are 16-byte aligned).
__device__ __forceinline__ uint32_t ld4u(const uint8_t *p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    return __funnelshift_r(q[0], q[1], (unsigned)(a & 3) * 8u);
}
// Four motion-compensated luma samples at integer base (x, y), phase ph: one
// plane, or the per-byte rounded mean (a + b + 1) >> 1 of two (__vavgu4).
__device__ __forceinline__ uint32_t mc_word(const RefPlanes &R, int x, int y, int ph) {
    const long s = R.ys, o = (long)y * s + x;
    switch (ph) {
    case 0: return ld4u(R.G + o);
    case 1: return __vavgu4(ld4u(R.G + o), ld4u(R.B + o));
    case 2: return ld4u(R.B + o);
    case 3: return __vavgu4(ld4u(R.B + o), ld4u(R.G + o + 1));
    case 4: return __vavgu4(ld4u(R.G + o), ld4u(R.H + o));
    case 5: return __vavgu4(ld4u(R.B + o), ld4u(R.H + o));
    case 6: return __vavgu4(ld4u(R.B + o), ld4u(R.J + o));
    case 7: return __vavgu4(ld4u(R.B + o), ld4u(R.H + o + 1));
    case 8: return ld4u(R.H + o);
    case 9: return __vavgu4(ld4u(R.H + o), ld4u(R.J + o));
    case 10: return ld4u(R.J + o);
    case 11: return __vavgu4(ld4u(R.J + o), ld4u(R.H + o + 1));
    case 12: return __vavgu4(ld4u(R.H + o), ld4u(R.G + o + s));
    case 13: return __vavgu4(ld4u(R.H + o), ld4u(R.B + o + s));
    case 14: return __vavgu4(ld4u(R.J + o), ld4u(R.B + o + s));
    default: return __vavgu4(ld4u(R.H + o + 1), ld4u(R.B + o + s));
    }
}

__device__ __forceinline__ void gbar(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// Candidate vectors of one search step (fdv.h:3382-3391).
__constant__ int c_LD[8][2] = {{0, 8}, {0, -8}, {8, 0}, {-8, 0}, {4, 4}, {4, -4}, {-4, 4}, {-4, -4}};
__constant__ int c_SD[4][2] = {{0, 4}, {0, -4}, {4, 0}, {-4, 0}};
__constant__ int c_SP[4][2] = {{0, -1}, {0, 1}, {-1, 0}, {1, 0}};

// SAD of the BS x BS block whose source words this lane holds (c0, c1),
// against the reference at (mvx, mvy).  BS = 16: the warp covers the block
// (lane -> row lane/2, 8 bytes); BS = 8: each half-warp covers one block
// (lane -> row (lane&15)/2, 4 bytes) and the result is per half.
template <int BS>
__device__ __forceinline__ int sad_packed(uint32_t c0, uint32_t c1, const RefPlanes &R, int bx, int by,
                                          int mvx, int mvy, int lane) {
    const int ph = (mvy & 3) * 4 + (mvx & 3);
    if (BS == 16) {
        const int row = lane >> 1, half = lane & 1;
        const int x = bx + (mvx >> 2) + half * 8, y = by + (mvy >> 2) + row;
        int v = __vsadu4(c0, mc_word(R, x, y, ph)) + __vsadu4(c1, mc_word(R, x + 4, y, ph));
        return __reduce_add_sync(FDVB_FULL, v);
    } else {
        const int l = lane & 15, row = l >> 1, half = l & 1;
        const int x = bx + (mvx >> 2) + half * 4, y = by + (mvy >> 2) + row;
        int v = __vsadu4(c0, mc_word(R, x, y, ph));
        v += __shfl_xor_sync(FDVB_FULL, v, 8);
        v += __shfl_xor_sync(FDVB_FULL, v, 4);
        v += __shfl_xor_sync(FDVB_FULL, v, 2);
        v += __shfl_xor_sync(FDVB_FULL, v, 1);
        return v;
    }
}

// The reference's motion search (fdv.h:3375-3466) run by one group of four
// warps (128 threads, named barrier `bar`): zero vector and EPZS seed, large
// diamond (<= 64 iterations, first strict improvement in pattern order), one
// small diamond, half- then quarter-pel crosses.  Each step's candidates are
// scored concurrently (16x16: two per warp; 8x8: one per half-warp); every
// thread of the group replays the update in the reference's order on the
// shared scores.  `cur` is the block's source (stride 16).
template <int BS>
__device__ int me_search_group(const uint8_t *cur, const RefPlanes &R, int bx, int by, int range, int pmx, int pmy,
                               int *mvx, int *mvy, int *s_sad, int gw, int lane, int bar) {
    const int lim = range * 4;
    uint32_t c0, c1 = 0;
    if (BS == 16) {
        const uint32_t *cw = reinterpret_cast<const uint32_t *>(cur + (lane >> 1) * 16 + (lane & 1) * 8);
        c0 = cw[0]; c1 = cw[1];
    } else {
        const int l = lane & 15;
        c0 = *reinterpret_cast<const uint32_t *>(cur + (l >> 1) * 16 + (l & 1) * 4);
    }
    // candidate k of the group's current step: warp gw scores k = gw, gw+4 (16x16)
    // or k = 2*gw + half (8x8)
    int px = (pmx >> 2) * 4, py = (pmy >> 2) * 4;
    px = px < -lim ? -lim : (px > lim ? lim : px);
    py = py < -lim ? -lim : (py > lim ? lim : py);
    const bool seed = px != 0 || py != 0;
    {   // step 0: the zero vector (k = 0) and the seed (k = 1)
        if (BS == 16) {
            if (gw == 0) { int v = sad_packed<16>(c0, c1, R, bx, by, 0, 0, lane); if (lane == 0) s_sad[0] = v; }
            if (gw == 1 && seed) { int v = sad_packed<16>(c0, c1, R, bx, by, px, py, lane); if (lane == 0) s_sad[1] = v; }
        } else if (gw == 0) {
            const int hk = lane >> 4;
            int v = sad_packed<8>(c0, c1, R, bx, by, hk ? px : 0, hk ? py : 0, lane);
            if ((lane & 15) == 0 && (hk == 0 || seed)) s_sad[hk] = v;
        }
        gbar(bar, 128);
    }
    int best = s_sad[0], bxv = 0, byv = 0;
    if (seed && s_sad[1] < best) { best = s_sad[1]; bxv = px; byv = py; }
    gbar(bar, 128);
    for (int it = 0; it < 64; ++it) {
        const int cx = bxv, cy = byv;
        if (BS == 16) {
            for (int k = gw; k < 8; k += 4) {
                const int nx = cx + c_LD[k][0], ny = cy + c_LD[k][1];
                if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
                int v = sad_packed<16>(c0, c1, R, bx, by, nx, ny, lane);
                if (lane == 0) s_sad[k] = v;
            }
        } else {
            const int k = 2 * gw + (lane >> 4);
            const int nx = cx + c_LD[k][0], ny = cy + c_LD[k][1];
            const bool in = !(nx < -lim || nx > lim || ny < -lim || ny > lim);
            int v = sad_packed<8>(c0, c1, R, bx, by, in ? nx : cx, in ? ny : cy, lane);
            if ((lane & 15) == 0 && in) s_sad[k] = v;
        }
        gbar(bar, 128);
        bool moved = false;
        for (int k = 0; k < 8; ++k) {
            const int nx = cx + c_LD[k][0], ny = cy + c_LD[k][1];
            if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
            const int sv = s_sad[k];
            if (sv < best) { best = sv; bxv = nx; byv = ny; moved = true; }
        }
        gbar(bar, 128);
        if (!moved) break;
    }
    {   // one small diamond
        const int cx = bxv, cy = byv;
        if (BS == 16) {
            const int k = gw;
            const int nx = cx + c_SD[k][0], ny = cy + c_SD[k][1];
            if (!(nx < -lim || nx > lim || ny < -lim || ny > lim)) {
                int v = sad_packed<16>(c0, c1, R, bx, by, nx, ny, lane);
                if (lane == 0) s_sad[k] = v;
            }
        } else if (gw < 2) {
            const int k = 2 * gw + (lane >> 4);
            const int nx = cx + c_SD[k][0], ny = cy + c_SD[k][1];
            const bool in = !(nx < -lim || nx > lim || ny < -lim || ny > lim);
            int v = sad_packed<8>(c0, c1, R, bx, by, in ? nx : cx, in ? ny : cy, lane);
            if ((lane & 15) == 0 && in) s_sad[k] = v;
        }
        gbar(bar, 128);
        for (int k = 0; k < 4; ++k) {
            const int nx = cx + c_SD[k][0], ny = cy + c_SD[k][1];
            if (nx < -lim || nx > lim || ny < -lim || ny > lim) continue;
            const int sv = s_sad[k];
            if (sv < best) { best = sv; bxv = nx; byv = ny; }
        }
        gbar(bar, 128);
    }
    for (int step = 2; step >= 1 && best > 0; step >>= 1) {   // half-, then quarter-pel cross
        const int cx = bxv, cy = byv;
        if (BS == 16) {
            const int k = gw;
            int v = sad_packed<16>(c0, c1, R, bx, by, cx + c_SP[k][0] * step, cy + c_SP[k][1] * step, lane);
            if (lane == 0) s_sad[k] = v;
        } else if (gw < 2) {
            const int k = 2 * gw + (lane >> 4);
            int v = sad_packed<8>(c0, c1, R, bx, by, cx + c_SP[k][0] * step, cy + c_SP[k][1] * step, lane);
            if ((lane & 15) == 0) s_sad[k] = v;
        }
        gbar(bar, 128);
        for (int k = 0; k < 4; ++k) {
            const int sv = s_sad[k];
            if (sv < best) { best = sv; bxv = cx + c_SP[k][0] * step; byv = cy + c_SP[k][1] * step; }
        }
        gbar(bar, 128);
    }
    *mvx = bxv;
    *mvy = byv;
    return best;
}

}  // namespace fdvb

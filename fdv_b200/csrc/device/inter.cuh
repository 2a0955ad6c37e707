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

// Bilinear chroma sample (fdv.h:3272-3282): quarter-pel chroma vector.
__device__ __forceinline__ int mc_cpx(const uint8_t *P, int s, int x, int y, int fx, int fy) {
    const uint8_t *p = P + (long)y * s + x;
    int a = p[0], b = p[1], c = p[s], d = p[s + 1];
    int top = a * (4 - fx) + b * fx, bot = c * (4 - fx) + d * fx;
    return (top * (4 - fy) + bot * fy + 8) >> 4;
}

// ------------------------------------------------ packed-byte versions --
// Four consecutive plane bytes from any alignment: two aligned loads and a
// funnel shift (plane rows and the (0,0) origin are 16-byte aligned).
__device__ __forceinline__ uint32_t ld4u(const uint8_t *p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    return __funnelshift_r(q[0], q[1], (unsigned)(a & 3) * 8u);
}

// The same loads through L2 only (ld.global.cg), for reference planes that
// other blocks of the same launch write (post.cuh): an L1 line filled by an
// earlier read could hold bytes of a tile written after it.
__device__ __forceinline__ int mc_cpx_cg(const uint8_t *P, int s, int x, int y, int fx, int fy) {
    const uint8_t *p = P + (long)y * s + x;
    int a = __ldcg(p), b = __ldcg(p + 1), c = __ldcg(p + s), d = __ldcg(p + s + 1);
    int top = a * (4 - fx) + b * fx, bot = c * (4 - fx) + d * fx;
    return (top * (4 - fy) + bot * fy + 8) >> 4;
}
__device__ __forceinline__ uint32_t ld4u_cg(const uint8_t *p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    return __funnelshift_r(__ldcg(q), __ldcg(q + 1), (unsigned)(a & 3) * 8u);
}

// Where a reference's four luma planes (0 = G, 1 = b, 2 = h, 3 = j) are read
// from: the padded planes in global memory ...
struct GlobalLuma {
    const uint8_t *G, *B, *H, *J;
    int ys;
    __device__ explicit GlobalLuma(const RefPlanes &R) : G(R.G), B(R.B), H(R.H), J(R.J), ys(R.ys) {}
    __device__ __forceinline__ uint32_t ld(int p, int x, int y) const {
        const uint8_t *pl = p == 0 ? G : (p == 1 ? B : (p == 2 ? H : J));
        return ld4u(pl + (long)y * ys + x);
    }
};
// ... the same through L2 only ...
struct GlobalLumaCG {
    const uint8_t *G, *B, *H, *J;
    int ys;
    __device__ explicit GlobalLumaCG(const RefPlanes &R) : G(R.G), B(R.B), H(R.H), J(R.J), ys(R.ys) {}
    __device__ __forceinline__ uint32_t ld(int p, int x, int y) const {
        const uint8_t *pl = p == 0 ? G : (p == 1 ? B : (p == 2 ? H : J));
        return ld4u_cg(pl + (long)y * ys + x);
    }
};
// ... or a window of them staged in shared memory by the P-frame kernel: per
// plane kWinRows rows of a ring of kWinRing columns (column x at x mod
// kWinRing), rows kWinStride bytes apart.  Row indices are clamped to the
// window, so no read leaves it whatever the vector.
constexpr int kWinRing = 128, kWinStride = 144, kWinRows = 88, kWinPlane = kWinRows * kWinStride;
struct WindowLuma {
    const uint8_t *base;      // plane p at base + p * kWinPlane
    int y0, rmax;             // plane row of window row 0; last window row
    __device__ __forceinline__ uint32_t ld(int p, int x, int y) const {
        int r = y - y0;
        r = r < 0 ? 0 : (r > rmax ? rmax : r);
        const uint8_t *row = base + p * kWinPlane + r * kWinStride;
        const int xa = x & ~3;
        const uint32_t a = *reinterpret_cast<const uint32_t *>(row + (xa & (kWinRing - 1)));
        const uint32_t b = *reinterpret_cast<const uint32_t *>(row + ((xa + 4) & (kWinRing - 1)));
        return __funnelshift_r(a, b, (unsigned)(x & 3) * 8u);
    }
};

// Four motion-compensated luma samples at integer base (x, y), phase ph: one
// plane, or the per-byte rounded mean (a + b + 1) >> 1 of two (__vavgu4).
template <class Src>
__device__ __forceinline__ uint32_t mc_word(const Src &R, int x, int y, int ph) {
    switch (ph) {
    case 0: return R.ld(0, x, y);
    case 1: return __vavgu4(R.ld(0, x, y), R.ld(1, x, y));
    case 2: return R.ld(1, x, y);
    case 3: return __vavgu4(R.ld(1, x, y), R.ld(0, x + 1, y));
    case 4: return __vavgu4(R.ld(0, x, y), R.ld(2, x, y));
    case 5: return __vavgu4(R.ld(1, x, y), R.ld(2, x, y));
    case 6: return __vavgu4(R.ld(1, x, y), R.ld(3, x, y));
    case 7: return __vavgu4(R.ld(1, x, y), R.ld(2, x + 1, y));
    case 8: return R.ld(2, x, y);
    case 9: return __vavgu4(R.ld(2, x, y), R.ld(3, x, y));
    case 10: return R.ld(3, x, y);
    case 11: return __vavgu4(R.ld(3, x, y), R.ld(2, x + 1, y));
    case 12: return __vavgu4(R.ld(2, x, y), R.ld(0, x, y + 1));
    case 13: return __vavgu4(R.ld(2, x, y), R.ld(1, x, y + 1));
    case 14: return __vavgu4(R.ld(3, x, y), R.ld(1, x, y + 1));
    default: return __vavgu4(R.ld(2, x + 1, y), R.ld(1, x, y + 1));
    }
}

// The same sample without a branch on the phase: the planes and offsets of
// its one or two taps are read from immediates indexed by the phase.  Lanes
// of one warp may then take different phases at no cost.
template <class Src>
__device__ __forceinline__ uint32_t mc_word_nb(const Src &R, int x, int y, int ph) {
    constexpr unsigned long long kPA = 0x2322332211101100ull;   // nibble ph: plane of the first tap
    constexpr unsigned long long kPB = 0x1110233223220110ull;   // nibble ph: plane of the second tap
    constexpr unsigned kAV = 0xfafa;    // bit ph: two taps, rounded mean
    constexpr unsigned kADX = 0x8000;   // bit ph: first tap at x + 1
    constexpr unsigned kBDX = 0x0888;   // bit ph: second tap at x + 1
    constexpr unsigned kBDY = 0xf000;   // bit ph: second tap at y + 1
    const int pa = (int)((kPA >> (4 * ph)) & 3), pb = (int)((kPB >> (4 * ph)) & 3);
    const uint32_t a = R.ld(pa, x + (int)((kADX >> ph) & 1), y);
    const uint32_t b = R.ld(pb, x + (int)((kBDX >> ph) & 1), y + (int)((kBDY >> ph) & 1));
    return ((kAV >> ph) & 1) ? __vavgu4(a, b) : a;
}

__device__ __forceinline__ void gbar(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// Candidate vectors of one search step (fdv.h:3382-3391), as arithmetic so
// that lanes of one warp can take different candidates without a divergent
// table lookup: large diamond (0,8) (0,-8) (8,0) (-8,0) (4,4) (4,-4) (-4,4)
// (-4,-4); small diamond (0,4) (0,-4) (4,0) (-4,0); cross (0,-1) (0,1) (-1,0) (1,0).
// Each offset is a signed nibble of a packed constant, picked by a shift, so
// that lanes taking different candidates run the same instructions (nested
// conditionals on k compile to divergent branches).
__device__ __forceinline__ int nib(unsigned pack, int k) { return (int)(pack << (28 - 4 * k)) >> 28; }
__device__ __forceinline__ int ld_dx(int k) { return 4 * nib(0xFF11E200u, k); }   //  0  0  8 -8  4  4 -4 -4
__device__ __forceinline__ int ld_dy(int k) { return 4 * nib(0xF1F100E2u, k); }   //  8 -8  0  0  4 -4  4 -4
__device__ __forceinline__ int sd_dx(int k) { return 4 * nib(0xF100u, k); }       //  0  0  4 -4
__device__ __forceinline__ int sd_dy(int k) { return 4 * nib(0x00F1u, k); }       //  4 -4  0  0
__device__ __forceinline__ int sp_dx(int k) { return nib(0x1F00u, k); }           //  0  0 -1  1
__device__ __forceinline__ int sp_dy(int k) { return nib(0x001Fu, k); }           // -1  1  0  0

// SAD of the BS x BS block whose source words this lane holds (c0, c1),
// against the reference at (mvx, mvy).  BS = 16: the warp covers the block
// (lane -> row lane/2, 8 bytes); BS = 8: each half-warp covers one block
// (lane -> row (lane&15)/2, 4 bytes), the two halves may score different
// candidates (different phases), and the result is per half.
//
// INT: the vector is whole-pel (every step of the diamond walks and their
// starting points), so the samples are the integer plane's alone; the sub-pel
// crosses take any phase through the branch-free form.  Both keep the code of
// a step small: the walks' many inlined steps otherwise overflow the SM's
// instruction cache.
template <int BS, bool INT = false, class Src>
__device__ __forceinline__ int sad_packed(uint32_t c0, uint32_t c1, const Src &R, int bx, int by,
                                          int mvx, int mvy, int lane) {
    const int ph = (mvy & 3) * 4 + (mvx & 3);
    if (BS == 16) {
        const int row = lane >> 1, half = lane & 1;
        const int x = bx + (mvx >> 2) + half * 8, y = by + (mvy >> 2) + row;
        int v;
        if (INT) v = __vsadu4(c0, R.ld(0, x, y)) + __vsadu4(c1, R.ld(0, x + 4, y));
        else v = __vsadu4(c0, mc_word_nb(R, x, y, ph)) + __vsadu4(c1, mc_word_nb(R, x + 4, y, ph));
        return __reduce_add_sync(FDVB_FULL, v);
    } else {
        const int l = lane & 15, row = l >> 1, half = l & 1;
        const int x = bx + (mvx >> 2) + half * 4, y = by + (mvy >> 2) + row;
        const int v = __vsadu4(c0, INT ? R.ld(0, x, y) : mc_word_nb(R, x, y, ph));
        const int lo = __reduce_add_sync(FDVB_FULL, lane < 16 ? v : 0);
        const int hi = __reduce_add_sync(FDVB_FULL, lane < 16 ? 0 : v);
        return lane < 16 ? lo : hi;
    }
}

// The reference's motion search (fdv.h:3375-3466) run by one group of four
// warps (128 threads, named barrier `bar`): zero vector and EPZS seed, large
// diamond (<= 64 iterations, first strict improvement in pattern order), one
// small diamond, half- then quarter-pel crosses.  Each step's candidates are
// scored concurrently (16x16: two per warp; 8x8: one per half-warp); every
// thread of the group replays the update in the reference's order on the
// shared scores.  For 8x8 the scores alternate between two arrays, so a step
// needs one barrier: a step writes one array while the last reads of it were
// two steps ago.  `cur` is the block's source (stride 16); s_sad holds 16
// scores.
template <int BS, class Src>
__device__ int me_search_group(const uint8_t *cur, const Src &R, int bx, int by, int range, int pmx, int pmy,
                               int *mvx, int *mvy, int *s_sad, int gw, int lane, int bar,
                               unsigned long long *iters = nullptr, const short2 *cands = nullptr, int ncands = 0,
                               int max_ld = 64) {
    constexpr bool DB = BS == 8;
    const int lim = range * 4;
    uint32_t c0, c1 = 0;
    if (BS == 16) {
        const uint32_t *cw = reinterpret_cast<const uint32_t *>(cur + (lane >> 1) * 16 + (lane & 1) * 8);
        c0 = cw[0]; c1 = cw[1];
    } else {
        const int l = lane & 15;
        c0 = *reinterpret_cast<const uint32_t *>(cur + (l >> 1) * 16 + (l & 1) * 4);
    }
    int step_no = 0;
    auto scores = [&]() { return s_sad + (DB ? (step_no & 1) * 8 : 0); };
    auto end_step = [&]() { if (!DB) gbar(bar, 128); ++step_no; };
    auto inb = [&](int x, int y) { return !(x < -lim || x > lim || y < -lim || y > lim); };
    int px = (pmx >> 2) * 4, py = (pmy >> 2) * 4;
    px = px < -lim ? -lim : (px > lim ? lim : px);
    py = py < -lim ? -lim : (py > lim ? lim : py);
    const bool seed = px != 0 || py != 0;
    int best, bxv = 0, byv = 0;
    // extra starting points: whole-pel positions of the proposals
    auto cand_at = [&](int k, int &x, int &y) {
        x = (cands[k].x >> 2) * 4;
        y = (cands[k].y >> 2) * 4;
        x = x < -lim ? -lim : (x > lim ? lim : x);
        y = y < -lim ? -lim : (y > lim ? lim : y);
    };
    {   // the zero vector (k = 0), the seed (k = 1) and any proposals (k = 2..)
        int *s = scores();
        if (BS == 16) {
            if (gw == 0) { int v = sad_packed<16, true>(c0, c1, R, bx, by, 0, 0, lane); if (lane == 0) s[0] = v; }
            if (gw == 1 && seed) { int v = sad_packed<16, true>(c0, c1, R, bx, by, px, py, lane); if (lane == 0) s[1] = v; }
            for (int k = 2 + gw; k < 2 + ncands; k += 4) {
                int x, y;
                cand_at(k - 2, x, y);
                int v = sad_packed<16, true>(c0, c1, R, bx, by, x, y, lane);
                if (lane == 0) s[k] = v;
            }
        } else if (gw == 0) {
            const int hk = lane >> 4;
            int v = sad_packed<8, true>(c0, c1, R, bx, by, hk ? px : 0, hk ? py : 0, lane);
            if ((lane & 15) == 0 && (hk == 0 || seed)) s[hk] = v;
        } else if (gw <= 2 && ncands > 0) {
            // up to four proposals on the half-warps of warps 1 and 2
            const int ci = 2 * (gw - 1) + (lane >> 4);
            int x, y;
            cand_at(ci < ncands ? ci : 0, x, y);
            int v = sad_packed<8, true>(c0, c1, R, bx, by, x, y, lane);
            if ((lane & 15) == 0 && ci < ncands) s[2 + ci] = v;
        }
        gbar(bar, 128);
        best = s[0];
        if (seed && s[1] < best) { best = s[1]; bxv = px; byv = py; }
        for (int k = 0; k < ncands; ++k) {
            int x, y;
            cand_at(k, x, y);
            if (s[2 + k] < best) { best = s[2 + k]; bxv = x; byv = y; }
        }
        end_step();
    }
    for (int it = 0; it < max_ld; ++it) {   // large diamond
        const int cx = bxv, cy = byv;
        int *s = scores();
        if (BS == 16) {
            for (int k = gw; k < 8; k += 4) {
                const int nx = cx + ld_dx(k), ny = cy + ld_dy(k);
                if (!inb(nx, ny)) continue;
                int v = sad_packed<16, true>(c0, c1, R, bx, by, nx, ny, lane);
                if (lane == 0) s[k] = v;
            }
        } else {
            const int k = 2 * gw + (lane >> 4);
            const int nx = cx + ld_dx(k), ny = cy + ld_dy(k);
            const bool in = inb(nx, ny);
            int v = sad_packed<8, true>(c0, c1, R, bx, by, in ? nx : cx, in ? ny : cy, lane);
            if ((lane & 15) == 0 && in) s[k] = v;
        }
        gbar(bar, 128);
        bool moved = false;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int nx = cx + ld_dx(k), ny = cy + ld_dy(k);
            const int sv = s[k];
            if (inb(nx, ny) && sv < best) { best = sv; bxv = nx; byv = ny; moved = true; }
        }
        end_step();
        if (iters && gw == 0 && lane == 0) atomicAdd(iters, 1ull);
        if (!moved) break;
    }
    {   // one small diamond
        const int cx = bxv, cy = byv;
        int *s = scores();
        if (BS == 16) {
            const int k = gw, nx = cx + sd_dx(k), ny = cy + sd_dy(k);
            if (inb(nx, ny)) {
                int v = sad_packed<16, true>(c0, c1, R, bx, by, nx, ny, lane);
                if (lane == 0) s[k] = v;
            }
        } else if (gw < 2) {
            const int k = 2 * gw + (lane >> 4), nx = cx + sd_dx(k), ny = cy + sd_dy(k);
            const bool in = inb(nx, ny);
            int v = sad_packed<8, true>(c0, c1, R, bx, by, in ? nx : cx, in ? ny : cy, lane);
            if ((lane & 15) == 0 && in) s[k] = v;
        }
        gbar(bar, 128);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int nx = cx + sd_dx(k), ny = cy + sd_dy(k);
            const int sv = s[k];
            if (inb(nx, ny) && sv < best) { best = sv; bxv = nx; byv = ny; }
        }
        end_step();
    }
    for (int step = 2; step >= 1 && best > 0; step >>= 1) {   // half-, then quarter-pel cross
        const int cx = bxv, cy = byv;
        int *s = scores();
        if (BS == 16) {
            const int k = gw;
            int v = sad_packed<16>(c0, c1, R, bx, by, cx + sp_dx(k) * step, cy + sp_dy(k) * step, lane);
            if (lane == 0) s[k] = v;
        } else if (gw < 2) {
            const int k = 2 * gw + (lane >> 4);
            int v = sad_packed<8>(c0, c1, R, bx, by, cx + sp_dx(k) * step, cy + sp_dy(k) * step, lane);
            if ((lane & 15) == 0) s[k] = v;
        }
        gbar(bar, 128);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int sv = s[k];
            if (sv < best) { best = sv; bxv = cx + sp_dx(k) * step; byv = cy + sp_dy(k) * step; }
        }
        end_step();
    }
    if (DB) gbar(bar, 128);   // the caller may reuse s_sad
    *mvx = bxv;
    *mvy = byv;
    return best;
}

}  // namespace fdvb

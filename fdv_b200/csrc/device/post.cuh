// The P-frame wavefront's reference output ("post" stage): while a frame's
// macroblock rows pass, every finished 16x16 tile of its reconstruction is
// deblocked and turned into the next frame's reference planes -- the integer
// plane G and the half-pel planes b, h, j with their replicated borders,
// chroma with its border -- so that the next frame's wavefront can start
// before this one has ended (several frames in one launch).
//
// The deblocking (fdv.h:3491-3501, :3617-3625) filters every vertical 8x8-grid
// edge of a plane, then every horizontal one; a filter reads two samples and
// writes one on each side of its edge, and edges are 8 apart, so a deblocked
// sample is a function of the reconstruction within 2 samples across the
// nearest vertical edge, then 2 rows across the nearest horizontal edge.  That
// local stencil is evaluated here per tile from the un-deblocked
// reconstruction (which the frame's own analysis keeps reading for its intra
// neighbours), giving the same samples as the two whole-plane passes
// (deblock_v_kernel, deblock_h_kernel).  The reference planes follow from the
// deblocked samples exactly as refprep_luma_kernel / refprep_chroma_kernel
// make them: 6-tap filters over border-clamped samples (fdv.h:2932-2959,
// :1603-1624).  Beyond 3 samples outside the picture every plane is constant
// along the clamped direction (all six taps read the edge sample), so a
// tile's border part replicates its samples at -3 / w+2 (and -3 / h+2).
//
// Tile (tr, tc) needs the reconstruction of macroblocks tr-1..tr+1 x
// tc-1..tc+1 (rows 16tr-4 .. 16tr+20, the same columns).  The wavefront row
// below posts it one macroblock behind its own progress; the last row posts
// its own tiles.  Per macroblock row, a count of posted tiles is released at
// GPU scope after the tile's stores (a block barrier between them).
#pragma once
#include "common.cuh"
#include "engine_dev.cuh"

namespace fdvb {

// Threads 32..511 of the P-frame block run the post stage (warp 0 is in the
// wavefront wait meanwhile); named barrier 15 joins them.
constexpr int kPostT0 = 32, kPostNT = 480;
__device__ __forceinline__ void post_bar() { asm volatile("bar.sync 15, 480;" ::: "memory"); }

struct PostScratch {
    uint8_t rec[25][28];       // reconstruction, rows vy0.., columns rx0..
    uint8_t vp[25][24];        // after the vertical-edge pass, columns dx0..
    uint8_t d[21][24];         // deblocked, rows dy0.., columns dx0..
    int16_t hs[21][22];        // horizontal 6-tap sums, rows dy0.., core columns cx0..
    uint8_t core[4][22][24];   // G, b, h, j at the core samples (rows cy0.., columns cx0..)
    uint8_t crec[2][12][12];   // chroma reconstruction, rows cry0.., columns crx0..
    uint8_t cv[2][12][8];      // chroma after the vertical-edge pass, columns 8tc..
    uint8_t cd[2][8][8];       // deblocked chroma tile
};

// The deblocked value of the sample at a[0], position x on a line of n samples
// (a[k * step] the sample at x + k): the filter of the grid edge it touches,
// as filter_edge (frame_ops.cuh) applies it.
__device__ __forceinline__ int dbk_sample(const uint8_t *a, int step, int x, int n, int alpha, int beta, int tc) {
    int p1, p0, q0, q1;
    bool pside;
    if ((x & 7) == 7 && x + 1 < n) {
        p1 = a[-step]; p0 = a[0]; q0 = a[step]; q1 = a[2 * step]; pside = true;
    } else if ((x & 7) == 0 && x > 0) {
        p1 = a[-2 * step]; p0 = a[-step]; q0 = a[0]; q1 = a[step]; pside = false;
    } else {
        return a[0];
    }
    if (abs(p0 - q0) < alpha && abs(p1 - p0) < beta && abs(q1 - q0) < beta) {
        int d = ((q0 - p0) * 4 + (p1 - q1) + 4) >> 3;
        d = d < -tc ? -tc : (d > tc ? tc : d);
        return pside ? clipb(p0 + d) : clipb(q0 - d);
    }
    return a[0];
}

__device__ __forceinline__ int tap6i(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Tile (tr, tc) of frame U into its reference output; t = thread index within
// the post threads (0..479).  Ends with the post barrier after its stores.
__device__ __noinline__ void post_tile(PostScratch &P, const UnitDev &U, int tr, int tc, int t) {
    const int w = U.w, h = U.h, cw = w >> 1, ch = h >> 1, mbw = U.mbw, mbh = U.mbh;
    const int B = U.range + 16;
    const int alpha = 6 + U.qp, beta = 2 + U.qp / 4, tcl = 1 + U.qp / 10;
    const int cx0 = tc == 0 ? -3 : 16 * tc, cx1 = tc == mbw - 1 ? w + 3 : 16 * tc + 16;
    const int cy0 = tr == 0 ? -3 : 16 * tr, cy1 = tr == mbh - 1 ? h + 3 : 16 * tr + 16;
    const int dx0 = max(0, cx0 - 2), dx1 = min(w, cx1 + 3), dy0 = max(0, cy0 - 2), dy1 = min(h, cy1 + 3);
    const int vy0 = max(0, dy0 - 2), vy1 = min(h, dy1 + 2), rx0 = max(0, dx0 - 2), rx1 = min(w, dx1 + 2);
    const int cry0 = max(0, 8 * tr - 2), cry1 = min(ch, 8 * tr + 10);
    const int crx0 = max(0, 8 * tc - 2), crx1 = min(cw, 8 * tc + 10);
    // a. the reconstruction (through L2: other blocks wrote most of it)
    {
        const int nrw = rx1 - rx0, nl = (vy1 - vy0) * nrw, ncw = crx1 - crx0, ncl = (cry1 - cry0) * ncw;
        for (int i = t; i < nl + 2 * ncl; i += kPostNT) {
            if (i < nl) {
                const int y = i / nrw, x = i - y * nrw;
                P.rec[y][x] = __ldcg(&U.rec[0][(size_t)(vy0 + y) * w + rx0 + x]);
            } else {
                const int k = i - nl, pl = k >= ncl ? 1 : 0, kk = k - pl * ncl, y = kk / ncw, x = kk - y * ncw;
                P.crec[pl][y][x] = __ldcg(&U.rec[1 + pl][(size_t)(cry0 + y) * cw + crx0 + x]);
            }
        }
    }
    post_bar();
    // b. vertical edges
    {
        const int ndw = dx1 - dx0, nv = (vy1 - vy0) * ndw, ncv = (cry1 - cry0) * 8;
        for (int i = t; i < nv + 2 * ncv; i += kPostNT) {
            if (i < nv) {
                const int y = i / ndw, x = dx0 + (i - y * ndw);
                P.vp[y][x - dx0] = (uint8_t)dbk_sample(&P.rec[y][x - rx0], 1, x, w, alpha, beta, tcl);
            } else {
                const int k = i - nv, pl = k >= ncv ? 1 : 0, kk = k - pl * ncv, y = kk >> 3, x = 8 * tc + (kk & 7);
                P.cv[pl][y][kk & 7] = (uint8_t)dbk_sample(&P.crec[pl][y][x - crx0], 1, x, cw, alpha, beta, tcl);
            }
        }
    }
    post_bar();
    // c. horizontal edges
    {
        const int ndw = dx1 - dx0, nd = (dy1 - dy0) * ndw;
        for (int i = t; i < nd + 2 * 64; i += kPostNT) {
            if (i < nd) {
                const int yy = i / ndw, xx = i - yy * ndw, y = dy0 + yy;
                P.d[yy][xx] = (uint8_t)dbk_sample(&P.vp[y - vy0][xx], 24, y, h, alpha, beta, tcl);
            } else {
                const int k = i - nd, pl = k >> 6, y = 8 * tr + ((k >> 3) & 7), x = k & 7;
                P.cd[pl][(k >> 3) & 7][x] = (uint8_t)dbk_sample(&P.cv[pl][y - cry0][x], 8, y, ch, alpha, beta, tcl);
            }
        }
    }
    post_bar();
    // d. horizontal 6-tap sums at the core columns, every deblocked row
    const int ncx = cx1 - cx0, ncy = cy1 - cy0;
    for (int i = t; i < (dy1 - dy0) * ncx; i += kPostNT) {
        const int yy = i / ncx, xx = i - yy * ncx, x = cx0 + xx;
        const uint8_t *r = P.d[yy];
        int v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = r[clampi(x - 2 + k, 0, w - 1) - dx0];
        P.hs[yy][xx] = (int16_t)tap6i(v[0], v[1], v[2], v[3], v[4], v[5]);
    }
    post_bar();
    // e. the four luma planes at the core samples
    for (int i = t; i < ncy * ncx; i += kPostNT) {
        const int yy = i / ncx, xx = i - yy * ncx, y = cy0 + yy, x = cx0 + xx;
        const int yc = clampi(y, 0, h - 1) - dy0, xc = clampi(x, 0, w - 1) - dx0;
        int rv[6], rh[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int ry = clampi(y - 2 + k, 0, h - 1) - dy0;
            rv[k] = P.d[ry][xc];
            rh[k] = P.hs[ry][xx];
        }
        const int v = tap6i(rv[0], rv[1], rv[2], rv[3], rv[4], rv[5]);
        const int jj = tap6i(rh[0], rh[1], rh[2], rh[3], rh[4], rh[5]);
        P.core[0][yy][xx] = P.d[yc][xc];
        P.core[1][yy][xx] = (uint8_t)clipb((P.hs[yc][xx] + 16) >> 5);
        P.core[2][yy][xx] = (uint8_t)clipb((v + 16) >> 5);
        P.core[3][yy][xx] = (uint8_t)clipb((jj + 512) >> 10);
    }
    post_bar();
    // f. the tile's part of the padded planes, border included, as 32-bit words
    {
        const int xa = tc == 0 ? -B : 16 * tc, xb = tc == mbw - 1 ? w + B : 16 * tc + 16;
        const int ya = tr == 0 ? -B : 16 * tr, yb = tr == mbh - 1 ? h + B : 16 * tr + 16;
        const int nwx = (xb - xa) >> 2, nl = 4 * (yb - ya) * nwx;
        const int xca = tc == 0 ? -B : 8 * tc, xcb = tc == mbw - 1 ? cw + B : 8 * tc + 8;
        const int yca = tr == 0 ? -B : 8 * tr, ycb = tr == mbh - 1 ? ch + B : 8 * tr + 8;
        const int ncwx = (xcb - xca) >> 2, ncl = (ycb - yca) * ncwx;
        uint8_t *const lp[4] = {U.out.G, U.out.B, U.out.H, U.out.J};
        for (int i = t; i < nl + 2 * ncl; i += kPostNT) {
            if (i < nl) {
                const int p = i / ((yb - ya) * nwx), k = i - p * (yb - ya) * nwx, yy = k / nwx, q = k - yy * nwx;
                const int y = ya + yy, x = xa + 4 * q;
                const uint8_t *cr = P.core[p][clampi(y, -3, h + 2) - cy0];
                uint32_t word = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) word |= (uint32_t)cr[clampi(x + b, -3, w + 2) - cx0] << (8 * b);
                *reinterpret_cast<uint32_t *>(lp[p] + (long)y * U.out.ys + x) = word;
            } else {
                const int k = i - nl, pl = k >= ncl ? 1 : 0, kk = k - pl * ncl, yy = kk / ncwx, q = kk - yy * ncwx;
                const int y = yca + yy, x = xca + 4 * q;
                const uint8_t *cr = P.cd[pl][clampi(y, 0, ch - 1) - 8 * tr];
                uint32_t word = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) word |= (uint32_t)cr[clampi(x + b, 0, cw - 1) - 8 * tc] << (8 * b);
                *reinterpret_cast<uint32_t *>((pl ? U.out.V : U.out.U) + (long)y * U.out.cs + x) = word;
            }
        }
    }
    post_bar();
}

}  // namespace fdvb

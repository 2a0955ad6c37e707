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
// below posts tiles in runs of up to kPostRun, behind its own progress; the
// last row posts its own tiles.  Per macroblock row, a count of posted tiles
// is released at GPU scope after the run's stores (a block barrier between).
// A run shares the stage's fixed latencies (six barriers, a round trip to L2)
// among its tiles.
#pragma once
#include "common.cuh"
#include "engine_dev.cuh"

namespace fdvb {

// Threads 32..511 of the P-frame block run the post stage (warp 0 is in the
// wavefront wait meanwhile); named barrier 15 joins them.
constexpr int kPostT0 = 32, kPostNT = 480;
constexpr int kPostRun = 4;                 // tiles per run (4 beat 1 by 9% and 8 by 2% on hd720)
constexpr int kPW = 16 * kPostRun + 16;     // luma scratch pitch (a run's widest row plus slack)
constexpr int kCW = 8 * kPostRun + 8;       // chroma scratch pitch
__device__ __forceinline__ void post_bar() { asm volatile("bar.sync 15, 480;" ::: "memory"); }

struct PostScratch {
    uint8_t rec[25][kPW];       // reconstruction, rows vy0.., columns from rx4 (rx0 rounded down to 4)
    uint8_t vp[25][kPW];        // after the vertical-edge pass, columns dx0..
    uint8_t d[21][kPW];         // deblocked, rows dy0.., columns dx0..
    int16_t hs[21][kPW];        // horizontal 6-tap sums, rows dy0.., core columns cx0..
    uint8_t core[4][22][kPW];   // G, b, h, j at the core samples (rows cy0.., columns cx0..)
    uint8_t crec[2][12][kCW];   // chroma reconstruction, rows cry0.., columns from crx4
    uint8_t cv[2][12][kCW];     // chroma after the vertical-edge pass, columns 8tc0..
    uint8_t cd[2][8][kCW];      // deblocked chroma, columns 8tc0..
};

// The deblocked value of the sample at a[0], position x on a line of n samples
// (a[k * step] the sample at x + k): the filter of the grid edge it touches,
// as filter_edge (frame_ops.cuh) applies it.  Without lane-dependent
// branches: a sample on no edge reads itself as all four taps, for which the
// filter returns it unchanged (d = 0), and the side it is on is selected
// arithmetically.
__device__ __forceinline__ int dbk_sample(const uint8_t *a, int step, int x, int n, int alpha, int beta, int tc) {
    const int e7 = ((x & 7) == 7 && x + 1 < n) ? 1 : 0;   // p0 of the edge after it
    const int e0 = ((x & 7) == 0 && x > 0) ? 1 : 0;       // q0 of the edge before it
    const int p1 = a[-step * (e7 + 2 * e0)], p0 = a[-step * e0], q0 = a[step * e7], q1 = a[step * (2 * e7 + e0)];
    int d = ((q0 - p0) * 4 + (p1 - q1) + 4) >> 3;
    d = d < -tc ? -tc : (d > tc ? tc : d);
    const int on = (abs(p0 - q0) < alpha && abs(p1 - p0) < beta && abs(q1 - q0) < beta) ? 1 : 0;
    const int pv = clipb(p0 + d), qv = clipb(q0 - d), a0 = a[0];
    const int fv = qv + ((pv - qv) & -e7);
    return a0 + ((fv - a0) & -on);
}

__device__ __forceinline__ int tap6i(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
// n / d for 0 <= n < 2^22, 0 < d < 2^10, from r = 1.0f / d: the float
// quotient is within one of the true one, and one correction each way makes
// it exact (a runtime integer division is a long instruction sequence).
__device__ __forceinline__ int fast_div(int n, int d, float r) {
    int q = __float2int_rz(__fmul_rn((float)n, r));
    q += (q + 1) * d <= n ? 1 : 0;
    q -= q * d > n ? 1 : 0;
    return q;
}

// Tiles tc0..tc1-1 (at most kPostRun) of tile row tr of frame U into its
// reference output; t = thread index within the post threads (0..479).  Ends
// with the post barrier after its stores.
__device__ __noinline__ void post_run(PostScratch &P, const UnitDev &U, int tr, int tc0, int tc1, int t) {
    const int w = U.w, h = U.h, cw = w >> 1, ch = h >> 1, mbw = U.mbw, mbh = U.mbh;
    const int B = U.range + 16;
    const int alpha = 6 + U.qp, beta = 2 + U.qp / 4, tcl = 1 + U.qp / 10;
    const int cx0 = tc0 == 0 ? -3 : 16 * tc0, cx1 = tc1 == mbw ? w + 3 : 16 * tc1;
    const int cy0 = tr == 0 ? -3 : 16 * tr, cy1 = tr == mbh - 1 ? h + 3 : 16 * tr + 16;
    const int dx0 = max(0, cx0 - 2), dx1 = min(w, cx1 + 3), dy0 = max(0, cy0 - 2), dy1 = min(h, cy1 + 3);
    const int vy0 = max(0, dy0 - 2), vy1 = min(h, dy1 + 2);
    const int rx4 = max(0, dx0 - 2) & ~3, rx1 = min(w, dx1 + 2);
    const int cry0 = max(0, 8 * tr - 2), cry1 = min(ch, 8 * tr + 10);
    const int ccx0 = 8 * tc0, ccx1 = 8 * tc1;
    const int crx4 = max(0, ccx0 - 2) & ~3, crx1 = min(cw, ccx1 + 2);
    // a. the reconstruction (through L2: other blocks wrote most of it), in
    // aligned 32-bit words (rows start 16-byte aligned, widths multiples of 8);
    // a thread's words are loaded before any is stored, so their L2 round
    // trips overlap
    {
        const int nlw = (rx1 - rx4 + 3) >> 2, ncw = (crx1 - crx4 + 3) >> 2;
        const int nl = (vy1 - vy0) * (kPW / 4), nc = (cry1 - cry0) * (kCW / 4);
        auto word_at = [&](int i, uint32_t *&dst) -> uint32_t {
            dst = nullptr;
            if (i < nl) {
                const int y = i / (kPW / 4), q = i - y * (kPW / 4);
                if (q >= nlw) return 0u;
                dst = reinterpret_cast<uint32_t *>(&P.rec[y][4 * q]);
                return __ldcg(reinterpret_cast<const uint32_t *>(&U.rec[0][(size_t)(vy0 + y) * w + rx4 + 4 * q]));
            }
            if (i >= nl + 2 * nc) return 0u;
            const int k = i - nl, pl = k >= nc ? 1 : 0, kk = k - pl * nc, y = kk / (kCW / 4), q = kk - y * (kCW / 4);
            if (q >= ncw) return 0u;
            dst = reinterpret_cast<uint32_t *>(&P.crec[pl][y][4 * q]);
            return __ldcg(reinterpret_cast<const uint32_t *>(&U.rec[1 + pl][(size_t)(cry0 + y) * cw + crx4 + 4 * q]));
        };
        for (int i = t; i < nl + 2 * nc; i += 2 * kPostNT) {
            uint32_t *d0, *d1;
            const uint32_t v0 = word_at(i, d0), v1 = word_at(i + kPostNT, d1);
            if (d0) *d0 = v0;
            if (d1) *d1 = v1;
        }
    }
    post_bar();
    // b. vertical edges
    {
        const int ndw = dx1 - dx0, nv = (vy1 - vy0) * kPW, ncv = (cry1 - cry0) * kCW, ncc = ccx1 - ccx0;
        for (int i = t; i < nv + 2 * ncv; i += kPostNT) {
            if (i < nv) {
                const int y = i / kPW, xx = i - y * kPW;
                if (xx < ndw) {
                    const int x = dx0 + xx;
                    P.vp[y][xx] = (uint8_t)dbk_sample(&P.rec[y][x - rx4], 1, x, w, alpha, beta, tcl);
                }
            } else {
                const int k = i - nv, pl = k >= ncv ? 1 : 0, kk = k - pl * ncv, y = kk / kCW, xx = kk - y * kCW;
                if (xx < ncc) {
                    const int x = ccx0 + xx;
                    P.cv[pl][y][xx] = (uint8_t)dbk_sample(&P.crec[pl][y][x - crx4], 1, x, cw, alpha, beta, tcl);
                }
            }
        }
    }
    post_bar();
    // c. horizontal edges
    {
        const int ndw = dx1 - dx0, nd = (dy1 - dy0) * kPW, ncc = ccx1 - ccx0;
        for (int i = t; i < nd + 2 * 8 * kCW; i += kPostNT) {
            if (i < nd) {
                const int yy = i / kPW, xx = i - yy * kPW, y = dy0 + yy;
                if (xx < ndw) P.d[yy][xx] = (uint8_t)dbk_sample(&P.vp[y - vy0][xx], kPW, y, h, alpha, beta, tcl);
            } else {
                const int k = i - nd, pl = k >= 8 * kCW ? 1 : 0, kk = k - pl * 8 * kCW, r = kk / kCW, xx = kk - r * kCW;
                const int y = 8 * tr + r;
                if (xx < ncc) P.cd[pl][r][xx] = (uint8_t)dbk_sample(&P.cv[pl][y - cry0][xx], kCW, y, ch, alpha, beta, tcl);
            }
        }
    }
    post_bar();
    // d. horizontal 6-tap sums at the core columns, every deblocked row
    const int ncx = cx1 - cx0, ncy = cy1 - cy0;
    for (int i = t; i < (dy1 - dy0) * kPW; i += kPostNT) {
        const int yy = i / kPW, xx = i - yy * kPW, x = cx0 + xx;
        if (xx >= ncx) continue;
        const uint8_t *r = P.d[yy];
        int v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = r[clampi(x - 2 + k, 0, w - 1) - dx0];
        P.hs[yy][xx] = (int16_t)tap6i(v[0], v[1], v[2], v[3], v[4], v[5]);
    }
    post_bar();
    // e. the four luma planes at the core samples
    for (int i = t; i < ncy * kPW; i += kPostNT) {
        const int yy = i / kPW, xx = i - yy * kPW, y = cy0 + yy, x = cx0 + xx;
        if (xx >= ncx) continue;
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
    // f. the run's part of the padded planes, border included, as 32-bit words
    {
        const int xa = tc0 == 0 ? -B : 16 * tc0, xb = tc1 == mbw ? w + B : 16 * tc1;
        const int ya = tr == 0 ? -B : 16 * tr, yb = tr == mbh - 1 ? h + B : 16 * tr + 16;
        const int nwx = (xb - xa) >> 2, npl = (yb - ya) * nwx, nl = 4 * npl;
        const int xca = tc0 == 0 ? -B : 8 * tc0, xcb = tc1 == mbw ? cw + B : 8 * tc1;
        const int yca = tr == 0 ? -B : 8 * tr, ycb = tr == mbh - 1 ? ch + B : 8 * tr + 8;
        const int ncwx = (xcb - xca) >> 2, ncl = (ycb - yca) * ncwx;
        uint8_t *const lp[4] = {U.out.G, U.out.B, U.out.H, U.out.J};
        const float rnpl = 1.0f / (float)npl, rnwx = 1.0f / (float)nwx, rncwx = 1.0f / (float)ncwx;
        // core columns start at cx0: a word inside the plane whose samples
        // are four aligned core bytes is one load
        const bool core_al = (cx0 & 3) == 0;
        for (int i = t; i < nl + 2 * ncl; i += kPostNT) {
            if (i < nl) {
                const int p = fast_div(i, npl, rnpl), k = i - p * npl, yy = fast_div(k, nwx, rnwx), q = k - yy * nwx;
                const int y = ya + yy, x = xa + 4 * q;
                const uint8_t *cr = P.core[p][clampi(y, -3, h + 2) - cy0];
                uint32_t word = 0;
                if (core_al && x >= 0 && x + 3 < w) {
                    word = *reinterpret_cast<const uint32_t *>(cr + x - cx0);
                } else {
#pragma unroll
                    for (int b = 0; b < 4; ++b) word |= (uint32_t)cr[clampi(x + b, -3, w + 2) - cx0] << (8 * b);
                }
                *reinterpret_cast<uint32_t *>(lp[p] + (long)y * U.out.ys + x) = word;
            } else {
                const int k = i - nl, pl = k >= ncl ? 1 : 0, kk = k - pl * ncl, yy = fast_div(kk, ncwx, rncwx), q = kk - yy * ncwx;
                const int y = yca + yy, x = xca + 4 * q;
                const uint8_t *cr = P.cd[pl][clampi(y, 0, ch - 1) - 8 * tr];
                uint32_t word = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) word |= (uint32_t)cr[clampi(x + b, 0, cw - 1) - ccx0] << (8 * b);
                *reinterpret_cast<uint32_t *>((pl ? U.out.V : U.out.U) + (long)y * U.out.cs + x) = word;
            }
        }
    }
    post_bar();
}

}  // namespace fdvb

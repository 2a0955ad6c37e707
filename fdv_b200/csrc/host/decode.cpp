// The decoder's host half (see decode.h): the frame blobs' stream layer --
// varints, static rANS with the serialised frequency tables, the adaptive
// range coder, the P-frame table cache -- and the per-macroblock / per-leaf
// symbol parse, restated from the reference decoder:
//
//   symbol readers                           fdv.h:1710-1740
//   rANS tables and decoding                 fdv.h:1851-1935
//   adaptive decoder                         fdv.h:2070-2078, :2120-2143
//   P-frame blob and macroblock parse        fdv.h:6492-6737 (chroma :6429-6455)
//   residual parse (4x4, 8x8, regions)       fdv.h:5280-5296, :5421-5465, :2205-2210
//   key-frame plane blob and quadtree parse  fdv.h:5040-5153, :4586-4640
//
// Every read is bounded and a malformed blob is rejected (-1), as the
// reference rejects it.
#include "decode.h"

#include <cstring>

#include "models.h"

using namespace fdvb::ent;

namespace fdvb {
namespace dec {
namespace {

// ---------------------------------------------------------- symbol reads --
struct Rd {
    const uint8_t *s;
    size_t p, end;
    bool *ok;
    int byte() {
        if (p >= end) { *ok = false; return 0; }
        return s[p++];
    }
    int count(int max) {
        const int c = byte();
        if (c > max) { *ok = false; return 0; }
        return c;
    }
    int level() {   // zigzag-coded signed LEB, at most 5 bytes
        uint32_t u = 0;
        int sh = 0;
        for (int k = 0; k < 5; ++k) {
            const int c = byte();
            u |= (uint32_t)(c & 0x7f) << sh;
            sh += 7;
            if (!(c & 0x80)) break;
        }
        return (int)(u >> 1) ^ -(int)(u & 1);
    }
};

uint32_t rd_count32(const uint8_t *s, size_t *p, size_t end, bool *ok) {
    uint32_t v = 0;
    for (int sh = 0;; sh += 7) {
        if (*p >= end || sh > 28) { *ok = false; return 0; }
        const uint8_t c = s[(*p)++];
        v |= (uint32_t)(c & 0x7f) << sh;
        if (!(c & 0x80)) return v;
    }
}
unsigned get16(const uint8_t *b, size_t *p) { const unsigned v = b[*p] | ((unsigned)b[*p + 1] << 8); *p += 2; return v; }
uint32_t get32(const uint8_t *b, size_t *p) {
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)b[*p + i] << (8 * i);
    *p += 4;
    return v;
}

// ------------------------------------------------------------------ rANS --
size_t read_freqs(const uint8_t *in, size_t p, size_t end, uint16_t freq[256], bool *ok) {
    memset(freq, 0, 256 * sizeof(uint16_t));
    if (p + 2 > end) { *ok = false; return p; }
    const int n = in[p] | ((int)in[p + 1] << 8);
    p += 2;
    uint32_t sum = 0;
    for (int k = 0; k < n; ++k) {
        if (p >= end) { *ok = false; return p; }
        const int s = in[p++];
        uint32_t f = 0;
        int sh = 0;
        uint8_t c;
        do {
            if (p >= end || sh > 28) { *ok = false; return p; }
            c = in[p++];
            f |= (uint32_t)(c & 0x7f) << sh;
            sh += 7;
        } while (c & 0x80);
        if (freq[s] != 0) { *ok = false; return p; }   // a symbol listed twice
        freq[s] = (uint16_t)f;
        sum += f;
    }
    if (sum != kScale) *ok = false;
    return p;
}

struct RansDec {
    uint16_t freq[256], cum[256];
    uint8_t slot[kScale];
    explicit RansDec(const uint16_t f[256]) {
        uint16_t c = 0;
        for (int s = 0; s < 256; ++s) {
            freq[s] = f[s];
            cum[s] = c;
            if (f[s]) memset(slot + c, s, f[s]);
            c = (uint16_t)(c + f[s]);
        }
    }
    // n symbols; stops feeding bytes at the end of the input (a corrupt
    // stream then decodes bounded garbage that the parse rejects).
    void decode(const uint8_t *in, size_t len, size_t n, uint8_t *out) const {
        const uint8_t *p = in, *e = in + len;
        uint32_t r = 0;
        for (int b = 0; b < 4; ++b) r |= (uint32_t)(p < e ? *p++ : 0) << (8 * b);
        for (size_t i = 0; i < n; ++i) {
            const uint8_t s = slot[r & (kScale - 1)];
            out[i] = s;
            uint32_t x = freq[s] * (r >> kScaleBits) + (r & (kScale - 1)) - cum[s];
            while (x < kRansLow && p < e) x = (x << 8) | *p++;
            r = x;
        }
    }
};

// ------------------------------------------------------ adaptive decoder --
// The adaptive model as the decoder keeps it: the frequencies alone.  The
// encoder's Fenwick tree serves its cumulative lookups; the decoder finds a
// symbol by a linear scan from symbol 0 instead -- the models are skewed
// towards small symbols, so the scan mostly stops after a few steps, and an
// increment is then a single add.  Same arithmetic as AModel (init, add,
// halving at kAdMax).
struct DModel {
    uint32_t f[256];
    uint32_t tot;
    void init(const uint32_t hist[256]) {   // AModel::init without the tree
        uint64_t s = 0;
        for (int i = 0; i < 256; ++i) s += hist[i];
        uint32_t t = 0;
        if (s <= kAdScale) {
            for (int i = 0; i < 256; ++i) t += (f[i] = kAdBase + hist[i]);
        } else {
            for (int i = 0; i < 256; ++i)   // a zero count scales to zero: no division
                t += (f[i] = kAdBase + (hist[i] ? (uint32_t)(((uint64_t)hist[i] * kAdScale + s / 2) / s) : 0));
        }
        tot = t;
    }
    void add(unsigned s, uint32_t d) {
        f[s] += d;
        tot += d;
        if (tot > kAdMax) {
            uint32_t t = 0;
            for (int i = 0; i < 256; ++i) t += (f[i] = (f[i] + 1) >> 1);
            tot = t;
        }
    }
};

struct ADec {
    const uint8_t *in;
    size_t len, p = 0;
    uint32_t range = 0xFFFFFFFFu, code = 0;
    ADec(const uint8_t *i, size_t l) : in(i), len(l) {
        for (int k = 0; k < 4; ++k) { code = (code << 8) | (p < len ? in[p] : 0); ++p; }
    }
    unsigned sym(DModel &m) {
        const uint32_t r = range / m.tot;
        uint32_t v = code / r;
        if (v >= m.tot) v = m.tot - 1;
        unsigned s = 0;
        uint32_t cum = 0;
        while (cum + m.f[s] <= v) cum += m.f[s++];   // ends by 255: v < tot
        code -= r * cum;
        range = r * m.f[s];
        while (range < (1u << 24)) {
            code = (code << 8) | (p < len ? in[p] : 0);
            ++p;
            range <<= 8;
        }
        m.add(s, kAdInc);
        return s;
    }
};

// -------------------------------------------------------------- residuals --
constexpr uint8_t kZZ4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
constexpr uint8_t kZZ8[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                              12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                              35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                              58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// The coefficient cursors of one frame (fdv_cr): 4x4 counts and levels
// (luma, chroma), 8x8 counts and levels, region flags.
struct Coef {
    Rd n, l, n8, l8, fl, nc, lc;
    bool chroma = false;
    // a 4x4 block into dst[16] (natural order)
    void block4(int16_t *dst) {
        Rd &cn = chroma ? nc : n, &cl = chroma ? lc : l;
        const int cnt = cn.count(16);
        for (int k = 0; k < cnt; ++k) dst[kZZ4[k]] = (int16_t)cl.level();
    }
    void block8(int16_t *dst) {
        const int cnt = n8.count(64);
        for (int k = 0; k < cnt; ++k) dst[kZZ8[k]] = (int16_t)l8.level();
    }
    // decode_residual for n >= 8: per 8x8 region (raster) a flag, then four
    // 4x4 blocks or one 8x8; region r lands at dst + 64 r, its flag in flags[r].
    bool residual(int n, int16_t *dst, uint8_t *flags) {
        const int nr = n / 8;
        for (int r = 0; r < nr * nr; ++r) {
            const int f = fl.byte();
            if (f > 2) return false;
            flags[r] = (uint8_t)f;
            int16_t *d = dst + 64 * r;
            if (f == 1)
                for (int b = 0; b < 4; ++b) block4(d + 16 * b);
            else if (f == 2)
                block8(d);
        }
        return true;
    }
};

// ------------------------------------------------------ P-frame helpers --
constexpr int kNS = 16;          // 9 structure streams + 7 coefficient streams
constexpr int kPsRef = 4, kPsMvx = 5, kPsMvy = 6, kPsSub = 7, kPsMerge = 8;

struct MbMv { int16_t x, y; uint8_t ref, inter; };

bool mv_in_bounds(int w, int h, int border, int x, int y, int bw, int bh, int mvx, int mvy) {
    const int ix = x + (mvx >> 2), iy = y + (mvy >> 2);
    if (ix - 3 < -border || iy - 3 < -border) return false;
    if (ix + bw + 3 > w + border || iy + bh + 3 > h + border) return false;
    return true;
}

}  // namespace

int pframe_symbols(const uint8_t *in, size_t len, int w, int h, fdvb_tabcache *tc, Syms &out) {
    if (len < 2) return -1;
    size_t p = 0;
    const int qp = in[p++];
    if (qp > 51) return -1;
    const int emode = in[p++];
    const size_t nmb = (size_t)((w + 15) / 16) * (size_t)(h / 16);
    const size_t maxsyms = nmb * (size_t)(16 + 384 * 6);
    if (emode > 3) return -1;
    const bool reuse = emode == 2;
    if (reuse && (!tc || !tc->have)) return -1;
    size_t sn[kNS], base[kNS], total = 0;
    for (int k = 0; k < kNS; ++k) {
        bool ok = true;
        const uint32_t v = rd_count32(in, &p, len, &ok);
        if (!ok || v > maxsyms) return -1;
        sn[k] = v;
        total += v;
        if (total > maxsyms) return -1;
    }
    for (size_t k = 0, o = 0; k < kNS; ++k) { base[k] = o; o += sn[k]; }
    out.qp = qp;
    std::vector<uint8_t> &syms = out.buf;
    syms.resize(total ? total : 1);
    for (int k = 0; k < kNS; ++k) { out.sn[k] = sn[k]; out.base[k] = base[k]; }
    if (!(emode & 1)) {   // one shared model
        uint16_t freq[256];
        bool ok = true;
        if (reuse) memcpy(freq, tc->f1, sizeof freq);
        else p = read_freqs(in, p, len, freq, &ok);
        if (!ok || p + 4 > len) return -1;
        const uint32_t l1 = get32(in, &p);
        if (p + l1 > len) return -1;
        RansDec d(freq);
        d.decode(in + p, l1, total, syms.data());
        if (!reuse && tc) { tab_store(tc->f1, freq); tc->have = 1; }
    } else {              // a model per stream
        if (p + 2 > len) return -1;
        const unsigned mask = get16(in, &p);
        unsigned am = 0;
        if (emode == 3) {
            if (!tc || !tc->hn) return -1;
            am = ad_select(sn, kNS, nullptr);
        }
        if ((mask & ~am) && (!tc || !tc->have)) return -1;
        for (int k = 0; k < kNS; ++k) {
            if (sn[k] == 0 || ((am >> k) & 1)) continue;
            bool ok = true;
            const bool reused = (mask >> k) & 1;
            uint16_t freq[256];
            if (reused) memcpy(freq, tc->fs[k], sizeof freq);
            else p = read_freqs(in, p, len, freq, &ok);
            if (!ok) return -1;
            const uint32_t n = rd_count32(in, &p, len, &ok);
            if (!ok || p + n > len) return -1;
            RansDec d(freq);
            d.decode(in + p, n, sn[k], syms.data() + base[k]);
            p += n;
            if (!reused && tc) tab_store(tc->fs[k], freq);
        }
        if (am) {
            bool ok = true;
            const uint32_t n = rd_count32(in, &p, len, &ok);
            if (!ok || p + n > len) return -1;
            ADec ad(in + p, n);
            for (int k = 0; k < kNS; ++k) {
                if (!((am >> k) & 1)) continue;
                DModel m;
                m.init(tc->hist[k]);
                for (size_t i = 0; i < sn[k]; ++i) syms[base[k] + i] = (uint8_t)ad.sym(m);
            }
            p += n;
        }
        if (tc) tc->have = 1;
    }
    if (tc) {   // the history the next frame's adaptive models start from
        for (int k = 0; k < kNS; ++k) {
            uint32_t c[256] = {0};
            for (size_t i = 0; i < sn[k]; ++i) c[syms[base[k] + i]]++;
            hist_add(tc->hist[k], c);
        }
        if (tc->hn < (1 << 20)) ++tc->hn;
    }
    return 0;
}

int pframe_records(const Syms &sy, int w, int h, int border, PFrame &out) {
    const int qp = sy.qp;
    bool ok = true;
    Rd S[kNS];
    for (int k = 0; k < kNS; ++k) S[k] = Rd{sy.buf.data(), sy.base[k], sy.base[k] + sy.sn[k], &ok};
    Coef R{S[9], S[10], S[11], S[12], S[13], S[14], S[15]};
    const int mbw = w / 16, mbh = h / 16;
    out.qp = qp;
    out.mbs.assign((size_t)mbw * mbh, PMB{});
    out.coef.clear();
    out.intra.clear();
    std::vector<uint8_t> mmap((size_t)mbw * mbh, 0);
    std::vector<MbMv> mvmap((size_t)mbw * mbh, MbMv{0, 0, 0, 0});
    auto new_block = [&](PMB &mb) {
        mb.coef = (int32_t)out.coef.size();
        out.coef.resize(out.coef.size() + 384, 0);
        return out.coef.data() + mb.coef;
    };
    for (int mby = 0; mby < mbh && ok; ++mby) {
        int pmvx = 0, pmvy = 0;
        for (int mbx = 0; mbx < mbw && ok; ++mbx) {
            const int bx = mbx * 16, by = mby * 16, cbx = bx / 2, cby = by / 2;
            const int L = mbx > 0 ? mmap[mby * mbw + mbx - 1] : 0, A = mby > 0 ? mmap[(mby - 1) * mbw + mbx] : 0;
            const int mc = (L != 0 ? 2 : 0) + (A != 0 ? 1 : 0);
            const int mode = S[mc].byte();
            mmap[mby * mbw + mbx] = (uint8_t)mode;
            PMB &mb = out.mbs[(size_t)mby * mbw + mbx];
            mb.mode = (uint8_t)mode;
            mb.coef = -1;
            if (mode == 2) {   // INTRA16: prediction needs the reconstruction, done on the GPU
                mb.sub = (uint8_t)S[kPsSub].byte();
                int16_t *cb = new_block(mb);
                uint8_t f[4];
                if (!R.residual(16, cb, f)) { ok = false; break; }
                cb = out.coef.data() + mb.coef;
                mb.lfl = (uint8_t)(f[0] | (f[1] << 2) | (f[2] << 4) | (f[3] << 6));
                R.chroma = true;
                for (int pl = 0; pl < 2; ++pl) {
                    uint8_t cf;
                    if (!R.residual(8, cb + 256 + 64 * pl, &cf)) { ok = false; break; }
                    mb.cfl |= (uint8_t)(cf << (2 * pl));
                }
                R.chroma = false;
                mvmap[(size_t)mby * mbw + mbx] = MbMv{0, 0, 0, 0};
                out.intra.push_back(mby * mbw + mbx);
                continue;   // the MV predictor is unchanged
            }
            if (mode == 3) {   // INTER8
                int qpx = pmvx, qpy = pmvy;
                int16_t *cb = new_block(mb);
                uint8_t f[4] = {0, 0, 0, 0};
                for (int q = 0; q < 4 && ok; ++q) {
                    const int mx = qpx + S[kPsMvx].level(), my = qpy + S[kPsMvy].level();
                    qpx = mx;
                    qpy = my;
                    mb.mv[q][0] = (int16_t)mx;
                    mb.mv[q][1] = (int16_t)my;
                    if (!ok || !mv_in_bounds(w, h, border, bx + (q & 1) * 8, by + (q >> 1) * 8, 8, 8, mx, my)) {
                        ok = false;
                        break;
                    }
                    if (!R.residual(8, cb + 64 * q, &f[q])) { ok = false; break; }
                }
                if (!ok) break;
                mb.lfl = (uint8_t)(f[0] | (f[1] << 2) | (f[2] << 4) | (f[3] << 6));
                pmvx = mb.mv[3][0];
                pmvy = mb.mv[3][1];
                mvmap[(size_t)mby * mbw + mbx] = MbMv{mb.mv[3][0], mb.mv[3][1], 0, 1};
                R.chroma = true;
                for (int pl = 0; pl < 2 && ok; ++pl)
                    for (int q = 0; q < 4 && ok; ++q) {
                        if (!mv_in_bounds(w / 2, h / 2, border, cbx + (q & 1) * 4, cby + (q >> 1) * 4, 4, 4,
                                          mb.mv[q][0] / 2, mb.mv[q][1] / 2)) {
                            ok = false;
                            break;
                        }
                        R.block4(cb + 256 + 64 * pl + 16 * q);
                    }
                R.chroma = false;
                mb.cfl = 1 | (1 << 2);
                continue;
            }
            if (mode != 0 && mode != 1) { ok = false; break; }
            int mvx, mvy, ridx = 0;
            const bool skip = mode == 0;
            if (skip) {   // merge candidates from the macroblocks decoded so far (fdv.h:5711-5729)
                MbMv cand[3];
                int nc = 0;
                cand[nc++] = MbMv{(int16_t)pmvx, (int16_t)pmvy, 0, 1};
                const int src[2][2] = {{mbx, mby - 1}, {mbx + 1, mby - 1}};
                for (int k = 0; k < 2 && nc < 3; ++k) {
                    const int cx = src[k][0], cy = src[k][1];
                    if (cx < 0 || cy < 0 || cx >= mbw) continue;
                    const MbMv &m = mvmap[(size_t)cy * mbw + cx];
                    if (!m.inter) continue;
                    bool dup = false;
                    for (int j = 0; j < nc; ++j)
                        if (cand[j].x == m.x && cand[j].y == m.y && cand[j].ref == m.ref) dup = true;
                    if (!dup) cand[nc++] = m;
                }
                int mi = 0;
                if (nc > 1) {
                    mi = S[kPsMerge].count(nc - 1);
                    if (!ok) break;
                }
                mvx = cand[mi].x;
                mvy = cand[mi].y;
                ridx = cand[mi].ref;
            } else {
                ridx = S[kPsRef].byte();
                if (ridx > 1) { ok = false; break; }
                mvx = pmvx + S[kPsMvx].level();
                mvy = pmvy + S[kPsMvy].level();
            }
            pmvx = mvx;
            pmvy = mvy;
            mvmap[(size_t)mby * mbw + mbx] = MbMv{(int16_t)mvx, (int16_t)mvy, (uint8_t)ridx, 1};
            mb.ref = (uint8_t)ridx;
            mb.mv[0][0] = (int16_t)mvx;
            mb.mv[0][1] = (int16_t)mvy;
            if (!ok || !mv_in_bounds(w, h, border, bx, by, 16, 16, mvx, mvy) ||
                !mv_in_bounds(w / 2, h / 2, border, cbx, cby, 8, 8, mvx / 2, mvy / 2)) {
                ok = false;
                break;
            }
            if (!skip) {
                int16_t *cb = new_block(mb);
                uint8_t f[4];
                if (!R.residual(16, cb, f)) { ok = false; break; }
                mb.lfl = (uint8_t)(f[0] | (f[1] << 2) | (f[2] << 4) | (f[3] << 6));
                R.chroma = true;
                for (int pl = 0; pl < 2; ++pl) {   // chroma_block_dec: an any-flag, then four 4x4 blocks
                    const int any = R.fl.byte();
                    if (any > 1) { ok = false; break; }
                    if (any)
                        for (int b = 0; b < 4; ++b) R.block4(cb + 256 + 64 * pl + 16 * b);
                    mb.cfl |= (uint8_t)(any << (2 * pl));
                }
                R.chroma = false;
            }
        }
    }
    return ok ? 0 : -1;
}

int parse_pframe(const uint8_t *in, size_t len, int w, int h, int border, fdvb_tabcache *tc, PFrame &out) {
    Syms sy;
    if (pframe_symbols(in, len, w, h, tc, sy)) return -1;
    return pframe_records(sy, w, h, border, out);
}

namespace {
constexpr int kIsModeB = 4, kIsMode0 = 5, kIsMode1 = 6, kIsN = 12;

struct IParse {
    int w, h, mmw;
    Rd *S;
    Coef *R;
    std::vector<uint8_t> mmap;
    IPlane *out;
    bool *ok;
    void node(int bx, int by, int n, int depth) {
        if (!*ok) return;
        const int hn = n / 2;
        if (bx + n > w || by + n > h) {   // a partial node: its children, no flag
            for (int k = 0; k < 4; ++k) {
                const int cx = bx + (k & 1) * hn, cy = by + (k >> 1) * hn;
                if (cx >= w || cy >= h) continue;
                node(cx, cy, hn, depth + 1);
            }
            return;
        }
        if (n == 4) {
            const int cx = bx / 4, cy = by / 4;
            const int L = cx > 0 ? mmap[cy * mmw + cx - 1] : 0, A = cy > 0 ? mmap[(cy - 1) * mmw + cx] : 0;
            const int mode = S[L == A ? kIsMode0 : kIsMode1].count(8);
            if (!*ok) return;
            mmap[cy * mmw + cx] = (uint8_t)mode;
            Leaf lf{(uint16_t)bx, (uint16_t)by, 4, (uint8_t)mode, 0, (int32_t)out->coef.size(), -1};
            out->coef.resize(out->coef.size() + 16, 0);
            R->block4(out->coef.data() + lf.coef);
            out->leaves.push_back(lf);
            return;
        }
        const int split = S[depth].count(1);
        if (!*ok) return;
        if (split) {
            for (int k = 0; k < 4; ++k) node(bx + (k & 1) * hn, by + (k >> 1) * hn, hn, depth + 1);
            return;
        }
        const int mode = S[kIsModeB].count(3);
        if (!*ok) return;
        const int nr = (n / 8) * (n / 8);
        Leaf lf{(uint16_t)bx, (uint16_t)by, (uint8_t)n, (uint8_t)mode, (uint16_t)nr, (int32_t)out->coef.size(),
                (int32_t)out->flags.size()};
        out->coef.resize(out->coef.size() + (size_t)n * n, 0);
        out->flags.resize(out->flags.size() + nr, 0);
        if (!R->residual(n, out->coef.data() + lf.coef, out->flags.data() + lf.fl)) { *ok = false; return; }
        out->leaves.push_back(lf);
        const int m4 = mode == 1 ? 1 : (mode == 2 ? 2 : 0);   // the 4x4 mode neighbours see
        for (int i = 0; i < n / 4; ++i) memset(&mmap[(size_t)(by / 4 + i) * mmw + bx / 4], m4, (size_t)(n / 4));
    }
};
}  // namespace

int iplane_symbols(const uint8_t *in, size_t len, int ew, int eh, Syms &out) {
    if (len < 6) return -1;
    size_t p = 0;
    const int w = (int)get16(in, &p), h = (int)get16(in, &p);
    const int qp = in[p++];
    if (w <= 0 || h <= 0 || (w & 3) || (h & 3) || w > 8192 || h > 8192 || qp > 51) return -1;
    if (w != ew || h != eh) return -1;
    const int imode = in[p++];
    if (imode > 2) return -1;
    const size_t ctus = (size_t)((w + 63) / 64) * ((h + 63) / 64), b4 = (size_t)(w / 4) * (h / 4);
    size_t cap[kIsN];
    for (int d = 0, k = 1; d < 4; ++d, k *= 4) cap[d] = (size_t)k * ctus;
    cap[kIsModeB] = cap[kIsMode0] = cap[kIsMode1] = b4;
    cap[7] = cap[9] = cap[11] = ctus * 328;
    cap[8] = cap[10] = ctus * 20544;
    size_t sn[kIsN], off[kIsN], total = 0;
    {
        bool ok = true;
        for (int k = 0; k < kIsN; ++k) {
            const uint32_t v = rd_count32(in, &p, len, &ok);
            if (!ok || v > cap[k]) return -1;
            off[k] = total;
            sn[k] = v;
            total += v;
        }
    }
    out.qp = qp;
    out.w = w;
    out.h = h;
    for (int k = 0; k < kIsN; ++k) { out.sn[k] = sn[k]; out.base[k] = off[k]; }
    std::vector<uint8_t> &syms = out.buf;
    syms.resize(total ? total : 1);
    if (imode == 2) {   // one adaptive blob, every model starting flat
        bool ok = true;
        const uint32_t la = rd_count32(in, &p, len, &ok);
        if (!ok || p + la > len) return -1;
        const uint32_t flat[256] = {0};
        ADec ad(in + p, la);
        for (int k = 0; k < kIsN; ++k) {
            DModel m;
            m.init(flat);
            for (size_t i = 0; i < sn[k]; ++i) syms[off[k] + i] = (uint8_t)ad.sym(m);
        }
    } else if (imode == 0) {   // one shared model
        uint16_t freq[256];
        bool ok = true;
        p = read_freqs(in, p, len, freq, &ok);
        if (!ok) return -1;
        const uint32_t l1 = rd_count32(in, &p, len, &ok);
        if (!ok || p + l1 > len) return -1;
        RansDec d(freq);
        d.decode(in + p, l1, total, syms.data());
    } else {   // a model per stream
        for (int k = 0; k < kIsN; ++k) {
            if (sn[k] == 0) continue;
            uint16_t freq[256];
            bool ok = true;
            p = read_freqs(in, p, len, freq, &ok);
            if (!ok) return -1;
            const uint32_t lk = rd_count32(in, &p, len, &ok);
            if (!ok || p + lk > len) return -1;
            RansDec d(freq);
            d.decode(in + p, lk, sn[k], syms.data() + off[k]);
            p += lk;
        }
    }
    return 0;
}

int iplane_records(const Syms &sy, IPlane &out) {
    const int w = sy.w, h = sy.h, qp = sy.qp;
    bool ok = true;
    Rd S[kIsN];
    for (int k = 0; k < kIsN; ++k) S[k] = Rd{sy.buf.data(), sy.base[k], sy.base[k] + sy.sn[k], &ok};
    Rd empty{sy.buf.data(), 0, 0, &ok};
    Coef R{S[7], S[8], S[9], S[10], S[11], empty, empty};
    out.w = w;
    out.h = h;
    out.qp = qp;
    out.leaves.clear();
    out.coef.clear();
    out.flags.clear();
    out.ctu_first.clear();
    IParse ip{w, h, w / 4, S, &R, std::vector<uint8_t>((size_t)(w / 4) * (h / 4), 0), &out, &ok};
    for (int by = 0; by < h && ok; by += 64)
        for (int bx = 0; bx < w && ok; bx += 64) {
            out.ctu_first.push_back((int32_t)out.leaves.size());
            ip.node(bx, by, 64, 0);
        }
    out.ctu_first.push_back((int32_t)out.leaves.size());
    return ok ? 0 : -1;
}

int parse_iplane(const uint8_t *in, size_t len, int w, int h, IPlane &out) {
    Syms sy;
    if (iplane_symbols(in, len, w, h, sy)) return -1;
    return iplane_records(sy, out);
}

}  // namespace dec
}  // namespace fdvb

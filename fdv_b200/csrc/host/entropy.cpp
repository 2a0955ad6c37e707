// The entropy tail of the encoder: turns the symbol streams the GPU analysis
// produced into a frame blob.  This part stays on the host CPU by design -- it
// is serial, adaptive and under 1% of the reference's encode time -- and it has
// to write exactly the bytes the reference writes, so the steps below follow
// the reference's stream format one for one, in code of this project:
//
//   * static byte-wise rANS, 12-bit scale, state in [2^23, 2^31)      fdv.h:1753-1948
//   * frequency normalisation and compact table serialisation         fdv.h:1804-1886
//   * the adaptive Fenwick-model range coder with carry propagation   fdv.h:2003-2118
//   * the budgeted choice of adaptively-coded streams                 fdv.h:482-499
//   * table cache: cached-table form, history accumulation            fdv.h:5641-5677
//   * the P-frame blob: four candidate arrangements, smallest wins    fdv.h:6172-6426
//   * the intra-plane blob: three candidate arrangements              fdv.h:4907-5032
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fdvb_internal.h"
#include "models.h"

using namespace fdvb::ent;

namespace {

// ---------------------------------------------------------------- tables --
void freqs_from_counts(const uint32_t counts[256], uint16_t freq[256]) {
    uint32_t total = 0;
    for (int i = 0; i < 256; ++i) total += counts[i];
    if (total == 0) {
        memset(freq, 0, 256 * sizeof(uint16_t));
        freq[0] = (uint16_t)kScale;
        return;
    }
    uint32_t sum = 0;
    int big = 0;
    for (int i = 0; i < 256; ++i) {
        if (counts[i] == 0) { freq[i] = 0; continue; }
        uint32_t f = (uint32_t)((uint64_t)counts[i] * kScale / total);
        if (f == 0) f = 1;
        freq[i] = (uint16_t)f;
        sum += f;
        if (f > freq[big]) big = i;
    }
    freq[big] = (uint16_t)((int)freq[big] + ((int)kScale - (int)sum));
}

size_t freqs_size(const uint16_t freq[256]) {
    size_t n = 2;
    for (int s = 0; s < 256; ++s) {
        if (!freq[s]) continue;
        n += 1;
        uint32_t f = freq[s];
        do { n += 1; f >>= 7; } while (f);
    }
    return n;
}

size_t write_freqs(uint8_t *out, size_t o, const uint16_t freq[256]) {
    int n = 0;
    for (int s = 0; s < 256; ++s) if (freq[s]) ++n;
    out[o++] = (uint8_t)(n & 0xff);
    out[o++] = (uint8_t)(n >> 8);
    for (int s = 0; s < 256; ++s) {
        if (!freq[s]) continue;
        out[o++] = (uint8_t)s;
        uint32_t f = freq[s];
        while (f >= 0x80) { out[o++] = (uint8_t)(f | 0x80); f >>= 7; }
        out[o++] = (uint8_t)f;
    }
    return o;
}

// Encode n symbols against a frequency table.  Returns the forward-readable
// stream (written from the front of `out`).
size_t rans_encode(const uint8_t *syms, size_t n, const uint16_t freq[256],
                   std::vector<uint8_t> &out) {
    uint16_t cum[256];
    uint16_t c = 0;
    for (int s = 0; s < 256; ++s) { cum[s] = c; c = (uint16_t)(c + freq[s]); }
    size_t cap = n * 2 + 1024;
    out.resize(cap);
    uint8_t *end = out.data() + cap, *p = end;
    uint32_t x = kRansLow;
    for (size_t i = n; i-- > 0;) {
        uint32_t f = freq[syms[i]];
        uint64_t x_max = ((uint64_t)(kRansLow >> kScaleBits) << 8) * f;
        while (x >= x_max) { *--p = (uint8_t)(x & 0xff); x >>= 8; }
        x = ((x / f) << kScaleBits) + (x % f) + cum[syms[i]];
    }
    p -= 4;
    p[0] = (uint8_t)x; p[1] = (uint8_t)(x >> 8); p[2] = (uint8_t)(x >> 16); p[3] = (uint8_t)(x >> 24);
    size_t len = (size_t)(end - p);
    memmove(out.data(), p, len);
    out.resize(len);
    return len;
}

// ------------------------------------------------------- adaptive coder --
struct AEnc {
    std::vector<uint8_t> out;
    size_t cap, n = 0;
    uint64_t low = 0;
    uint32_t range = 0xFFFFFFFFu;
    uint8_t cache = 0;
    uint64_t csize = 1;
    int fail = 0;
    explicit AEnc(size_t c) : out(c), cap(c) {}
    void shift() {
        if ((uint32_t)low < 0xFF000000u || (uint32_t)(low >> 32) != 0) {
            uint8_t c = cache, carry = (uint8_t)(low >> 32);
            do {
                if (n < cap) out[n++] = (uint8_t)(c + carry);
                else fail = 1;
                c = 0xFF;
            } while (--csize);
            cache = (uint8_t)((uint32_t)low >> 24);
        }
        csize++;
        low = (uint32_t)((uint32_t)low << 8);
    }
    void sym(AModel &m, unsigned s) {
        uint32_t r = range / m.tot;
        low += (uint64_t)r * m.cum(s);
        range = r * m.f[s];
        while (range < (1u << 24)) { shift(); range <<= 8; }
        m.add(s, kAdInc);
    }
    // Flush; the stream is out[0..len).  0 when the buffer ran out.
    size_t finish() {
        for (int i = 0; i < 5; ++i) shift();
        if (fail || n < 1) return 0;
        memmove(out.data(), out.data() + 1, n - 1);
        return n - 1;
    }
};

bool tab_covers(const uint16_t freq[256], const uint32_t cnt[256]) {
    for (int i = 0; i < 256; ++i) if (cnt[i] && !freq[i]) return false;
    return true;
}

}  // namespace

size_t fdvb_put16(uint8_t *b, size_t p, unsigned v) { b[p] = (uint8_t)v; b[p + 1] = (uint8_t)(v >> 8); return p + 2; }
size_t fdvb_put32(uint8_t *b, size_t p, uint32_t v) { for (int i = 0; i < 4; ++i) b[p + i] = (uint8_t)(v >> (8 * i)); return p + 4; }
size_t fdvb_leb_put(uint8_t *b, size_t p, uint32_t u) {
    while (u >= 0x80) { b[p++] = (uint8_t)(u | 0x80); u >>= 7; }
    b[p++] = (uint8_t)u;
    return p;
}
int fdvb_leb_size(uint32_t u) { int n = 1; while (u >= 0x80) { u >>= 7; ++n; } return n; }

size_t fdvb_pframe_blob(const fdvb_streams *st, int qp, fdvb_tabcache *tc,
                        uint8_t *out, size_t cap, int *emode_out) {
    const int NS = PS_NS;
    const size_t *sn = st->n;
    size_t total = 0;
    for (int k = 0; k < NS; ++k) total += sn[k];
    std::vector<uint8_t> all(total ? total : 1);
    {
        size_t o = 0;
        for (int k = 0; k < NS; ++k) { if (sn[k]) memcpy(all.data() + o, st->s[k], sn[k]); o += sn[k]; }
    }
    // per-stream symbol counts (counted on the GPU when the streams came from
    // the engine) and their sum, the one-model counts
    static thread_local uint32_t ck[16][256];
    for (int k = 0; k < NS; ++k) {
        if (st->hist) memcpy(ck[k], st->hist + (size_t)k * 256, sizeof ck[k]);
        else {
            memset(ck[k], 0, sizeof ck[k]);
            for (size_t i = 0; i < sn[k]; ++i) ck[k][st->s[k][i]]++;
        }
    }
    uint32_t c1[256] = {0};
    for (int k = 0; k < NS; ++k)
        for (int v = 0; v < 256; ++v) c1[v] += ck[k][v];
    uint16_t f1[256];
    freqs_from_counts(c1, f1);
    std::vector<uint8_t> p1;
    size_t l1 = rans_encode(all.data(), total, f1, p1);

    uint16_t fk[16][256];
    std::vector<uint8_t> pay[16];
    size_t len[16];
    for (int k = 0; k < NS; ++k) {
        freqs_from_counts(ck[k], fk[k]);
        len[k] = rans_encode(st->s[k], sn[k], fk[k], pay[k]);
    }
    size_t hdr = 0;
    for (int k = 0; k < NS; ++k) hdr += (size_t)fdvb_leb_size((uint32_t)sn[k]);
    size_t size_one = hdr + freqs_size(f1) + 4 + l1;

    const size_t NONE = (size_t)-1;
    size_t l1r = 0, lenr[16] = {0};
    size_t size_one_r = NONE, size_two_r = NONE;
    std::vector<uint8_t> p1r, payr[16];
    if (tc && tc->have) {
        if (tab_covers(tc->f1, c1)) {
            l1r = rans_encode(all.data(), total, tc->f1, p1r);
            if (l1r) size_one_r = hdr + 4 + l1r;
        }
        bool cover = true;
        for (int k = 0; k < NS; ++k) if (!tab_covers(tc->fs[k], ck[k])) cover = false;
        if (cover) {
            for (int k = 0; k < NS; ++k) lenr[k] = rans_encode(st->s[k], sn[k], tc->fs[k], payr[k]);
            size_two_r = hdr;
            for (int k = 0; k < NS; ++k) size_two_r += 4 + lenr[k];
        }
    }
    bool have_reuse = tc && tc->have && size_two_r != NONE;
    size_t size_mix = hdr + 2;
    unsigned mask = 0;
    for (int k = 0; k < NS; ++k) {
        if (sn[k] == 0) continue;
        size_t fresh = freqs_size(fk[k]) + (size_t)fdvb_leb_size((uint32_t)len[k]) + len[k];
        size_t reused = have_reuse ? (size_t)fdvb_leb_size((uint32_t)lenr[k]) + lenr[k] : NONE;
        if (reused < fresh) { size_mix += reused; mask |= 1u << k; }
        else size_mix += fresh;
    }

    size_t size_ada = NONE, lada = 0;
    unsigned amask = 0;
    std::vector<uint8_t> pada;
    if (tc && tc->hn) {
        size_t asyms = 0;
        amask = ad_select(sn, NS, &asyms);
        if (amask) {
            AEnc ae(asyms * 3 + 64);
            for (int k = 0; k < NS; ++k) {
                if (!((amask >> k) & 1)) continue;
                AModel m;
                m.init(tc->hist[k]);
                for (size_t i = 0; i < sn[k]; ++i) ae.sym(m, st->s[k][i]);
            }
            lada = ae.finish();
            if (lada) {
                pada.assign(ae.out.begin(), ae.out.begin() + (long)lada);
                size_ada = hdr + 2 + (size_t)fdvb_leb_size((uint32_t)lada) + lada;
                for (int k = 0; k < NS; ++k) {
                    if (sn[k] == 0 || ((amask >> k) & 1)) continue;
                    size_t fresh = freqs_size(fk[k]) + (size_t)fdvb_leb_size((uint32_t)len[k]) + len[k];
                    size_t reused = have_reuse ? (size_t)fdvb_leb_size((uint32_t)lenr[k]) + lenr[k] : NONE;
                    size_ada += reused < fresh ? reused : fresh;
                }
            }
        }
    }

    int emode = 0;
    size_t best = size_one;
    if (size_mix < best) { best = size_mix; emode = 1; }
    if (size_one_r < best) { best = size_one_r; emode = 2; }
    if (size_ada < best) { best = size_ada; emode = 3; }
    if (emode_out) *emode_out = emode;
    if (2 + best > cap) return 0;

    size_t o = 0;
    out[o++] = (uint8_t)qp;
    out[o++] = (uint8_t)emode;
    for (int k = 0; k < NS; ++k) o = fdvb_leb_put(out, o, (uint32_t)sn[k]);
    if (!(emode & 1)) {
        if (!(emode & 2)) o = write_freqs(out, o, f1);
        size_t n = (emode & 2) ? l1r : l1;
        const uint8_t *q = (emode & 2) ? p1r.data() : p1.data();
        o = fdvb_put32(out, o, (uint32_t)n);
        memcpy(out + o, q, n); o += n;
    } else {
        unsigned am = (emode == 3) ? amask : 0u;
        o = fdvb_put16(out, o, mask & ~am);
        for (int k = 0; k < NS; ++k) {
            if (sn[k] == 0 || ((am >> k) & 1)) continue;
            int reused = (mask >> k) & 1;
            if (!reused) o = write_freqs(out, o, fk[k]);
            size_t n = reused ? lenr[k] : len[k];
            const uint8_t *q = reused ? payr[k].data() : pay[k].data();
            o = fdvb_leb_put(out, o, (uint32_t)n);
            memcpy(out + o, q, n); o += n;
        }
        if (emode == 3) {
            o = fdvb_leb_put(out, o, (uint32_t)lada);
            memcpy(out + o, pada.data(), lada); o += lada;
        }
    }
    if (tc) {
        if (emode == 0) { tab_store(tc->f1, f1); tc->have = 1; }
        else if (emode == 1 || emode == 3) {
            unsigned am = (emode == 3) ? amask : 0u;
            for (int k = 0; k < NS; ++k)
                if (sn[k] && !((am >> k) & 1) && !((mask >> k) & 1)) tab_store(tc->fs[k], fk[k]);
            tc->have = 1;
        }
        for (int k = 0; k < NS; ++k) hist_add(tc->hist[k], ck[k]);
        if (tc->hn < (1 << 20)) ++tc->hn;
    }
    return o;
}

size_t fdvb_image_blob(const fdvb_streams *st, int w, int h, int qp,
                       uint8_t *out, size_t cap, int *emode_out) {
    const int N = IS_N;
    const size_t *sn = st->n;
    size_t total = 0;
    for (int k = 0; k < N; ++k) total += sn[k];
    std::vector<uint8_t> all(total ? total : 1);
    {
        size_t o = 0;
        for (int k = 0; k < N; ++k) { if (sn[k]) memcpy(all.data() + o, st->s[k], sn[k]); o += sn[k]; }
    }
    uint32_t ck[IS_N][256];
    for (int k = 0; k < N; ++k) {
        if (st->hist) memcpy(ck[k], st->hist + (size_t)k * 256, sizeof ck[k]);
        else {
            memset(ck[k], 0, sizeof ck[k]);
            for (size_t i = 0; i < sn[k]; ++i) ck[k][st->s[k][i]]++;
        }
    }
    uint32_t c1[256] = {0};
    for (int k = 0; k < N; ++k)
        for (int v = 0; v < 256; ++v) c1[v] += ck[k][v];
    uint16_t f1[256];
    freqs_from_counts(c1, f1);
    std::vector<uint8_t> p1;
    size_t l1 = rans_encode(all.data(), total, f1, p1);
    uint16_t fk[IS_N][256];
    std::vector<uint8_t> pay[IS_N];
    size_t len[IS_N];
    for (int k = 0; k < N; ++k) {
        freqs_from_counts(ck[k], fk[k]);
        len[k] = rans_encode(st->s[k], sn[k], fk[k], pay[k]);
    }
    size_t hdr = 0;
    for (int k = 0; k < N; ++k) hdr += (size_t)fdvb_leb_size((uint32_t)sn[k]);
    size_t size_one = hdr + freqs_size(f1) + (size_t)fdvb_leb_size((uint32_t)l1) + l1;
    size_t size_two = hdr;
    for (int k = 0; k < N; ++k) {
        if (sn[k] == 0) continue;
        size_two += freqs_size(fk[k]) + (size_t)fdvb_leb_size((uint32_t)len[k]) + len[k];
    }
    size_t size_ada = (size_t)-1, lada = 0;
    AEnc ae(total * 3 + 4096);
    {
        uint32_t flat[256] = {0};
        for (int k = 0; k < N; ++k) {
            AModel m;
            m.init(flat);
            for (size_t i = 0; i < sn[k]; ++i) ae.sym(m, st->s[k][i]);
        }
        lada = ae.finish();
        if (lada) size_ada = hdr + (size_t)fdvb_leb_size((uint32_t)lada) + lada;
    }
    int imode = 0;
    size_t best = size_one;
    if (size_two < best) { best = size_two; imode = 1; }
    if (size_ada < best) { best = size_ada; imode = 2; }
    if (emode_out) *emode_out = imode == 2 ? 3 : imode;
    if (5 + best > cap) return 0;
    size_t o = 0;
    o = fdvb_put16(out, o, (unsigned)w);
    o = fdvb_put16(out, o, (unsigned)h);
    out[o++] = (uint8_t)qp;
    out[o++] = (uint8_t)imode;
    for (int k = 0; k < N; ++k) o = fdvb_leb_put(out, o, (uint32_t)sn[k]);
    if (imode == 2) {
        o = fdvb_leb_put(out, o, (uint32_t)lada);
        memcpy(out + o, ae.out.data(), lada); o += lada;
    } else if (imode == 0) {
        o = write_freqs(out, o, f1);
        o = fdvb_leb_put(out, o, (uint32_t)l1);
        memcpy(out + o, p1.data(), l1); o += l1;
    } else {
        for (int k = 0; k < N; ++k) {
            if (sn[k] == 0) continue;
            o = write_freqs(out, o, fk[k]);
            o = fdvb_leb_put(out, o, (uint32_t)len[k]);
            memcpy(out + o, pay[k].data(), len[k]); o += len[k];
        }
    }
    return o;
}

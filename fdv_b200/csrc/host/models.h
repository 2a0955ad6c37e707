// Entropy models shared by the encoder's tail (entropy.cpp) and the decoder's
// stream reader (decode.cpp): the rANS scale, the adaptive coder's Fenwick
// frequency model (fdv.h:2003-2078) and its budgeted stream choice
// (fdv.h:482-499), and the table cache's history and cached-table forms
// (fdv.h:5641-5677), restated.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

namespace fdvb {
namespace ent {

inline constexpr uint32_t kScaleBits = 12;
inline constexpr uint32_t kScale = 1u << kScaleBits;
inline constexpr uint32_t kRansLow = 1u << 23;
inline constexpr size_t kAdBudget = 65536;
inline constexpr uint32_t kAdInc = 128, kAdBase = 1, kAdScale = 8192, kAdMax = 65536;
inline constexpr uint64_t kAdHist = 1u << 21;

struct AModel {
    uint32_t f[256];
    uint32_t t[257];
    uint32_t tot;
    void build() {
        uint32_t s = 0;
        t[0] = 0;
        for (int i = 0; i < 256; ++i) { t[i + 1] = f[i]; s += f[i]; }
        for (int i = 1; i <= 256; ++i) {
            int j = i + (i & -i);
            if (j <= 256) t[j] += t[i];
        }
        tot = s;
    }
    void init(const uint32_t hist[256]) {
        uint64_t s = 0;
        for (int i = 0; i < 256; ++i) s += hist[i];
        if (s <= kAdScale)
            for (int i = 0; i < 256; ++i) f[i] = kAdBase + hist[i];
        else
            for (int i = 0; i < 256; ++i)
                f[i] = kAdBase + (uint32_t)(((uint64_t)hist[i] * kAdScale + s / 2) / s);
        build();
    }
    uint32_t cum(unsigned s) const {
        uint32_t r = 0;
        for (int i = (int)s; i > 0; i -= i & -i) r += t[i];
        return r;
    }
    void add(unsigned s, uint32_t d) {
        f[s] += d;
        tot += d;
        if (tot > kAdMax) {
            for (int i = 0; i < 256; ++i) f[i] = (f[i] + 1) >> 1;
            build();
            return;
        }
        for (int i = (int)s + 1; i <= 256; i += i & -i) t[i] += d;
    }
};


inline unsigned ad_select(const size_t *sn, int ns, size_t *total) {
    int order[16];
    for (int i = 0; i < ns; ++i) order[i] = i;
    for (int i = 1; i < ns; ++i)
        for (int j = i; j > 0 && sn[order[j]] < sn[order[j - 1]]; --j) {
            int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t;
        }
    unsigned mask = 0;
    size_t tot = 0;
    for (int i = 0; i < ns; ++i) {
        int k = order[i];
        if (!sn[k] || tot + sn[k] > kAdBudget) continue;
        mask |= 1u << k;
        tot += sn[k];
    }
    if (total) *total = tot;
    return mask;
}

inline void hist_add(uint32_t h[256], const uint32_t c[256]) {
    uint64_t s = 0;
    for (int i = 0; i < 256; ++i) { h[i] += c[i]; s += h[i]; }
    if (s > kAdHist) for (int i = 0; i < 256; ++i) h[i] >>= 1;
}

inline void tab_store(uint16_t dst[256], const uint16_t src[256]) {
    int add = 0, big = 0;
    for (int i = 0; i < 256; ++i) {
        if (!src[i]) ++add;
        if (src[i] > src[big]) big = i;
    }
    if (src[big] <= (uint16_t)add) { memcpy(dst, src, 256 * sizeof *dst); return; }
    for (int i = 0; i < 256; ++i) dst[i] = src[i] ? src[i] : 1;
    dst[big] = (uint16_t)(dst[big] - add);
}

}  // namespace ent
}  // namespace fdvb

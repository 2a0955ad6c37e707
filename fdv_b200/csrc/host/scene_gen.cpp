// Seeded synthetic I420 content for the encoder benchmarks and parity tests.
//
// The reference benchmarks on its own scene renderer (include/fdv_scene.h); the
// workloads this library is measured on specify their own generator instead: a
// band-limited noise background (Gaussian noise low-passed with sigma 3 px,
// luma mean 128 / sd 30, chroma sd 10), textured rectangles moving at constant
// quarter-pel velocities, an optional global pan, and an optional static
// textured region so SKIP is common.  Everything here is integer arithmetic on
// a splitmix64 stream, so a (params, seed) pair renders the same bytes on every
// machine; moving content is resampled with the H.264 six-tap quarter-pel
// filter (luma) and eighth-pel bilinear (chroma) so a true motion vector exists.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fdvb_internal.h"

namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    int uniform(int lo, int hi) {  // inclusive
        return lo + (int)(next() % (uint64_t)(hi - lo + 1));
    }
};

// Integer Gaussian kernel, sigma = 3 px, radius 9: round(4096 * exp(-k^2 / 18)).
const int kBlur[10] = {4096, 3855, 3210, 2365, 1542, 889, 453, 204, 81, 29};

// A texture: w x h bytes with the requested mean and standard deviation.
struct Tex {
    int w = 0, h = 0;
    std::vector<uint8_t> px;
    uint8_t at(int x, int y) const {
        x = x < 0 ? 0 : (x >= w ? w - 1 : x);
        y = y < 0 ? 0 : (y >= h ? h - 1 : y);
        return px[(size_t)y * w + x];
    }
};

int64_t isqrt64(int64_t v) {
    if (v <= 0) return 0;
    int64_t r = 0, bit = (int64_t)1 << 62;
    while (bit > v) bit >>= 2;
    while (bit) {
        if (v >= r + bit) { v -= r + bit; r = (r >> 1) + bit; }
        else r >>= 1;
        bit >>= 2;
    }
    return r;
}

// Mirror an index into [0, n) (one reflection, then clamped for tiny n).
inline int reflect(int i, int n) {
    i = i < 0 ? -i : (i >= n ? 2 * n - 2 - i : i);
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// Gaussian-ish white noise (sum of four uniforms), low-passed by the separable
// kernel above, then mapped affinely to (mean, sd) and clipped to [0, 255].
Tex make_noise_tex(Rng &rng, int w, int h, int mean, int sd) {
    Tex t; t.w = w; t.h = h; t.px.resize((size_t)w * h);
    std::vector<int32_t> n((size_t)w * h), a((size_t)w * h);
    for (auto &v : n) {
        uint64_t r = rng.next();
        int s = (int)(r & 0xffff) + (int)((r >> 16) & 0xffff) + (int)((r >> 32) & 0xffff) +
                (int)((r >> 48) & 0xffff) - 2 * 65535;
        v = s >> 4;                                   // keep products in int32 range
    }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int64_t acc = 0;
            for (int k = -9; k <= 9; ++k) {
                int xx = reflect(x + k, w);
                acc += (int64_t)kBlur[k < 0 ? -k : k] * n[(size_t)y * w + xx];
            }
            a[(size_t)y * w + x] = (int32_t)(acc >> 12);
        }
    int64_t sum = 0, sumsq = 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int64_t acc = 0;
            for (int k = -9; k <= 9; ++k) {
                int yy = reflect(y + k, h);
                acc += (int64_t)kBlur[k < 0 ? -k : k] * a[(size_t)yy * w + x];
            }
            int32_t v = (int32_t)(acc >> 12);
            n[(size_t)y * w + x] = v;
            sum += v;
            sumsq += (int64_t)v * v;
        }
    int64_t cnt = (int64_t)w * h;
    int64_t mu = sum / cnt;
    int64_t var = sumsq / cnt - mu * mu;
    int64_t stdv = isqrt64(var);
    if (stdv < 1) stdv = 1;
    for (size_t i = 0; i < t.px.size(); ++i) {
        int64_t d = (int64_t)(n[i] - mu) * sd * 2;
        int64_t q = d >= 0 ? (d + stdv) / (2 * stdv) : -((-d + stdv) / (2 * stdv));
        int64_t v = mean + q;
        t.px[i] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
    }
    return t;
}

inline int clip8(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
inline int tap6(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}

// H.264 quarter-pel luma sample of texture t at (x + fx/4, y + fy/4).
int sample_qpel(const Tex &t, int x, int y, int fx, int fy) {
    auto P = [&](int xx, int yy) { return (int)t.at(xx, yy); };
    auto hf = [&](int xx, int yy) {
        return tap6(P(xx - 2, yy), P(xx - 1, yy), P(xx, yy), P(xx + 1, yy), P(xx + 2, yy), P(xx + 3, yy));
    };
    auto vf = [&](int xx, int yy) {
        return tap6(P(xx, yy - 2), P(xx, yy - 1), P(xx, yy), P(xx, yy + 1), P(xx, yy + 2), P(xx, yy + 3));
    };
    auto hb = [&](int xx, int yy) { return clip8((hf(xx, yy) + 16) >> 5); };
    auto hh = [&](int xx, int yy) { return clip8((vf(xx, yy) + 16) >> 5); };
    auto hj = [&](int xx, int yy) {
        int jj = tap6(hf(xx, yy - 2), hf(xx, yy - 1), hf(xx, yy), hf(xx, yy + 1), hf(xx, yy + 2), hf(xx, yy + 3));
        return clip8((jj + 512) >> 10);
    };
    switch (fy * 4 + fx) {
    case 0: return P(x, y);
    case 1: return (P(x, y) + hb(x, y) + 1) >> 1;
    case 2: return hb(x, y);
    case 3: return (hb(x, y) + P(x + 1, y) + 1) >> 1;
    case 4: return (P(x, y) + hh(x, y) + 1) >> 1;
    case 5: return (hb(x, y) + hh(x, y) + 1) >> 1;
    case 6: return (hb(x, y) + hj(x, y) + 1) >> 1;
    case 7: return (hb(x, y) + hh(x + 1, y) + 1) >> 1;
    case 8: return hh(x, y);
    case 9: return (hh(x, y) + hj(x, y) + 1) >> 1;
    case 10: return hj(x, y);
    case 11: return (hj(x, y) + hh(x + 1, y) + 1) >> 1;
    case 12: return (hh(x, y) + P(x, y + 1) + 1) >> 1;
    case 13: return (hh(x, y) + hb(x, y + 1) + 1) >> 1;
    case 14: return (hj(x, y) + hb(x, y + 1) + 1) >> 1;
    default: return (hh(x + 1, y) + hb(x, y + 1) + 1) >> 1;
    }
}

// Eighth-pel bilinear chroma sample of texture t at (x + fx/8, y + fy/8).
int sample_epel(const Tex &t, int x, int y, int fx, int fy) {
    int a = t.at(x, y), b = t.at(x + 1, y), c = t.at(x, y + 1), d = t.at(x + 1, y + 1);
    return ((a * (8 - fx) + b * fx) * (8 - fy) + (c * (8 - fx) + d * fx) * fy + 32) >> 6;
}

// Floor division / modulo for possibly negative quarter-pel positions.
inline int fdiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
inline int fmod_pos(int a, int b) { int r = a % b; return r < 0 ? r + b : r; }

struct Rect {
    int sw, sh;          // size in luma px (even)
    int x0, y0;          // start position, quarter-pel (luma)
    int vx, vy;          // velocity, quarter-pel per frame
    Tex ty, tu, tv;
};

}  // namespace

struct fdvb_scene_state {
    fdvb_scene_params p;
    Tex bgy, bgu, bgv;          // background canvases
    Tex sty, stu, stv;          // static region textures
    int stx = 0, sty_ = 0, stw = 0, sth = 0;   // static region rect (luma px, even)
    std::vector<Rect> rects;
};

// Position along one axis after f frames of constant velocity v starting at s,
// reflecting at [0, span] (all in quarter-pel).
static int bounce(int s, int v, int f, int span) {
    if (span <= 0) return 0;
    long long p = (long long)s + (long long)v * f;
    long long period = 2LL * span;
    long long m = p % period; if (m < 0) m += period;
    return (int)(m <= span ? m : period - m);
}

extern "C" fdvb_scene_state *fdvb_scene_open(const fdvb_scene_params *params) {
    if (!params || params->w <= 0 || params->h <= 0 || (params->w & 1) || (params->h & 1)) return nullptr;
    auto *s = new fdvb_scene_state();
    s->p = *params;
    Rng rng{params->seed * 0x2545F4914F6CDD1Dull + 1};
    const auto &p = s->p;
    int nf = p.nframes > 0 ? p.nframes : 1;
    int panx = (abs(p.pan_qx) * nf) / 4 + 16, pany = (abs(p.pan_qy) * nf) / 4 + 16;
    int cwid = p.w + panx + 16, chgt = p.h + pany + 16;
    s->bgy = make_noise_tex(rng, cwid, chgt, 128, 30);
    s->bgu = make_noise_tex(rng, cwid / 2 + 8, chgt / 2 + 8, 128, 10);
    s->bgv = make_noise_tex(rng, cwid / 2 + 8, chgt / 2 + 8, 128, 10);
    if (p.static_pct > 0) {
        // A fixed rectangle of (static_pct)% of the frame, same aspect as the frame.
        long long area = (long long)p.w * p.h * p.static_pct / 100;
        int sw = (int)isqrt64(area * p.w / p.h);
        sw &= ~15; if (sw > p.w) sw = p.w & ~15;
        int sh = sw > 0 ? (int)(area / sw) : 0;
        sh &= ~15; if (sh > p.h) sh = p.h & ~15;
        s->stw = sw; s->sth = sh;
        s->stx = ((p.w - sw) / 4) & ~1;
        s->sty_ = ((p.h - sh) / 4) & ~1;
        if (sw > 0 && sh > 0) {
            s->sty = make_noise_tex(rng, sw, sh, rng.uniform(70, 190), 30);
            s->stu = make_noise_tex(rng, sw / 2, sh / 2, rng.uniform(100, 156), 10);
            s->stv = make_noise_tex(rng, sw / 2, sh / 2, rng.uniform(100, 156), 10);
        }
    }
    for (int i = 0; i < p.nrects; ++i) {
        Rect r;
        r.sw = rng.uniform(p.rect_min, p.rect_max) & ~1;
        r.sh = rng.uniform(p.rect_min, p.rect_max) & ~1;
        if (r.sw < 2) r.sw = 2;
        if (r.sh < 2) r.sh = 2;
        int spanx = (p.w - r.sw) * 4, spany = (p.h - r.sh) * 4;
        r.x0 = spanx > 0 ? rng.uniform(0, spanx) : 0;
        r.y0 = spany > 0 ? rng.uniform(0, spany) : 0;
        r.vx = rng.uniform(-p.vmax_qpel, p.vmax_qpel);
        r.vy = rng.uniform(-p.vmax_qpel, p.vmax_qpel);
        r.ty = make_noise_tex(rng, r.sw + 8, r.sh + 8, rng.uniform(50, 206), 30);
        r.tu = make_noise_tex(rng, r.sw / 2 + 4, r.sh / 2 + 4, rng.uniform(90, 166), 10);
        r.tv = make_noise_tex(rng, r.sw / 2 + 4, r.sh / 2 + 4, rng.uniform(90, 166), 10);
        s->rects.push_back(std::move(r));
    }
    return s;
}

extern "C" void fdvb_scene_close(fdvb_scene_state *s) { delete s; }

extern "C" int fdvb_scene_frame(const fdvb_scene_state *s, int f, uint8_t *i420) {
    if (!s || !i420 || f < 0) return -1;
    const auto &p = s->p;
    int w = p.w, h = p.h, cw = w / 2, ch = h / 2;
    uint8_t *Y = i420, *U = Y + (size_t)w * h, *V = U + (size_t)cw * ch;
    // Background: the canvas seen through a window that pans by (pan_qx, pan_qy)
    // quarter-pels per frame.  The window starts at the canvas position that
    // keeps every frame's window inside the canvas.
    int ox = p.pan_qx >= 0 ? 8 * 4 : ((s->bgy.w - w - 8) * 4);
    int oy = p.pan_qy >= 0 ? 8 * 4 : ((s->bgy.h - h - 8) * 4);
    int qx = ox + p.pan_qx * f, qy = oy + p.pan_qy * f;
    int ix = fdiv(qx, 4), iy = fdiv(qy, 4), fx = fmod_pos(qx, 4), fy = fmod_pos(qy, 4);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
            Y[(size_t)y * w + x] = (uint8_t)sample_qpel(s->bgy, ix + x, iy + y, fx, fy);
    // Chroma moves half as far in its own pels: quarter-pel luma = eighth-pel chroma.
    int cix = fdiv(qx, 8), ciy = fdiv(qy, 8), cfx = fmod_pos(qx, 8), cfy = fmod_pos(qy, 8);
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) {
            U[(size_t)y * cw + x] = (uint8_t)sample_epel(s->bgu, cix + x, ciy + y, cfx, cfy);
            V[(size_t)y * cw + x] = (uint8_t)sample_epel(s->bgv, cix + x, ciy + y, cfx, cfy);
        }
    // Moving rectangles, drawn in order.
    for (const Rect &r : s->rects) {
        int px = bounce(r.x0, r.vx, f, (w - r.sw) * 4);
        int py = bounce(r.y0, r.vy, f, (h - r.sh) * 4);
        int rx = px >> 2, ry = py >> 2, rfx = px & 3, rfy = py & 3;
        // The rectangle occupies integer pels [rx, rx+sw) x [ry, ry+sh); the
        // texture is sampled at the sub-pel offset so it moves smoothly.
        for (int y = 0; y < r.sh; ++y)
            for (int x = 0; x < r.sw; ++x) {
                int X = rx + x, Yy = ry + y;
                if (X < 0 || X >= w || Yy < 0 || Yy >= h) continue;
                Y[(size_t)Yy * w + X] = (uint8_t)sample_qpel(r.ty, x + 4 - (rfx ? 1 : 0), y + 4 - (rfy ? 1 : 0),
                                                             rfx ? 4 - rfx : 0, rfy ? 4 - rfy : 0);
            }
        int cpx = px / 2, cpy = py / 2;            // eighth-pel chroma position
        int crx = cpx >> 3, cry = cpy >> 3, cfx2 = cpx & 7, cfy2 = cpy & 7;
        for (int y = 0; y < r.sh / 2; ++y)
            for (int x = 0; x < r.sw / 2; ++x) {
                int X = crx + x, Yy = cry + y;
                if (X < 0 || X >= cw || Yy < 0 || Yy >= ch) continue;
                int sx = x + 2 - (cfx2 ? 1 : 0), sy = y + 2 - (cfy2 ? 1 : 0);
                int ex = cfx2 ? 8 - cfx2 : 0, ey = cfy2 ? 8 - cfy2 : 0;
                U[(size_t)Yy * cw + X] = (uint8_t)sample_epel(r.tu, sx, sy, ex, ey);
                V[(size_t)Yy * cw + X] = (uint8_t)sample_epel(r.tv, sx, sy, ex, ey);
            }
    }
    // The static region is drawn last, so nothing moves across it.
    if (s->stw > 0 && s->sth > 0) {
        for (int y = 0; y < s->sth; ++y)
            memcpy(Y + (size_t)(s->sty_ + y) * w + s->stx, &s->sty.px[(size_t)y * s->stw], s->stw);
        for (int y = 0; y < s->sth / 2; ++y) {
            memcpy(U + (size_t)(s->sty_ / 2 + y) * cw + s->stx / 2, &s->stu.px[(size_t)y * (s->stw / 2)], s->stw / 2);
            memcpy(V + (size_t)(s->sty_ / 2 + y) * cw + s->stx / 2, &s->stv.px[(size_t)y * (s->stw / 2)], s->stw / 2);
        }
    }
    return 0;
}

// ------------------------------------------------------------------------
// Camera-like stress content: a fractal canvas seen through a window that pans
// and zooms by a fixed factor per frame, many small textured objects moving
// fast across it, additive sensor noise, and a hard cut to a new canvas and
// new objects every cut_every frames.  Integer arithmetic throughout, like the
// generator above, so a (params, seed) pair renders the same bytes anywhere.
namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sum of value-noise octaves whose amplitude is proportional to the lattice
// spacing (amplitude ~ 1/f, power ~ 1/f^2), spacings 2^kmax down to 2 px,
// bilinear between lattice points; mapped to (mean, sd) and clipped.
Tex make_fractal_tex(uint64_t seed, int w, int h, int kmax, int mean, int sd) {
    Tex t; t.w = w; t.h = h; t.px.resize((size_t)w * h);
    std::vector<int32_t> acc((size_t)w * h, 0);
    for (int k = kmax; k >= 1; --k) {
        const int c = 1 << k;
        const int gw = w / c + 2, gh = h / c + 2;
        std::vector<int32_t> lat((size_t)gw * gh);
        for (int j = 0; j < gh; ++j)
            for (int i = 0; i < gw; ++i)
                lat[(size_t)j * gw + i] =
                    (int32_t)(mix64(seed ^ ((uint64_t)k << 56) ^ ((uint64_t)j << 28) ^ (uint64_t)i) & 2047) - 1024;
        for (int y = 0; y < h; ++y) {
            const int j = y >> k, fy = y & (c - 1);
            for (int x = 0; x < w; ++x) {
                const int i = x >> k, fx = x & (c - 1);
                const int32_t *l0 = &lat[(size_t)j * gw + i], *l1 = l0 + gw;
                const int64_t top = (int64_t)l0[0] * (c - fx) + (int64_t)l0[1] * fx;
                const int64_t bot = (int64_t)l1[0] * (c - fx) + (int64_t)l1[1] * fx;
                // (bilinear value x c^2) x amplitude c / c^2
                acc[(size_t)y * w + x] += (int32_t)((top * (c - fy) + bot * fy) >> k);
            }
        }
    }
    int64_t sum = 0, sumsq = 0;
    for (int32_t v : acc) { sum += v; sumsq += (int64_t)v * v; }
    const int64_t cnt = (int64_t)w * h, mu = sum / cnt;
    int64_t stdv = isqrt64(sumsq / cnt - mu * mu);
    if (stdv < 1) stdv = 1;
    for (size_t i = 0; i < t.px.size(); ++i) {
        const int64_t d = (int64_t)(acc[i] - mu) * sd * 2;
        const int64_t q = d >= 0 ? (d + stdv) / (2 * stdv) : -((-d + stdv) / (2 * stdv));
        t.px[i] = (uint8_t)clip8((int)(mean + q));
    }
    return t;
}

// Additive noise of standard deviation sd_x16 / 16 at index i of frame f: the
// sum of four 16-bit uniforms (sd 65536 / sqrt(3)) scaled and rounded.
inline int sensor_noise(uint64_t key, int f, size_t i, int sd_x16) {
    if (sd_x16 <= 0) return 0;
    const uint64_t r = mix64(key ^ ((uint64_t)f << 40) ^ (uint64_t)i);
    const int64_t s = (int64_t)(r & 0xffff) + (int64_t)((r >> 16) & 0xffff) + (int64_t)((r >> 32) & 0xffff) +
                      (int64_t)((r >> 48) & 0xffff) - 2 * 65535;
    const int64_t num = s * sd_x16, den = (int64_t)16 * 37837;   // 37837 = 65536 / sqrt(3)
    return (int)(num >= 0 ? (num + den / 2) / den : -((-num + den / 2) / den));
}

// Bilinear sample of t at Q16.16 position (X, Y), clamped to the texture.
inline int sample_q16(const Tex &t, int64_t X, int64_t Y) {
    const int ix = (int)(X >> 16), iy = (int)(Y >> 16);
    const int fx = (int)((X >> 8) & 255), fy = (int)((Y >> 8) & 255);
    const int a = t.at(ix, iy), b = t.at(ix + 1, iy), c = t.at(ix, iy + 1), d = t.at(ix + 1, iy + 1);
    return (((a * (256 - fx) + b * fx) * (256 - fy) + (c * (256 - fx) + d * fx) * fy) + 32768) >> 16;
}

struct CamSegment {
    Tex cy, cu, cv;                   // canvases (chroma at half resolution)
    int64_t cx0 = 0, cy0 = 0;         // view centre at the segment's first frame, Q16.16 luma canvas px
    bool zoom_in = true;
    std::vector<Rect> objs;
};

}  // namespace

struct fdvb_camscene_state {
    fdvb_camscene_params p;
    std::vector<CamSegment> seg;
};

extern "C" fdvb_camscene_state *fdvb_camscene_open(const fdvb_camscene_params *params) {
    if (!params || params->w <= 0 || params->h <= 0 || (params->w & 1) || (params->h & 1) || params->nframes <= 0 ||
        params->zoom_ppm < 0 || params->zoom_ppm > 100000 || params->obj_min < 2 || params->obj_max < params->obj_min ||
        params->nobjects < 0 || params->cut_every < 0)
        return nullptr;
    auto *s = new fdvb_camscene_state();
    s->p = *params;
    const auto &p = s->p;
    const int L = p.cut_every > 0 ? std::min(p.cut_every, p.nframes) : p.nframes;
    const int nseg = p.cut_every > 0 ? (p.nframes + p.cut_every - 1) / p.cut_every : 1;
    // widest view of a segment (zooming out L - 1 frames), in luma px
    int64_t inv = 65536;
    for (int t = 1; t < L; ++t) inv = inv * (1000000 + p.zoom_ppm) / 1000000;
    const int vw = (int)(((int64_t)p.w * inv) >> 16) + 8, vh = (int)(((int64_t)p.h * inv) >> 16) + 8;
    const int panx = (int)(((int64_t)abs(p.pan_qx) * L) / 4) + 8, pany = (int)(((int64_t)abs(p.pan_qy) * L) / 4) + 8;
    const int W = (vw + panx + 32) & ~1, H = (vh + pany + 32) & ~1;
    for (int g = 0; g < nseg; ++g) {
        CamSegment S;
        const uint64_t gs = mix64(p.seed * 0x2545F4914F6CDD1Dull + (uint64_t)g * 0x9E37ull + 7);
        S.cy = make_fractal_tex(gs ^ 1, W, H, 8, 128, 40);
        S.cu = make_fractal_tex(gs ^ 2, W / 2 + 4, H / 2 + 4, 7, 128, 14);
        S.cv = make_fractal_tex(gs ^ 3, W / 2 + 4, H / 2 + 4, 7, 128, 14);
        S.zoom_in = (g & 1) == 0;
        // start so every frame's view stays inside the canvas
        const int64_t x0 = p.pan_qx >= 0 ? 16 + vw / 2 : W - 16 - vw / 2;
        const int64_t y0 = p.pan_qy >= 0 ? 16 + vh / 2 : H - 16 - vh / 2;
        S.cx0 = x0 << 16;
        S.cy0 = y0 << 16;
        Rng rng{gs};
        for (int i = 0; i < p.nobjects; ++i) {
            Rect r;
            r.sw = std::max(2, rng.uniform(p.obj_min, p.obj_max) & ~1);
            r.sh = std::max(2, rng.uniform(p.obj_min, p.obj_max) & ~1);
            const int spanx = (p.w - r.sw) * 4, spany = (p.h - r.sh) * 4;
            r.x0 = spanx > 0 ? rng.uniform(0, spanx) : 0;
            r.y0 = spany > 0 ? rng.uniform(0, spany) : 0;
            r.vx = rng.uniform(-p.vmax_qpel, p.vmax_qpel);
            r.vy = rng.uniform(-p.vmax_qpel, p.vmax_qpel);
            r.ty = make_noise_tex(rng, r.sw + 8, r.sh + 8, rng.uniform(40, 216), 30);
            r.tu = make_noise_tex(rng, r.sw / 2 + 4, r.sh / 2 + 4, rng.uniform(80, 176), 12);
            r.tv = make_noise_tex(rng, r.sw / 2 + 4, r.sh / 2 + 4, rng.uniform(80, 176), 12);
            S.objs.push_back(std::move(r));
        }
        s->seg.push_back(std::move(S));
    }
    return s;
}

extern "C" void fdvb_camscene_close(fdvb_camscene_state *s) { delete s; }

extern "C" int fdvb_camscene_frame(const fdvb_camscene_state *s, int f, uint8_t *i420) {
    if (!s || !i420 || f < 0 || f >= s->p.nframes) return -1;
    const auto &p = s->p;
    const int g = p.cut_every > 0 ? f / p.cut_every : 0, t = p.cut_every > 0 ? f - g * p.cut_every : f;
    const CamSegment &S = s->seg[(size_t)g];
    const int w = p.w, h = p.h, cw = w / 2, ch = h / 2;
    uint8_t *Y = i420, *U = Y + (size_t)w * h, *V = U + (size_t)cw * ch;
    // canvas px per output px after t frames of zoom, Q16.16
    int64_t inv = 65536;
    for (int k = 0; k < t; ++k)
        inv = S.zoom_in ? inv * 1000000 / (1000000 + p.zoom_ppm) : inv * (1000000 + p.zoom_ppm) / 1000000;
    const int64_t cx = S.cx0 + (int64_t)p.pan_qx * t * 16384, cy = S.cy0 + (int64_t)p.pan_qy * t * 16384;
    const uint64_t nkey = mix64(p.seed ^ 0x5EED5EEDull);
    for (int y = 0; y < h; ++y) {
        const int64_t Yq = cy + (int64_t)(2 * y + 1 - h) * inv / 2;
        for (int x = 0; x < w; ++x) {
            const int64_t Xq = cx + (int64_t)(2 * x + 1 - w) * inv / 2;
            Y[(size_t)y * w + x] = (uint8_t)sample_q16(S.cy, Xq, Yq);
        }
    }
    for (int y = 0; y < ch; ++y) {
        const int64_t Yq = cy / 2 + (int64_t)(2 * y + 1 - ch) * inv / 2;
        for (int x = 0; x < cw; ++x) {
            const int64_t Xq = cx / 2 + (int64_t)(2 * x + 1 - cw) * inv / 2;
            U[(size_t)y * cw + x] = (uint8_t)sample_q16(S.cu, Xq, Yq);
            V[(size_t)y * cw + x] = (uint8_t)sample_q16(S.cv, Xq, Yq);
        }
    }
    // objects: constant quarter-pel velocities, bouncing, drawn in order
    for (const Rect &r : S.objs) {
        const int px = bounce(r.x0, r.vx, t, (w - r.sw) * 4), py = bounce(r.y0, r.vy, t, (h - r.sh) * 4);
        const int rx = px >> 2, ry = py >> 2, rfx = px & 3, rfy = py & 3;
        for (int y = 0; y < r.sh; ++y)
            for (int x = 0; x < r.sw; ++x) {
                const int X = rx + x, Yy = ry + y;
                if (X < 0 || X >= w || Yy < 0 || Yy >= h) continue;
                Y[(size_t)Yy * w + X] = (uint8_t)sample_qpel(r.ty, x + 4 - (rfx ? 1 : 0), y + 4 - (rfy ? 1 : 0),
                                                             rfx ? 4 - rfx : 0, rfy ? 4 - rfy : 0);
            }
        const int cpx = px / 2, cpy = py / 2;
        const int crx = cpx >> 3, cry = cpy >> 3, cfx = cpx & 7, cfy = cpy & 7;
        for (int y = 0; y < r.sh / 2; ++y)
            for (int x = 0; x < r.sw / 2; ++x) {
                const int X = crx + x, Yy = cry + y;
                if (X < 0 || X >= cw || Yy < 0 || Yy >= ch) continue;
                const int sx = x + 2 - (cfx ? 1 : 0), sy = y + 2 - (cfy ? 1 : 0);
                const int ex = cfx ? 8 - cfx : 0, ey = cfy ? 8 - cfy : 0;
                U[(size_t)Yy * cw + X] = (uint8_t)sample_epel(r.tu, sx, sy, ex, ey);
                V[(size_t)Yy * cw + X] = (uint8_t)sample_epel(r.tv, sx, sy, ex, ey);
            }
    }
    // sensor noise on every sample
    const size_t ny = (size_t)w * h, nc = (size_t)cw * ch;
    for (size_t i = 0; i < ny; ++i) Y[i] = (uint8_t)clip8(Y[i] + sensor_noise(nkey, f, i, p.noise_y_x16));
    for (size_t i = 0; i < 2 * nc; ++i) U[i] = (uint8_t)clip8(U[i] + sensor_noise(nkey ^ 0xC0ull, f, i, p.noise_c_x16));
    return 0;
}

// The public C ABI of libfdvb200: the fdv.h encode entry points on top of the
// batched GPU engine, the inner engine ABI, the host entropy tail and the
// synthetic content generator (include/fdv_b200.h).
//
// The stream containers written here follow the reference byte for byte:
//   video stream     [nframes u16][w u16][h u16][qp u8][keyint u8] then per
//                    frame [blob_len u32][blob]                     fdv.h:6764-6805
//   key-frame blob   three [len u32][intra plane blob], Y U V       fdv.h:5529-5538
//   tiled container  [w u16][h u16][nframes u16][qp u8][keyint u8][nbands u16]
//                    [band_mbrows u16] then per band [len u32][video stream]
//                                                                   fdv.h:7098-7101, :7174-7236
//   file head        "FDV1" [version u8][kind u8][fps u16][payload_len u32]
//                                                                   fdv.h:7448-7464
#include <algorithm>
#include <deque>
#include <cmath>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <map>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "fdvb_internal.h"

namespace {

thread_local std::string g_api_err;
int g_range = 16;
int g_device = 0;

void set_err(const char *m) { g_api_err = m; }
void set_engine_err() { g_api_err = std::string("engine: ") + fdvb_engine_error(); }

// One unit's host-side stream state: the entropy cache and the coded bytes.
struct UnitStream {
    std::unique_ptr<fdvb_tabcache> tc{new fdvb_tabcache()};
    std::vector<uint8_t> bytes;
    int w = 0, h = 0;
    size_t tmp_cap = 0;
    std::vector<uint8_t> tmp;
    int fail = 0;
};

void stream_header(std::vector<uint8_t> &b, int nframes, int w, int h, int qp, int keyint) {
    uint8_t hd[8];
    size_t o = 0;
    o = fdvb_put16(hd, o, (unsigned)nframes);
    o = fdvb_put16(hd, o, (unsigned)w);
    o = fdvb_put16(hd, o, (unsigned)h);
    hd[o++] = (uint8_t)qp;
    hd[o++] = (uint8_t)keyint;
    b.insert(b.end(), hd, hd + o);
}

// Entropy-code unit u's analysis output of the engine's last step into
// us.tmp; returns the blob length (0 on failure).
// The blob of one unit-frame from its streams (P-frame: s[0]; key frame:
// s[0..2], the planes).
size_t code_blob_streams(const fdvb_streams *s, UnitStream &us, int is_intra, int qp) {
    size_t blob = 0;
    if (us.tmp.size() < us.tmp_cap) us.tmp.resize(us.tmp_cap);
    if (is_intra) {
        memset(us.tc.get(), 0, sizeof(fdvb_tabcache));
        const int pw[3] = {us.w, us.w / 2, us.w / 2}, ph[3] = {us.h, us.h / 2, us.h / 2};
        size_t o = 0;
        for (int p = 0; p < 3; ++p) {
            size_t bcap = (size_t)pw[p] * ph[p] * 2 + 4096;
            std::vector<uint8_t> pb(bcap);
            size_t bl = fdvb_image_blob(&s[p], pw[p], ph[p], qp, pb.data(), bcap, nullptr);
            if (!bl || o + 4 + bl > us.tmp_cap) return 0;
            o = fdvb_put32(us.tmp.data(), o, (uint32_t)bl);
            memcpy(us.tmp.data() + o, pb.data(), bl);
            o += bl;
        }
        blob = o;
    } else {
        blob = fdvb_pframe_blob(&s[0], qp, us.tc.get(), us.tmp.data(), us.tmp_cap, nullptr);
    }
    return blob;
}

size_t code_unit_blob(fdvb_engine *E, int u, UnitStream &us, int is_intra, int qp) {
    size_t blob = 0;
    if (us.tmp.size() < us.tmp_cap) us.tmp.resize(us.tmp_cap);
    if (is_intra) {
        // A key frame restarts the table chain and the adaptive history.
        memset(us.tc.get(), 0, sizeof(fdvb_tabcache));
        const int pw[3] = {us.w, us.w / 2, us.w / 2}, ph[3] = {us.h, us.h / 2, us.h / 2};
        size_t o = 0;
        for (int p = 0; p < 3; ++p) {
            const fdvb_streams *s = fdvb_engine_istreams(E, u, p);
            if (!s) return 0;
            size_t bcap = (size_t)pw[p] * ph[p] * 2 + 4096;
            std::vector<uint8_t> pb(bcap);
            size_t bl = fdvb_image_blob(s, pw[p], ph[p], qp, pb.data(), bcap, nullptr);
            if (!bl || o + 4 + bl > us.tmp_cap) return 0;
            o = fdvb_put32(us.tmp.data(), o, (uint32_t)bl);
            memcpy(us.tmp.data() + o, pb.data(), bl);
            o += bl;
        }
        blob = o;
    } else {
        const fdvb_streams *s = fdvb_engine_pstreams(E, u);
        if (!s) return 0;
        blob = fdvb_pframe_blob(s, qp, us.tc.get(), us.tmp.data(), us.tmp_cap, nullptr);
    }
    return blob;
}

// Append [blob_len u32][blob] from us.tmp to the unit's stream.
void append_blob(UnitStream &us, size_t blob) {
    uint8_t l4[4];
    fdvb_put32(l4, 0, (uint32_t)blob);
    us.bytes.insert(us.bytes.end(), l4, l4 + 4);
    us.bytes.insert(us.bytes.end(), us.tmp.begin(), us.tmp.begin() + (long)blob);
}

// Entropy-code unit u's output of the engine's last step and append it (the
// tail of fdv_video_encode's frame loop).
int code_unit_frame(fdvb_engine *E, int u, UnitStream &us, int is_intra, int qp) {
    const size_t blob = code_unit_blob(E, u, us, is_intra, qp);
    if (!blob) return -1;
    append_blob(us, blob);
    return 0;
}

// Entropy-code every unit, spreading units over up to nthreads host threads.
int code_all(fdvb_engine *E, std::vector<UnitStream> &us, int is_intra, int qp, int nthreads) {
    const int n = (int)us.size();
    int nt = std::max(1, std::min(nthreads, n));
    if (nt == 1) {
        for (int u = 0; u < n; ++u) if (code_unit_frame(E, u, us[u], is_intra, qp) != 0) return -1;
        return 0;
    }
    std::vector<int> rc(nt, 0);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (int u = t; u < n; u += nt) if (code_unit_frame(E, u, us[u], is_intra, qp) != 0) rc[t] = -1;
        });
    for (auto &x : th) x.join();
    for (int r : rc) if (r) return -1;
    return 0;
}

int default_threads() {
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

// A fixed team of host threads (the caller plus n - 1 workers) that runs the
// tasks 0..ntasks-1 of one job at a time; run() returns when all are done.
class Pool {
  public:
    explicit Pool(int n) {
        for (int i = 1; i < n; ++i) th_.emplace_back([this] { work(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            quit_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void run(int ntasks, const std::function<void(int)> &fn) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            fn_ = &fn;
            ntasks_ = ntasks;
            next_.store(0);
            left_ = ntasks;
            ++gen_;
        }
        cv_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return left_ == 0; });
        fn_ = nullptr;
    }

  private:
    void drain() {
        for (;;) {
            const int i = next_.fetch_add(1);
            if (i >= ntasks_) return;
            (*fn_)(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--left_ == 0) done_cv_.notify_all();
        }
    }
    void work() {
        long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
                if (quit_) return;
                seen = gen_;
            }
            drain();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *fn_ = nullptr;
    std::atomic<int> next_{0};
    int ntasks_ = 0, left_ = 0;
    long gen_ = 0;
    bool quit_ = false;
};

// Engines are kept between calls (keyed by device, search range and unit
// sizes): creating one allocates device and pinned memory, which costs more
// than coding a short clip.  Taken out while in use; at most kCacheMax kept.
struct CachedEngine {
    int device, range;
    std::vector<int> w, h;
    fdvb_engine *E;
    int lver;   // version of the learned-proposal setting the engine carries (0: plain)
};
constexpr size_t kCacheMax = 4;
std::mutex g_cache_mu;
std::vector<CachedEngine> *g_cache = new std::vector<CachedEngine>();   // never destroyed: outlives the CUDA runtime

// The process-wide learned-proposal setting of the fdv_* encoders
// (fdvb_set_learned): parameters, confidence threshold, and a version that
// engines compare against the one they carry.
std::mutex g_learn_mu;
std::vector<float> *g_learn_params = new std::vector<float>();
float g_learn_conf = 0.8f;
int g_learn_ver = 0;       // bumped on every change; 0 never reused
int g_learn_on = 0;
std::map<fdvb_engine *, int> *g_engine_lver = new std::map<fdvb_engine *, int>();

// Launch shapes chosen for engine geometries (fdvb_set_tuning, written by the
// autotuner): key = search range and unit sizes; value = P-frames per launch
// and P-kernel blocks.  Applied whenever the fdv_* encoders take an engine.
std::mutex g_tune_mu;
std::map<std::vector<int>, std::pair<int, int>> *g_tune = new std::map<std::vector<int>, std::pair<int, int>>();
std::vector<int> tune_key(int n, const int *w, const int *h, int range) {
    std::vector<int> k{range, n};
    for (int i = 0; i < n; ++i) { k.push_back(w[i]); k.push_back(h[i]); }
    return k;
}
// The engine's launch shape: the tuned one for its geometry, else the default
// (up to sixty P-frames per launch, one block per SM).
void apply_tuning(fdvb_engine *E, int n, const int *w, const int *h, int range) {
    std::pair<int, int> t{0, 0};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune->find(tune_key(n, w, h, range));
        if (it != g_tune->end()) t = it->second;
    }
    if (t.first > 0) fdvb_engine_set_tuning(E, t.first, t.second);
    else fdvb_engine_set_tuning(E, 60, 0);
}

fdvb_engine *engine_acquire(int n, const int *w, const int *h, int range, int device) {
    fdvb_engine *E = nullptr;
    int ver = 0;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (size_t i = 0; i < g_cache->size(); ++i) {
            CachedEngine &c = (*g_cache)[i];
            if (c.device == device && c.range == range && (int)c.w.size() == n &&
                std::equal(c.w.begin(), c.w.end(), w) && std::equal(c.h.begin(), c.h.end(), h)) {
                E = c.E;
                ver = c.lver;
                g_cache->erase(g_cache->begin() + (long)i);
                break;
            }
        }
    }
    if (!E) E = fdvb_engine_create(n, w, h, range, device);
    if (!E) return nullptr;
    apply_tuning(E, n, w, h, range);
    std::vector<float> params;
    float conf;
    int want, on;
    {
        std::lock_guard<std::mutex> lk(g_learn_mu);
        want = g_learn_ver;
        on = g_learn_on;
        conf = g_learn_conf;
        if (on && want != ver) params = *g_learn_params;
    }
    if (want != ver) {
        if (fdvb_engine_set_learned(E, on ? params.data() : nullptr, conf) != 0) {
            fdvb_engine_destroy(E);
            return nullptr;
        }
        ver = want;
    }
    std::lock_guard<std::mutex> lk(g_cache_mu);
    (*g_engine_lver)[E] = ver;
    return E;
}
void engine_release(fdvb_engine *E, int n, const int *w, const int *h, int range, int device) {
    fdvb_engine *evict = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        const int ver = (*g_engine_lver)[E];
        g_cache->push_back({device, range, std::vector<int>(w, w + n), std::vector<int>(h, h + n), E, ver});
        if (g_cache->size() > kCacheMax) {
            evict = g_cache->front().E;
            g_cache->erase(g_cache->begin());
            g_engine_lver->erase(evict);
        }
    }
    if (evict) fdvb_engine_destroy(evict);
}

}  // namespace

struct fdv_encoder {
    int w = 0, h = 0, qp = 0, keyint = 0, n = 0, key_due = 0;
    int nbands = 0, band_mbrows = 0, nthreads = 1;   // nbands == 0: single stream
    fdvb_engine *E = nullptr;
    std::vector<UnitStream> us;
    std::vector<int> by0, bh;
    int use_rc = 0;                                  // average-bitrate control on
    fdv_rc rc{};
};

extern "C" {

const char *fdvb_last_error(void) { return g_api_err.c_str(); }

void fdvb_release_engines(void) {
    fdvd_release_cached();
    std::vector<CachedEngine> v;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        v.swap(*g_cache);
        for (auto &c : v) g_engine_lver->erase(c.E);
    }
    for (auto &c : v) fdvb_engine_destroy(c.E);
}

int fdvb_set_search_range(int range) {
    if (range != 16 && range != 32 && range != 64) { set_err("search range must be 16, 32 or 64"); return -1; }
    int old = g_range;
    g_range = range;
    return old;
}
int fdvb_get_search_range(void) { return g_range; }
}  // extern "C"
int fdvb_device_setting(void) { return g_device; }
extern "C" {
int fdvb_set_device(int device) {
    if (device < 0) return -1;
    int old = g_device;
    g_device = device;
    return old;
}

size_t fdv_wrap(uint8_t *out, size_t cap, int kind, int fps, const uint8_t *payload, size_t payload_len) {
    if (!out || payload_len > 0xffffffffu || cap < 12 + payload_len) return 0;
    if (kind != 0 && kind != 1) return 0;
    if (fps <= 0 || fps > 65535) fps = 25;
    memmove(out + 12, payload, payload_len);
    memcpy(out, "FDV1", 4);
    out[4] = 1;
    out[5] = (uint8_t)kind;
    size_t o = 6;
    o = fdvb_put16(out, o, (unsigned)fps);
    fdvb_put32(out, o, (uint32_t)payload_len);
    return 12 + payload_len;
}

// Encode nframes over a set of horizontal bands (nbands == 1: the plain
// stream) and leave each band's video stream in us[b].bytes.  Runs of
// consecutive P-frames go to the GPU as batches (one wavefront launch each,
// the frames overlapping); the host entropy-codes one batch's frames, bands in
// parallel, while the GPU analyses the next batch.
//
// band_capped: each band's stream is held to the capacity the reference's
// tiled encoder gives it, twice the band's I420 frame size plus 64 KiB for all
// frames (encode_band, fdv.h:7111-7113, checked per frame as fdv_video_encode
// does, :6800-6804): a band that outgrows it fails the call, as there.
// Host timing of the last whole-array encode (fdvb_encode_stats), ms since
// its start: the first submission, the last frame collected, the end of its
// coding, the end of the call; and the summed time the calling thread spent
// waiting in collects and in the band coding.
namespace {
struct EncTiming {
    double first_submit = 0, last_collect = 0, coded = 0, total = 0, collect_wait = 0, coding = 0;
};
EncTiming g_enc_timing;
std::mutex g_enc_timing_mu;
double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

extern "C" void fdvb_encode_stats(double ms[6]) {
    if (!ms) return;
    std::lock_guard<std::mutex> lk(g_enc_timing_mu);
    const EncTiming &t = g_enc_timing;
    ms[0] = t.first_submit; ms[1] = t.last_collect; ms[2] = t.coded; ms[3] = t.total;
    ms[4] = t.collect_wait; ms[5] = t.coding;
}

static int encode_bands(const uint8_t *const *frames, int nframes, int w, int h, int qp, int keyint,
                        int bh_full, int nthreads, std::vector<UnitStream> &us, bool band_capped = false) {
    const auto t_start = std::chrono::steady_clock::now();
    EncTiming tm;
    const int nb = (h + bh_full - 1) / bh_full, cw = w / 2, ch = h / 2;
    std::vector<int> W(nb, w), H(nb), Y0(nb);
    for (int b = 0; b < nb; ++b) { Y0[b] = b * bh_full; H[b] = std::min(bh_full, h - Y0[b]); }
    const int range = g_range, device = g_device;
    fdvb_engine *E = engine_acquire(nb, W.data(), H.data(), range, device);
    if (!E) { set_engine_err(); return -1; }
    us.clear();
    us.resize(nb);
    for (int b = 0; b < nb; ++b) {
        us[b].w = w; us[b].h = H[b];
        us[b].tmp_cap = (size_t)w * H[b] * 3 + 8192;
        stream_header(us[b].bytes, nframes, w, H[b], qp, keyint);
    }
    const int kmax = std::max(1, fdvb_engine_max_batch(E));
    std::vector<const uint8_t *> planes(3 * nb * kmax), kplanes(3 * nb);
    std::vector<int> intra(nb * kmax), qps(nb * kmax, qp);
    Pool pool(std::max(1, std::min(nthreads, nb)));
    std::vector<int> urc(nb);
    auto key_at = [&](int f) { return f == 0 || (keyint > 0 && f % keyint == 0) ? 1 : 0; };
    std::deque<int> types;    // frame types in flight, oldest first
    int rc = 0;
    // frames in one submission from f: a key frame alone, else a run of
    // P-frames
    auto run_len = [&](int f) {
        int K = 1;
        if (!key_at(f))
            while (K < kmax && f + K < nframes && !key_at(f + K)) ++K;
        return K;
    };
    auto submit_at = [&](int f, int K) -> int {
        for (int k = 0; k < K; ++k) {
            const uint8_t *fy = frames[f + k], *fu = fy + (size_t)w * h, *fv = fu + (size_t)cw * ch;
            for (int b = 0; b < nb; ++b) {
                const int j = k * nb + b;
                planes[3 * j] = fy + (size_t)Y0[b] * w;
                planes[3 * j + 1] = fu + (size_t)(Y0[b] / 2) * cw;
                planes[3 * j + 2] = fv + (size_t)(Y0[b] / 2) * cw;
                intra[j] = key_at(f + k);
            }
        }
        if (key_at(f)) {
            // the sequence's next key frame is analysed in this key frame's
            // launch (fdvb_engine_key_lookahead)
            int f2 = f + 1;
            while (f2 < nframes && !key_at(f2)) ++f2;
            if (f2 < nframes) {
                const uint8_t *fy = frames[f2], *fu = fy + (size_t)w * h, *fv = fu + (size_t)cw * ch;
                for (int b = 0; b < nb; ++b) {
                    kplanes[3 * b] = fy + (size_t)Y0[b] * w;
                    kplanes[3 * b + 1] = fu + (size_t)(Y0[b] / 2) * cw;
                    kplanes[3 * b + 2] = fv + (size_t)(Y0[b] / 2) * cw;
                }
                if (fdvb_engine_key_lookahead(E, kplanes.data(), qps.data()) != 0) { set_engine_err(); return -1; }
            }
        }
        if (fdvb_engine_submit_batch(E, K, planes.data(), intra.data(), qps.data(), nullptr, nullptr) != 0) {
            set_engine_err();
            return -1;
        }
        for (int k = 0; k < K; ++k) types.push_back(key_at(f + k));
        return 0;
    };
    // the caller's frames stay valid for the whole call: pinned ones are
    // copied to the GPU without staging; P-frames are streamed out of their
    // launches, so the host codes each frame while the GPU goes on
    fdvb_engine_direct_upload(E, 1);
    fdvb_engine_stream_frames(E, 1);
    for (int f = 0; rc == 0;) {
        // keep the engine busy: whole runs, up to two runs' worth of frames in flight
        while (f < nframes) {
            const int K = run_len(f);
            if ((int)types.size() + K > 2 * kmax) break;
            if (submit_at(f, K) != 0) { rc = -1; break; }
            if (f == 0) tm.first_submit = ms_since(t_start);
            f += K;
        }
        if (rc != 0 || types.empty()) break;
        // the oldest frame as soon as it is ready, and any later ones ready
        // by then; every band codes them in order as one task (their streams
        // stay in their slots until the next submission)
        std::vector<int> btype;
        std::vector<std::vector<fdvb_streams>> bst(nb);
        do {
            const int ti = types.front();
            types.pop_front();
            const double tc0 = ms_since(t_start);
            if (fdvb_engine_collect(E) != 0) { set_engine_err(); rc = -1; break; }
            tm.collect_wait += ms_since(t_start) - tc0;
            if (types.empty() && f >= nframes) tm.last_collect = ms_since(t_start);
            btype.push_back(ti);
            for (int b = 0; b < nb; ++b)
                for (int p = 0; p < (ti ? 3 : 1); ++p) {
                    const fdvb_streams *s = ti ? fdvb_engine_istreams(E, b, p) : fdvb_engine_pstreams(E, b);
                    if (!s) { set_err("no streams for a collected frame"); rc = -1; break; }
                    bst[b].push_back(*s);
                }
        } while (rc == 0 && !types.empty() && btype.size() < 16 && fdvb_engine_ready(E) == 1);
        if (rc == 0 && !btype.empty()) {
            const double tp0 = ms_since(t_start);
            std::fill(urc.begin(), urc.end(), 0);
            pool.run(nb, [&](int u) {
                size_t o = 0;
                const size_t band_cap = (size_t)w * H[u] * 3 + 65536;   // 2 x (w*bh + 2 * (w/2)*(bh/2)) + 65536
                for (int ti : btype) {
                    const size_t blob = code_blob_streams(&bst[u][o], us[u], ti, qp);
                    if (!blob) { urc[u] = -1; return; }
                    if (band_capped && us[u].bytes.size() + 4 + blob > band_cap) { urc[u] = -2; return; }
                    append_blob(us[u], blob);
                    o += ti ? 3 : 1;
                }
            });
            for (int r : urc)
                if (r) { set_err(r == -2 ? "a band's stream outgrew the tiled encoder's capacity" : "entropy coding failed"); rc = -1; }
            tm.coding += ms_since(t_start) - tp0;
            tm.coded = ms_since(t_start);
        }
    }
    while (!types.empty()) {
        types.pop_front();
        fdvb_engine_collect(E);
    }
    fdvb_engine_key_lookahead(E, nullptr, nullptr);   // the next call's frames are other buffers
    fdvb_engine_direct_upload(E, 0);
    fdvb_engine_stream_frames(E, 0);
    if (rc == 0) engine_release(E, nb, W.data(), H.data(), range, device);
    else fdvb_engine_destroy(E);
    tm.total = ms_since(t_start);
    {
        std::lock_guard<std::mutex> lk(g_enc_timing_mu);
        g_enc_timing = tm;
    }
    return rc;
}

size_t fdv_video_encode(const uint8_t *const *frames, int nframes, int w, int h, int qp, int keyint,
                        uint8_t *out, size_t cap) {
    if (!frames || !out || nframes <= 0 || w <= 0 || h <= 0 || (w & 15) || (h & 15)) { set_err("bad arguments"); return 0; }
    if (qp < 0 || qp > 51 || nframes > 65535 || w > 8192 || h > 8192) { set_err("bad arguments"); return 0; }
    if (keyint < 0) keyint = 0;
    if (keyint > 255) keyint = 255;
    std::vector<UnitStream> us;
    if (encode_bands(frames, nframes, w, h, qp, keyint, h, 1, us) != 0) return 0;
    const auto &b = us[0].bytes;
    if (b.size() > cap) { set_err("output buffer too small"); return 0; }
    memcpy(out, b.data(), b.size());
    return b.size();
}

size_t fdv_vtile_encode(const uint8_t *const *frames, int nframes, int w, int h, int qp, int keyint,
                        int band_mbrows, int nthreads, uint8_t *out, size_t cap) {
    if (!frames || !out || nframes <= 0 || w <= 0 || h <= 0 || (w & 15) || (h & 15) || band_mbrows < 1) {
        set_err("bad arguments");
        return 0;
    }
    if (cap < 12 || qp < 0 || qp > 51 || nframes > 65535 || w > 8192 || h > 8192) { set_err("bad arguments"); return 0; }
    const int bh_full = band_mbrows * 16, nbands = (h + bh_full - 1) / bh_full;
    if (keyint < 0) keyint = 0;
    if (keyint > 255) keyint = 255;
    if (nthreads < 1) nthreads = 1;
    std::vector<UnitStream> us;
    if (encode_bands(frames, nframes, w, h, qp, keyint, bh_full, nthreads, us, true) != 0) return 0;
    size_t o = 0;
    o = fdvb_put16(out, o, (unsigned)w);
    o = fdvb_put16(out, o, (unsigned)h);
    o = fdvb_put16(out, o, (unsigned)nframes);
    out[o++] = (uint8_t)qp;
    out[o++] = (uint8_t)keyint;
    o = fdvb_put16(out, o, (unsigned)nbands);
    o = fdvb_put16(out, o, (unsigned)band_mbrows);
    for (int b = 0; b < nbands; ++b) {
        const auto &s = us[b].bytes;
        if (o + 4 + s.size() > cap) { set_err("output buffer too small"); return 0; }
        o = fdvb_put32(out, o, (uint32_t)s.size());
        memcpy(out + o, s.data(), s.size());
        o += s.size();
    }
    return o;
}

// ------------------------------------------------------------ streaming --
static fdv_encoder *enc_new(int w, int h, int qp, int keyint, int band_mbrows, int nthreads, bool tiled) {
    if (w <= 0 || h <= 0 || (w & 15) || (h & 15) || w > 8192 || h > 8192) { set_err("bad dimensions"); return nullptr; }
    if (qp < 0 || qp > 51) { set_err("bad qp"); return nullptr; }
    if (tiled && band_mbrows < 1) { set_err("bad band_mbrows"); return nullptr; }
    if (keyint < 0) keyint = 0;
    if (keyint > 255) keyint = 255;
    auto *e = new fdv_encoder();
    e->w = w; e->h = h; e->qp = qp; e->keyint = keyint;
    const int bh_full = tiled ? band_mbrows * 16 : h;
    const int nb = (h + bh_full - 1) / bh_full;
    if (tiled && nb > 65535) { delete e; set_err("too many bands"); return nullptr; }
    e->nbands = tiled ? nb : 0;
    e->band_mbrows = band_mbrows;
    e->nthreads = nthreads < 1 ? 1 : nthreads;
    std::vector<int> W(nb, w), H(nb);
    for (int b = 0; b < nb; ++b) { e->by0.push_back(b * bh_full); H[b] = std::min(bh_full, h - b * bh_full); e->bh.push_back(H[b]); }
    e->E = fdvb_engine_create(nb, W.data(), H.data(), g_range, g_device);
    if (!e->E) { set_engine_err(); delete e; return nullptr; }
    apply_tuning(e->E, nb, W.data(), H.data(), g_range);
    e->us.resize(nb);
    for (int b = 0; b < nb; ++b) {
        e->us[b].w = w; e->us[b].h = H[b];
        e->us[b].tmp_cap = (size_t)w * H[b] * 3 + 8192;
        stream_header(e->us[b].bytes, 0, w, H[b], qp, keyint);   // frame count patched at finish
    }
    return e;
}

fdv_encoder *fdv_enc_open(int w, int h, int qp, int keyint) { return enc_new(w, h, qp, keyint, 0, 1, false); }
fdv_encoder *fdv_enc_open_tiled(int w, int h, int qp, int keyint, int band_mbrows, int nthreads) {
    return enc_new(w, h, qp, keyint, band_mbrows, nthreads, true);
}

void fdv_enc_close(fdv_encoder *e) {
    if (!e) return;
    fdvb_engine_destroy(e->E);
    delete e;
}

int fdv_enc_count(const fdv_encoder *e) { return e ? e->n : 0; }
size_t fdv_enc_bytes(const fdv_encoder *e) {
    if (!e) return 0;
    size_t t = 0;
    for (const auto &u : e->us) t += u.bytes.size();
    return t;
}
int fdv_enc_set_bitrate(fdv_encoder *e, int bits_per_second, int fps, double bufsecs) {
    if (!e || bits_per_second <= 0 || e->n != 0) { set_err("bitrate control must be set before the first frame"); return -1; }
    fdv_rc_init(&e->rc, bits_per_second, fps, e->w, e->h, e->keyint, bufsecs, 0, 0);
    e->use_rc = 1;
    return 0;
}

// enc_push (fdv.h:8231-8377): one frame for every band at once; a held frame
// re-emits the reference as all-SKIP and carries a due key frame to the next
// real one.  With bitrate control a single stream takes its QP and lambda
// fraction from the controller and is coded again, coarser, while it lands
// more than 1.5x over its allocation (at most three times, fdv.h:8281-8335);
// a tiled stream gives every band the controller's whole QP (bands_push,
// fdv.h:8066-8127).
static int enc_push(fdv_encoder *e, const uint8_t *i420, int force_skip) {
    if (!e || (!i420 && !force_skip)) return -1;
    if (e->n >= 65535) { set_err("frame count limit"); return -1; }
    const int f = e->n;
    int is_intra = (f == 0) || e->key_due || (e->keyint > 0 && f % e->keyint == 0);
    if (force_skip) { e->key_due = is_intra; is_intra = 0; }
    else e->key_due = 0;
    const int nb = (int)e->us.size(), w = e->w, h = e->h, cw = w / 2, ch = h / 2;
    std::vector<const uint8_t *> planes(3 * nb, nullptr);
    std::vector<int> intra(nb, is_intra), fs(nb, force_skip);
    if (i420) {
        const uint8_t *fy = i420, *fu = fy + (size_t)w * h, *fv = fu + (size_t)cw * ch;
        for (int b = 0; b < nb; ++b) {
            planes[3 * b] = fy + (size_t)e->by0[b] * w;
            planes[3 * b + 1] = fu + (size_t)(e->by0[b] / 2) * cw;
            planes[3 * b + 2] = fv + (size_t)(e->by0[b] / 2) * cw;
        }
    }
    if (e->nbands > 0 || !e->use_rc) {
        // fixed QP, or the tiled form of bitrate control: one whole QP per frame
        int fqp = e->qp;
        const size_t before = fdv_enc_bytes(e);
        if (e->use_rc) fqp = force_skip ? e->rc.used_qp : fdv_rc_pick(&e->rc, is_intra);
        std::vector<int> qps(nb, fqp);
        if (fdvb_engine_step(e->E, planes.data(), intra.data(), qps.data(), nullptr, fs.data()) != 0) { set_engine_err(); return -1; }
        if (code_all(e->E, e->us, is_intra, fqp, e->nthreads) != 0) { set_err("entropy coding failed"); return -1; }
        ++e->n;
        if (e->use_rc) {
            const size_t used = fdv_enc_bytes(e) - before;
            if (force_skip) fdv_rc_skip(&e->rc, used);
            else fdv_rc_update(&e->rc, is_intra, used);
        }
        return 0;
    }
    // single stream under bitrate control
    UnitStream &us = e->us[0];
    int fqp = force_skip ? e->rc.used_qp : fdv_rc_pick(&e->rc, is_intra);
    double lscale = e->rc.lscale;
    double qreal = (double)fqp + log(lscale) / log(fdvb_rc_lfrac());
    const fdvb_tabcache tc_before = *us.tc;   // a second coding starts from the same entropy state
    fdvb_engine_defer_refs(e->E, 1);
    auto code = [&](int q, double ls) -> size_t {
        *us.tc = tc_before;
        if (fdvb_engine_step(e->E, planes.data(), intra.data(), &q, &ls, fs.data()) != 0) return 0;
        return code_unit_blob(e->E, 0, us, is_intra, q);
    };
    size_t blob = code(fqp, lscale);
    if (blob > 0) {
        for (int tries = 0; tries < 3 && qreal < (double)e->rc.qpmax; ++tries) {
            const double alloc = e->rc.last_target > 1.0 ? e->rc.last_target : 1.0;
            const double over = (double)blob * 8.0 / alloc;
            if (over <= 1.5) break;
            double step = 2.0 * log2(over);
            if (step < 0.25) step = 0.25;
            if (step > 4.0) step = 4.0;
            double qn = qreal + step;
            if (qn > (double)e->rc.qpmax) qn = (double)e->rc.qpmax;
            int retry;
            double rls;
            fdv_rc_split(&e->rc, qn, &retry, &rls);
            const size_t again = code(retry, rls);
            if (!again) break;
            blob = again; fqp = retry; qreal = qn; e->rc.used_qp = retry;
        }
        fdv_rc_adopt(&e->rc, is_intra, qreal);
    }
    fdvb_engine_defer_refs(e->E, 0);
    if (blob == 0 || fdvb_engine_commit_refs(e->E) != 0) { set_engine_err(); return -1; }
    append_blob(us, blob);
    if (force_skip) fdv_rc_skip(&e->rc, blob);
    else fdv_rc_update(&e->rc, is_intra, blob);
    ++e->n;
    return 0;
}

int fdv_enc_frame(fdv_encoder *e, const uint8_t *i420) {
    if (!e || !i420) return -1;
    return enc_push(e, i420, 0);
}
int fdv_enc_repeat(fdv_encoder *e) {
    if (!e || e->n == 0) return -1;
    return enc_push(e, nullptr, 1);
}

uint8_t *fdv_enc_finish(fdv_encoder *e, int fps, size_t *len) {
    if (!e) return nullptr;
    if (e->n == 0) { fdv_enc_close(e); return nullptr; }
    for (auto &u : e->us) fdvb_put16(u.bytes.data(), 0, (unsigned)e->n);
    size_t payload = 0;
    if (e->nbands == 0) payload = e->us[0].bytes.size();
    else { payload = 12; for (auto &u : e->us) payload += 4 + u.bytes.size(); }
    size_t cap = 12 + payload;
    uint8_t *buf = static_cast<uint8_t *>(malloc(cap));
    if (!buf) { fdv_enc_close(e); return nullptr; }
    size_t o = 12;
    if (e->nbands == 0) {
        memcpy(buf + o, e->us[0].bytes.data(), payload);
    } else {
        o = fdvb_put16(buf, o, (unsigned)e->w);
        o = fdvb_put16(buf, o, (unsigned)e->h);
        o = fdvb_put16(buf, o, (unsigned)e->n);
        buf[o++] = (uint8_t)e->qp;
        buf[o++] = (uint8_t)e->keyint;
        o = fdvb_put16(buf, o, (unsigned)e->nbands);
        o = fdvb_put16(buf, o, (unsigned)e->band_mbrows);
        for (auto &u : e->us) {
            o = fdvb_put32(buf, o, (uint32_t)u.bytes.size());
            memcpy(buf + o, u.bytes.data(), u.bytes.size());
            o += u.bytes.size();
        }
    }
    size_t flen = fdv_wrap(buf, cap, e->nbands == 0 ? 0 : 1, fps, buf + 12, payload);
    fdv_enc_close(e);
    if (!flen) { free(buf); return nullptr; }
    if (len) *len = flen;
    return buf;
}

// --------------------------------------------------------- engine ABI --
fdvg_ctx *fdvg_create(int nunits, const int *w, const int *h, int range, int device) {
    fdvb_engine *E = fdvb_engine_create(nunits, w, h, range, device);
    if (!E) set_engine_err();
    return E;
}
void fdvg_destroy(fdvg_ctx *g) { fdvb_engine_destroy(g); }
int fdvg_frame(fdvg_ctx *g, const uint8_t *const *planes, const int *is_intra, const int *qp,
               const double *lscale, const int *force_skip) {
    int rc = fdvb_engine_step(g, planes, is_intra, qp, lscale, force_skip);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_submit(fdvg_ctx *g, const uint8_t *const *planes, const int *is_intra, const int *qp,
                const double *lscale, const int *force_skip) {
    int rc = fdvb_engine_submit(g, planes, is_intra, qp, lscale, force_skip);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_collect(fdvg_ctx *g) {
    int rc = fdvb_engine_collect(g);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_pframe_streams(fdvg_ctx *g, int u, const uint8_t **s16, size_t *n16) {
    const fdvb_streams *s = fdvb_engine_pstreams(g, u);
    if (!s || !s16 || !n16) { set_err("no P-frame streams for this unit"); return -1; }
    for (int k = 0; k < 16; ++k) { s16[k] = s->s[k]; n16[k] = s->n[k]; }
    return 0;
}
int fdvg_iframe_streams(fdvg_ctx *g, int u, int plane, const uint8_t **s12, size_t *n12) {
    const fdvb_streams *s = fdvb_engine_istreams(g, u, plane);
    if (!s || !s12 || !n12) { set_err("no key-frame streams for this unit/plane"); return -1; }
    for (int k = 0; k < 12; ++k) { s12[k] = s->s[k]; n12[k] = s->n[k]; }
    return 0;
}
int fdvg_pframe_hist(fdvg_ctx *g, int u, uint32_t *hist) {
    const fdvb_streams *s = fdvb_engine_pstreams(g, u);
    if (!s || !s->hist || !hist) { set_err("no P-frame counts for this unit"); return -1; }
    memcpy(hist, s->hist, sizeof(uint32_t) * 16 * 256);
    return 0;
}
int fdvg_iframe_hist(fdvg_ctx *g, int u, int plane, uint32_t *hist) {
    const fdvb_streams *s = fdvb_engine_istreams(g, u, plane);
    if (!s || !s->hist || !hist) { set_err("no key-frame counts for this unit/plane"); return -1; }
    memcpy(hist, s->hist, sizeof(uint32_t) * 12 * 256);
    return 0;
}
int fdvg_recon(fdvg_ctx *g, int u, uint8_t *i420) {
    int rc = fdvb_engine_recon(g, u, i420);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_set_refs(fdvg_ctx *g, int u, const uint8_t *near_i420, const uint8_t *far_i420) {
    int rc = fdvb_engine_set_refs(g, u, near_i420, far_i420);
    if (rc) set_engine_err();
    return rc;
}

int fdvg_submit_batch(fdvg_ctx *g, int nframes, const uint8_t *const *planes, const int *is_intra, const int *qp,
                      const double *lscale, const int *force_skip) {
    int rc = fdvb_engine_submit_batch(g, nframes, planes, is_intra, qp, lscale, force_skip);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_max_batch(const fdvg_ctx *g) { return fdvb_engine_max_batch(g); }
int fdvg_key_lookahead(fdvg_ctx *g, const uint8_t *const *planes, const int *qp) {
    const int rc = fdvb_engine_key_lookahead(g, planes, qp);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_set_tuning(fdvg_ctx *g, int max_batch, int p_grid) {
    const int rc = fdvb_engine_set_tuning(g, max_batch, p_grid);
    if (rc) set_engine_err();
    return rc;
}
void fdvg_get_tuning(const fdvg_ctx *g, int *max_batch, int *p_grid, int *nsm) {
    fdvb_engine_get_tuning(g, max_batch, p_grid, nsm);
}
int fdvb_set_tuning(int nunits, const int *w, const int *h, int range, int max_batch, int p_grid) {
    if (nunits <= 0 || !w || !h || max_batch < 0 || max_batch > 60 || p_grid < 0) { set_err("bad tuning"); return -1; }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (max_batch == 0) g_tune->erase(tune_key(nunits, w, h, range));
    else (*g_tune)[tune_key(nunits, w, h, range)] = {max_batch, p_grid};
    return 0;
}

// nframes frame steps from device sources, runs of P-frames batched, each
// batch collected while the next one runs; the stream views then describe the
// last frame.
int fdvg_frames_device(fdvg_ctx *g, int nframes, const uint8_t *const *dplanes, const int *is_intra, const int *qp) {
    if (!g || nframes <= 0 || !dplanes || !is_intra || !qp) { set_err("bad arguments"); return -1; }
    const int nu = fdvb_engine_units(g), kmax = std::max(1, fdvb_engine_max_batch(g));
    auto key_at = [&](int f) {
        for (int i = 0; i < nu; ++i) if (is_intra[(size_t)f * nu + i]) return true;
        return false;
    };
    fdvb_engine_src_on_device(g, 1);
    int rc = 0, prev = 0;
    auto all_key = [&](int f) {
        for (int i = 0; i < nu; ++i) if (!is_intra[(size_t)f * nu + i]) return false;
        return true;
    };
    for (int f = 0; f < nframes;) {
        int K = 1;
        if (!key_at(f))
            while (K < kmax && f + K < nframes && !key_at(f + K)) ++K;
        if (all_key(f)) {
            // the next all-key frame is analysed in this one's launch
            int f2 = f + 1;
            while (f2 < nframes && !all_key(f2)) ++f2;
            if (f2 < nframes && fdvb_engine_key_lookahead(g, dplanes + (size_t)3 * nu * f2, qp + (size_t)nu * f2) != 0) {
                rc = -1;
                break;
            }
        }
        rc = fdvb_engine_submit_batch(g, K, dplanes + (size_t)3 * nu * f, is_intra + (size_t)nu * f,
                                      qp + (size_t)nu * f, nullptr, nullptr);
        if (rc) break;
        // the previous batch, all of it even after an error
        for (int n = prev; n > 0; --n) {
            const int r = fdvb_engine_collect(g);
            if (!rc) rc = r;
        }
        prev = K;
        if (rc) break;
        f += K;
    }
    for (; prev > 0; --prev) {
        const int r = fdvb_engine_collect(g);
        if (!rc) rc = r;
    }
    fdvb_engine_key_lookahead(g, nullptr, nullptr);
    fdvb_engine_src_on_device(g, 0);
    if (rc) set_engine_err();
    return rc;
}

int fdvg_frame_device(fdvg_ctx *g, const uint8_t *const *dplanes, const int *is_intra, const int *qp,
                      const double *lscale, const int *force_skip) {
    fdvb_engine_src_on_device(g, 1);
    int rc = fdvb_engine_step(g, dplanes, is_intra, qp, lscale, force_skip);
    fdvb_engine_src_on_device(g, 0);
    if (rc) set_engine_err();
    return rc;
}
void fdvg_stats(const fdvg_ctx *g, double *step_ms, double *analysis_p_ms, long long *p_launches,
                double *analysis_i_ms, long long *i_launches, long long *kernel_launches, long long *steps,
                long long *d2h_bytes) {
    fdvb_engine_stats(g, step_ms, analysis_p_ms, p_launches, analysis_i_ms, i_launches, kernel_launches, steps,
                      d2h_bytes);
}
void fdvg_stats_reset(fdvg_ctx *g) { fdvb_engine_stats_reset(g); }
void fdvg_set_wait_timeout_ns(fdvg_ctx *g, unsigned long long ns) { fdvb_engine_set_wait_ns(g, ns); }
void fdvg_inject_stall(fdvg_ctx *g, int u, int row) { fdvb_engine_inject_stall(g, u, row); }
int fdvg_phase_profile(fdvg_ctx *g, int enable, unsigned long long *out32) { return fdvb_engine_profile(g, enable, out32); }
int fdvg_mb_timeline(fdvg_ctx *g, int u, unsigned long long *out) { return fdvb_engine_timeline(g, u, out); }

int fdvg_set_learned(fdvg_ctx *g, const float *params, float conf) {
    if (!g) { set_err("null context"); return -1; }
    const int rc = fdvb_engine_set_learned(g, params, conf);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_set_learned_conf(fdvg_ctx *g, const float *conf5) {
    if (!g || !conf5) { set_err("null argument"); return -1; }
    return fdvb_engine_learned_conf(g, conf5);
}
int fdvg_set_records(fdvg_ctx *g, int enable) {
    const int rc = fdvb_engine_records(g, enable);
    if (rc) set_engine_err();
    return rc;
}
int fdvg_mb_records(fdvg_ctx *g, int u, uint8_t *mode, int16_t *mv, uint8_t *ref, float *cost) {
    const int rc = fdvb_engine_mb_records(g, u, mode, mv, ref, cost);
    if (rc) set_engine_err();
    return rc;
}

int fdvb_set_learned(const float *params, float conf) {
    if (params && !(conf > 0.f && conf <= 1.f)) { set_err("confidence threshold must be in (0, 1]"); return -1; }
    std::lock_guard<std::mutex> lk(g_learn_mu);
    if (params) g_learn_params->assign(params, params + fdvl_nparams());
    else g_learn_params->clear();
    g_learn_on = params != nullptr;
    g_learn_conf = conf;
    ++g_learn_ver;
    return 0;
}

// ---------------------------------------------------- entropy tail ABI --
fdvb_tabcache *fdvb_tabcache_new(void) { return new fdvb_tabcache(); }
void fdvb_tabcache_reset(fdvb_tabcache *tc) { if (tc) memset(tc, 0, sizeof *tc); }
void fdvb_tabcache_free(fdvb_tabcache *tc) { delete tc; }
size_t fdvb_entropy_pframe(const uint8_t *const *s16, const size_t *n16, int qp, fdvb_tabcache *tc,
                           uint8_t *out, size_t cap) {
    fdvb_streams st;
    for (int k = 0; k < 16; ++k) { st.s[k] = s16[k]; st.n[k] = n16[k]; }
    return fdvb_pframe_blob(&st, qp, tc, out, cap, nullptr);
}
size_t fdvb_entropy_image(const uint8_t *const *s12, const size_t *n12, int w, int h, int qp,
                          uint8_t *out, size_t cap) {
    fdvb_streams st;
    for (int k = 0; k < 16; ++k) { st.s[k] = k < 12 ? s12[k] : nullptr; st.n[k] = k < 12 ? n12[k] : 0; }
    return fdvb_image_blob(&st, w, h, qp, out, cap, nullptr);
}

}  // extern "C"

// The batched GPU encoder engine: owns the device state of a set of
// independent encoder units (the horizontal bands of a tile-parallel stream,
// or whole streams) and advances all of them by one frame per step.
//
// One step, on one CUDA stream:
//   1. source frames host -> device (through a pinned staging buffer);
//   2. analysis: the P-frame wavefront kernel over every P unit's macroblock
//      rows and the intra CTU-wavefront kernel over every key-frame unit's
//      plane CTU rows;
//   3. key frames: deblock, vertical edges then horizontal edges, every plane
//      (P-frames deblock inside the wavefront, post.cuh, except single-frame
//      launches whose rows fill the SMs and the learned form's single frames,
//      which are deblocked as key frames);
//   4. compaction of the per-block symbol slots into the per-stream byte
//      arrays the entropy tail reads, written straight into mapped host memory;
//   5. key frames: reference preparation, the deblocked reconstruction becomes
//      the unit's new nearest reference (integer + half-pel planes); P-frames
//      write theirs tile by tile inside the wavefront (with the same
//      exceptions as in 3).
// The reference pool rotates as fdv_video_encode's (fdv.h:6842-6846): the
// nearest and second-nearest references are the last two coded frames; they
// live in a ring of kRefSlots planes sets, reference q in slot q % kRefSlots.
//
// Up to kMaxBatch consecutive P-frames go into one launch (a batch): frame
// k + 1's rows start as soon as the reference tiles they read have been
// written by frame k's rows, so the frames' wavefronts overlap and fill the
// SMs that one frame's rows leave idle.  Each frame of a batch has its own
// lane of per-frame buffers.
//
// A step is a submit (everything above enqueued, nothing waited on) and a
// collect (wait for the oldest submitted frame, check its error word, point
// the stream views at its output).  Up to kSlots frames can be in flight (two
// batches): staging, output buffers and events are per in-flight frame, so a
// host can entropy-code one batch while the GPU analyses the next.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <thread>
#include <deque>
#include <cstring>
#include <string>
#include <vector>

#include "../host/engine.h"
#include "../host/fdvb_internal.h"
#include "common.cuh"
#include "engine_dev.cuh"

namespace fdvb {
// kernels (pframe.cu, iframe.cu, frame_ops.cu)
void launch_lrn_preskip(const UnitDev *units, const int2 *pu, int np, int total, cudaStream_t st);
void launch_pframe(const UnitDev *units, const RowTask *rows, int nrows, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, int range, bool learned, cudaStream_t st,
                   const FrameSync *fsync = nullptr, const void *ctasks = nullptr, int *fdone = nullptr, int nu = 1,
                   int nunits = 0);
struct IPlaneDev;
struct ITask;
size_t iframe_smem_bytes();
int iframe_slot_bytes();
void iframe_slot_offsets(int off[12]);
void launch_iframe(const void *planes, const void *tasks, int ntasks, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, cudaStream_t st);
struct PrepTask;
struct DbTask;
struct CompactTask;
void launch_refprep(const void *tasks, int ntasks, int maxw, int maxh, int border, cudaStream_t st);
void launch_deblock(const void *tasks, int ntasks, cudaStream_t st);
void launch_compact(const void *tasks, int ntasks, unsigned *err, cudaStream_t st);
int upload_tables(const int32_t c8[64], const int32_t q8[52]);
}  // namespace fdvb

using namespace fdvb;

namespace {

thread_local std::string g_err;

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) {                                                                  \
            g_err = std::string(#x) + ": " + cudaGetErrorString(e_);                              \
            return -3;                                                                            \
        }                                                                                         \
    } while (0)

// Host mirrors of device descriptor layouts (must match iframe.cu / frame_ops.cu).
struct IPlaneDevH {
    const uint8_t *src;
    uint8_t *rec;
    uint8_t *mmap;
    int *progress;
    uint8_t *slots;
    int w, h, cols, rows, qp;
    double lambda;
    unsigned long long *prof;
};
struct ITaskH { int plane, row; };
struct PrepTaskH {
    const uint8_t *rec[3];
    uint8_t *G, *B, *H, *J, *U, *V;
    int w, h, ys, cs, border;
};
struct DbTaskH { uint8_t *p; int w, h, qp; };
struct CompactTaskH {
    const uint8_t *slots;
    int nslots, slot_bytes, nstreams;
    const int *off;
    uint8_t *out;
    size_t cap;
    uint32_t *hist;
    uint8_t *tmp;
};

constexpr int kMaxBatch = 60;               // P-frames per launch at most (a 60-frame GOP's P-frames in one launch)
constexpr int kRefSlots = kMaxBatch + 2;    // reference ring: a batch's outputs never alias its inputs
constexpr int kSlots = 2 * kMaxBatch;       // frames in flight: two batches

struct RefSlot {
    uint8_t *mem = nullptr;
    RefPlanes rp{};
    uint8_t *G, *B, *H, *J, *U, *V;
};

struct Unit {
    int w, h, mbw, mbh, cw, ch;
    // per lane (frame of a batch; key frames use lane 0): source (inside the
    // engine's lane buffer, units back to back in the staging order),
    // reconstruction (un-deblocked for P-frames), records, progress words
    // (P rows: 64-bit words, then per row the count of reference tiles
    // written; then I rows for Y, U, V), macroblock symbol slots
    uint8_t *rec[kMaxBatch] = {};
    size_t src_off = 0;           // this unit's planes in a lane's source buffer
    MBInfo *mbi[kMaxBatch] = {};
    int *progress[kMaxBatch] = {};
    uint8_t *slots[kMaxBatch] = {};
    uint8_t *cout[kMaxBatch] = {};  // per lane: the compaction's device scratch (out_cap bytes)
    int nprog = 0;                  // a lane's progress words (P rows, tile counts, I rows)
    RefSlot ref[kRefSlots];
    long long seq = 0;            // references made so far (the next one goes to slot seq % kRefSlots)
    int nref = 0;
    int recon_slot = -1;          // ring slot holding the last coded frame's deblocked reconstruction
                                  // (-1: it is in lane 0's reconstruction, deblocked in place)
    uint8_t *islots[3] = {nullptr, nullptr, nullptr};
    uint8_t *mmap[3] = {nullptr, nullptr, nullptr};
    int icols[3], irows[3], pw[3], ph[3];
    uint8_t *out_h[kSlots] = {}, *out_d[kSlots] = {};   // per in-flight slot
    // per in-flight slot: the streams' symbol counts, [16][256] for a P-frame,
    // [3][12][256] for a key frame (host-mapped, written by the compaction)
    uint32_t *hist_h[kSlots] = {}, *hist_d[kSlots] = {};
    size_t out_cap = 0, out_off_i[3] = {0, 0, 0};
    int last_intra = 0, last_qp = 0;
    int mb_off = 0;               // first macroblock of this unit in engine-wide per-macroblock arrays
    fdvb_streams ps{}, is[3]{};
    // the key-frame lookahead lane (allocated at first use): a later key
    // frame analysed in the launch of an earlier one -- its reconstruction
    // (deblocked there), per-CTU symbol slots, mode maps and CTU-row progress
    uint8_t *krec = nullptr, *kislots[3] = {nullptr, nullptr, nullptr}, *kmmap[3] = {nullptr, nullptr, nullptr};
    int *kprog = nullptr;
    RefSlot &slot_of(long long q) { return ref[(int)(((q % kRefSlots) + kRefSlots) % kRefSlots)]; }
};

// Words of a lane's progress array before the I rows.
static int p_progress_words(const Unit &u) { return 3 * u.mbh; }

// One in-flight frame: pinned staging of its sources (and, for the first
// frame of a batch, the batch's descriptors), its error word, its events, and
// what its units were.
struct Slot {
    uint8_t *stage = nullptr;
    size_t stage_cap = 0;
    unsigned *err_h = nullptr;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<int> intra;
    bool has_p = false, has_i = false;
    int batch = 0;                // frames of the batch when this is its last frame, else 0
    bool streamed = false;        // compacted inside the P launch: ready once its ready word says so
    unsigned ready_val = 0;
};

}  // namespace

struct fdvb_engine {
    int device = 0, range = 16, border = 32, nsm = 0;
    cudaStream_t st = nullptr;
    std::vector<Unit> units;
    UnitDev *d_units = nullptr;
    RowTask *d_rows = nullptr;
    IPlaneDevH *d_planes = nullptr;
    ITaskH *d_itasks = nullptr;
    PrepTaskH *d_prep = nullptr;
    DbTaskH *d_db = nullptr;
    CompactTaskH *d_cmp = nullptr;
    int *d_ticket = nullptr;
    unsigned *d_err = nullptr;
    int *d_poff = nullptr, *d_ioff = nullptr;
    int maxrows = 0, maxitasks = 0;
    unsigned long long wait_ns = 4000000000ull;
    Slot slot[kSlots];
    // in-flight frames in submission order (slot indices); new frames take the
    // lowest free slots, so callers with one or two frames in flight only
    // ever use (and allocate output buffers for) the first slots
    std::deque<int> order;
    bool busy[kSlots] = {};
    int inflight = 0;
    size_t src_stage_bytes = 0;    // a slot's staging of one frame's sources (64-byte multiple)
    size_t src_bytes = 0;          // one frame's sources, all units
    // per lane, in two sets alternating by submission: every unit's source
    // planes, uploaded on their own stream (st_up) so that a submission's
    // copies overlap the previous submission's kernels
    uint8_t *lane_src[2][kMaxBatch] = {};
    int upar = 0;                        // the set the next submission uploads into
    cudaStream_t st_up = nullptr;
    cudaEvent_t ev_up = nullptr, ev_srcfree[2] = {nullptr, nullptr};
    int lanes = 0;                       // lanes allocated so far (at first use)
    size_t stage_cap = 0;                // a slot's pinned staging (allocated at first use)
    // timing (CUDA events on the engine's stream) and launch counts
    double step_ms = 0, pk_ms = 0, ik_ms = 0;
    long long steps = 0, pk_n = 0, ik_n = 0, launches = 0, d2h = 0;
    int src_on_device = 0;
    int direct_upload = 0;       // host sources that stay valid until collected: pinned ones are copied without staging
    // Frames streamed out of P launches (fdvb_engine_stream_frames): each
    // frame is compacted inside the launch as soon as its rows are done and
    // its host-mapped ready word set, so a host can collect and entropy-code
    // it while the launch goes on.
    int stream_frames = 0;
    unsigned *ready_h = nullptr, *ready_d = nullptr;   // per in-flight slot (host-mapped)
    unsigned ready_seq = 0;
    FrameSync *d_fsync = nullptr;                      // per lane of a launch
    int *d_fdone = nullptr;                            // per unit-frame: rows finished; per frame: units compacted
    int stall_unit = -1, stall_row = -1;
    int defer_refs = 0;                     // leave the reference pool alone until commit
    std::vector<int> pending_intra;         // frame types of the uncommitted step
    std::vector<int> pending_prep;          // its units whose reference is prepared at commit
    bool pending = false;
    unsigned long long *d_prof = nullptr;   // phase profile accumulators (when enabled)
    unsigned long long *d_tl = nullptr;     // per-macroblock timeline (with the phase profile)
    // learned proposals: a private inference network, its per-macroblock
    // hints and the P units of the current step ({unit, first macroblock})
    fdvl_net *lnet = nullptr;
    float3 lconf = {0.8f, 0.8f, 0.8f};       // per class: SKIP, inter, intra (> 1: never)
    double lgate = 0.0;                      // confident SKIP needs J <= lgate * lambda (0: always)
    int linter8 = 0;                         // confident inter also tries INTER8
    lrn::Hint *d_hints = nullptr;            // two buffers (by batch parity) of kMaxBatch x total_mbs
    float *d_prejs = nullptr;                // per hinted macroblock: the SKIP pre-analysis (lrn_preskip_kernel)
    int2 *d_pu = nullptr;
    // The inference runs on its own stream.  With device-resident sources a
    // batch's inference needs nothing of the batch before it (every frame
    // infers against the previous frame's source), so it runs while that
    // batch is analysed, on SMs the analysis leaves free; otherwise the
    // inference stream waits for the main one.
    cudaStream_t st_inf = nullptr;
    cudaEvent_t ev_inf = nullptr, ev_main = nullptr, ev_hfree[2] = {nullptr, nullptr};
    UnitDev *d_units_inf[2] = {nullptr, nullptr};
    int2 *d_pu_inf[2] = {nullptr, nullptr};
    unsigned *d_err_inf = nullptr;           // two words, by batch parity
    int hpar = 0;                            // hint buffer of the next batch
    std::vector<const uint8_t *> prev_luma;  // per unit: the last submitted frame's luma (device sources)
    int total_mbs = 0;
    float *d_mbcost = nullptr;              // per-macroblock RD cost records (when enabled)
    // run-time launch shape (fdvb_engine_set_tuning): P-frames per launch at
    // most, and blocks of the P-frame wavefront kernel (macroblock rows in
    // flight; 0: one per SM)
    int tune_k = kMaxBatch, tune_pgrid = 0;
    // Key-frame lookahead (fdvb_engine_key_lookahead).  A key frame's
    // analysis is a latency-bound chain per CTU row that keeps few SMs busy,
    // and it reads nothing but its own source: the next key frame of a
    // sequence is analysed in the same launch as the current one (its rows
    // after the current frame's luma rows) into the units' lookahead lanes, and
    // its own submission then only compacts its symbols and prepares its
    // reference.  `ka_*`: the frame armed for the next key submission;
    // `kr_*`: the frame analysed and waiting.
    bool ka_armed = false, kr_ready = false;
    std::vector<const uint8_t *> ka_planes, kr_planes;
    std::vector<int> ka_qp, kr_qp;
    uint8_t *key_src = nullptr, *key_stage = nullptr;   // host sources: device copy and pinned staging
};

static int round_up(int v, int a) { return (v + a - 1) / a * a; }

extern "C" const char *fdvb_engine_error(void) { return g_err.c_str(); }

static int alloc_unit(fdvb_engine *E, Unit &u, int w, int h) {
    u.w = w; u.h = h; u.mbw = w / 16; u.mbh = h / 16; u.cw = w / 2; u.ch = h / 2;
    const int B = E->border;
    const int ys = round_up(w + 2 * B, 64), cs = round_up(u.cw + 2 * B, 64);
    const size_t lsz = (size_t)ys * (h + 2 * B), csz = (size_t)cs * (u.ch + 2 * B);
    for (int r = 0; r < kRefSlots; ++r) {
        RefSlot &s = u.ref[r];
        CK(cudaMalloc(&s.mem, 4 * lsz + 2 * csz));
        CK(cudaMemset(s.mem, 0, 4 * lsz + 2 * csz));
        uint8_t *m = s.mem;
        s.G = m + (size_t)B * ys + B; m += lsz;
        s.B = m + (size_t)B * ys + B; m += lsz;
        s.H = m + (size_t)B * ys + B; m += lsz;
        s.J = m + (size_t)B * ys + B; m += lsz;
        s.U = m + (size_t)B * cs + B; m += csz;
        s.V = m + (size_t)B * cs + B;
        s.rp.G = s.G; s.rp.B = s.B; s.rp.H = s.H; s.rp.J = s.J; s.rp.U = s.U; s.rp.V = s.V;
        s.rp.ys = ys; s.rp.cs = cs;
    }
    const int nmb = u.mbw * u.mbh;
    u.pw[0] = w; u.ph[0] = h; u.pw[1] = u.pw[2] = u.cw; u.ph[1] = u.ph[2] = u.ch;
    // P-frame rows: one 64-bit progress word each, then the reference tile counts
    int nprog = p_progress_words(u);
    for (int p = 0; p < 3; ++p) {
        u.icols[p] = (u.pw[p] + 63) / 64; u.irows[p] = (u.ph[p] + 63) / 64;
        nprog += u.irows[p];
        CK(cudaMalloc(&u.islots[p], (size_t)iframe_slot_bytes() * u.icols[p] * u.irows[p]));
        CK(cudaMalloc(&u.mmap[p], (size_t)(u.pw[p] / 4) * (u.ph[p] / 4)));
    }
    u.nprog = nprog;
    // host-mapped output: P-frame streams, or the three planes of a key frame
    size_t pcap = 64 + (size_t)nmb * kSlotData;
    size_t icap[3];
    for (int p = 0; p < 3; ++p) icap[p] = 64 + (size_t)iframe_slot_bytes() * u.icols[p] * u.irows[p];
    for (int p = 0; p < 3; ++p) icap[p] = (icap[p] + 15) / 16 * 16;   // planes' outputs 16-byte aligned
    u.out_off_i[0] = 0; u.out_off_i[1] = icap[0]; u.out_off_i[2] = icap[0] + icap[1];
    u.out_cap = std::max(pcap, icap[0] + icap[1] + icap[2]);
    return 0;
}

// Lanes 0..n-1 of every unit (per frame of a batch: reconstruction, records,
// symbol slots, progress words, compaction scratch, source planes), allocated
// at first use: a batch of K frames needs K lanes, and engines that only ever
// step one frame at a time (many streams in one engine) hold one.
static int ensure_lanes(fdvb_engine *E, int n) {
    for (int k = E->lanes; k < n; ++k) {
        for (auto &u : E->units) {
            const size_t fs = (size_t)u.w * u.h * 3 / 2;
            const int nmb = u.mbw * u.mbh;
            CK(cudaMalloc(&u.rec[k], fs));
            CK(cudaMemset(u.rec[k], 0, fs));
            CK(cudaMalloc(&u.mbi[k], sizeof(MBInfo) * nmb));
            CK(cudaMalloc(&u.slots[k], (size_t)kSlotBytes * nmb));
            CK(cudaMalloc(&u.progress[k], sizeof(int) * u.nprog));
            CK(cudaMalloc(&u.cout[k], u.out_cap));
        }
        CK(cudaMalloc(&E->lane_src[0][k], E->src_bytes));
        CK(cudaMalloc(&E->lane_src[1][k], E->src_bytes));
        E->lanes = k + 1;
    }
    return 0;
}

// A unit's host-mapped output of in-flight slot k, allocated at first use.
static int unit_out(Unit &u, int k) {
    if (u.out_h[k]) return 0;
    CK(cudaHostAlloc(&u.out_h[k], u.out_cap, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(&u.out_d[k], u.out_h[k], 0));
    CK(cudaHostAlloc(&u.hist_h[k], sizeof(uint32_t) * 36 * 256, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(&u.hist_d[k], u.hist_h[k], 0));
    return 0;
}

static void free_unit(Unit &u) {
    for (int k = 0; k < kMaxBatch; ++k) {
        cudaFree(u.rec[k]); cudaFree(u.cout[k]);
        cudaFree(u.mbi[k]); cudaFree(u.slots[k]); cudaFree(u.progress[k]);
    }
    for (int r = 0; r < kRefSlots; ++r) cudaFree(u.ref[r].mem);
    for (int p = 0; p < 3; ++p) { cudaFree(u.islots[p]); cudaFree(u.mmap[p]); }
    cudaFree(u.krec); cudaFree(u.kprog);
    for (int p = 0; p < 3; ++p) { cudaFree(u.kislots[p]); cudaFree(u.kmmap[p]); }
    for (int k = 0; k < kSlots; ++k) if (u.out_h[k]) cudaFreeHost(u.out_h[k]);
    for (int k = 0; k < kSlots; ++k) if (u.hist_h[k]) cudaFreeHost(u.hist_h[k]);
}

// Bytes of the descriptor area of a slot's staging buffer (each array 64-byte aligned).
static size_t stage_desc_bytes(int nu, int maxrows, int maxitasks) {
    auto a = [](size_t n) { return (n + 63) / 64 * 64; };
    // key-frame descriptors twice over: a key frame and the lookahead beside it
    return a(sizeof(UnitDev) * kMaxBatch * nu) + a(sizeof(RowTask) * kMaxBatch * maxrows) +
           a(sizeof(IPlaneDevH) * 6 * nu) + a(sizeof(ITaskH) * 2 * maxitasks) + 2 * a(sizeof(PrepTaskH) * nu) +
           a(sizeof(DbTaskH) * 6 * nu) + a(sizeof(CompactTaskH) * 3 * kMaxBatch * nu) + a(sizeof(int2) * nu) +
           a(sizeof(FrameSync) * kMaxBatch);
}

extern "C" fdvb_engine *fdvb_engine_create(int nunits, const int *w, const int *h, int range, int device) {
    if (nunits <= 0 || !w || !h) { g_err = "bad arguments"; return nullptr; }
    if (range != 16 && range != 32 && range != 64) { g_err = "search range must be 16, 32 or 64"; return nullptr; }
    for (int i = 0; i < nunits; ++i)
        if (w[i] <= 0 || h[i] <= 0 || (w[i] & 15) || (h[i] & 15) || w[i] > 8192 || h[i] > 8192) {
            g_err = "unit dimensions must be positive multiples of 16, at most 8192";
            return nullptr;
        }
    auto *E = new fdvb_engine();
    E->device = device;
    E->range = range;
    E->border = range + 16;
    if (cudaSetDevice(device) != cudaSuccess) { g_err = "cudaSetDevice failed (no GPU?)"; delete E; return nullptr; }
    cudaDeviceGetAttribute(&E->nsm, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&E->st_inf, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_inf, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_main, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_hfree[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_hfree[1], cudaEventDisableTiming) != cudaSuccess) {
        g_err = "stream create failed";
        fdvb_engine_destroy(E);
        return nullptr;
    }
    for (auto &sl : E->slot) for (auto &e : sl.ev) cudaEventCreate(&e);
    int32_t c8[64], q8[52];
    fdvb_c8_tables(c8, q8);
    if (upload_tables(c8, q8) != 0) { g_err = "table upload failed"; fdvb_engine_destroy(E); return nullptr; }
    E->units.resize(nunits);
    int maxrows = 0, maxitasks = 0;
    for (int i = 0; i < nunits; ++i) {
        if (alloc_unit(E, E->units[i], w[i], h[i]) != 0) { fdvb_engine_destroy(E); return nullptr; }
        maxrows += E->units[i].mbh;
        for (int p = 0; p < 3; ++p) maxitasks += E->units[i].irows[p];
    }
    E->maxrows = maxrows; E->maxitasks = maxitasks;
    E->prev_luma.assign(nunits, nullptr);
    for (auto &u : E->units) { u.mb_off = E->total_mbs; E->total_mbs += u.mbw * u.mbh; }
    bool ok = cudaMalloc(&E->d_units, sizeof(UnitDev) * kMaxBatch * nunits) == cudaSuccess &&
              cudaMalloc(&E->d_rows, sizeof(RowTask) * kMaxBatch * maxrows) == cudaSuccess &&
              cudaMalloc(&E->d_planes, sizeof(IPlaneDevH) * 6 * nunits) == cudaSuccess &&
              cudaMalloc(&E->d_itasks, sizeof(ITaskH) * 2 * maxitasks) == cudaSuccess &&
              cudaMalloc(&E->d_prep, sizeof(PrepTaskH) * nunits) == cudaSuccess &&
              cudaMalloc(&E->d_db, sizeof(DbTaskH) * 6 * nunits) == cudaSuccess &&
              cudaMalloc(&E->d_cmp, sizeof(CompactTaskH) * 3 * kMaxBatch * nunits) == cudaSuccess &&
              cudaMalloc(&E->d_ticket, sizeof(int) * 2) == cudaSuccess &&
              cudaMalloc(&E->d_err, sizeof(unsigned)) == cudaSuccess &&
              cudaMalloc(&E->d_err_inf, 2 * sizeof(unsigned)) == cudaSuccess &&
              cudaMalloc(&E->d_poff, sizeof(int) * 16) == cudaSuccess &&
              cudaMalloc(&E->d_ioff, sizeof(int) * 12) == cudaSuccess &&
              cudaMalloc(&E->d_fsync, sizeof(FrameSync) * kMaxBatch) == cudaSuccess &&
              cudaMalloc(&E->d_fdone, sizeof(int) * kMaxBatch * (nunits + 1)) == cudaSuccess &&
              cudaHostAlloc(&E->ready_h, sizeof(unsigned) * kSlots, cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer(&E->ready_d, E->ready_h, 0) == cudaSuccess;
    if (!ok) { g_err = "device allocation failed"; fdvb_engine_destroy(E); return nullptr; }
    size_t src_bytes = 0;
    for (auto &u : E->units) src_bytes += (size_t)u.w * u.h * 3 / 2;
    E->src_bytes = src_bytes;
    E->src_stage_bytes = (src_bytes + 63) / 64 * 64;
    {
        size_t off = 0;
        for (auto &u : E->units) { u.src_off = off; off += (size_t)u.w * u.h * 3 / 2; }
    }
    if (cudaStreamCreateWithFlags(&E->st_up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_up, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_srcfree[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&E->ev_srcfree[1], cudaEventDisableTiming) != cudaSuccess) {
        g_err = "stream create failed";
        fdvb_engine_destroy(E);
        return nullptr;
    }
    if (ensure_lanes(E, 1) != 0) { fdvb_engine_destroy(E); return nullptr; }
    E->stage_cap = E->src_stage_bytes + stage_desc_bytes(nunits, maxrows, maxitasks);
    for (auto &sl : E->slot) {
        sl.stage_cap = E->stage_cap;
        if (cudaHostAlloc(&sl.err_h, 64, cudaHostAllocDefault) != cudaSuccess) {
            g_err = "pinned allocation failed";
            fdvb_engine_destroy(E);
            return nullptr;
        }
        sl.intra.assign(nunits, 0);
    }
    int poff[16], ioff[12];
    for (int k = 0; k < 16; ++k) { int o = 0; for (int i = 0; i < k; ++i) o += kSlotCap[i]; poff[k] = o; }
    iframe_slot_offsets(ioff);
    cudaMemcpy(E->d_poff, poff, sizeof poff, cudaMemcpyHostToDevice);
    cudaMemcpy(E->d_ioff, ioff, sizeof ioff, cudaMemcpyHostToDevice);
    cudaMemset(E->d_err, 0, sizeof(unsigned));
    if (cudaDeviceSynchronize() != cudaSuccess) { g_err = "device init failed"; fdvb_engine_destroy(E); return nullptr; }
    return E;
}

extern "C" void fdvb_engine_destroy(fdvb_engine *E) {
    if (!E) return;
    if (E->st) cudaStreamSynchronize(E->st);
    for (auto &u : E->units) free_unit(u);
    cudaFree(E->d_units); cudaFree(E->d_rows); cudaFree(E->d_planes); cudaFree(E->d_itasks);
    cudaFree(E->d_prep); cudaFree(E->d_db); cudaFree(E->d_cmp); cudaFree(E->d_ticket); cudaFree(E->d_err);
    cudaFree(E->d_poff); cudaFree(E->d_ioff); cudaFree(E->d_fsync); cudaFree(E->d_fdone);
    if (E->ready_h) cudaFreeHost(E->ready_h);
    for (int s = 0; s < 2; ++s) for (auto *p : E->lane_src[s]) cudaFree(p);
    if (E->st_up) { cudaStreamSynchronize(E->st_up); cudaStreamDestroy(E->st_up); }
    for (cudaEvent_t e : {E->ev_up, E->ev_srcfree[0], E->ev_srcfree[1]}) if (e) cudaEventDestroy(e);
    if (E->d_prof) cudaFree(E->d_prof);
    if (E->d_tl) cudaFree(E->d_tl);
    if (E->lnet) fdvl_destroy(E->lnet);
    cudaFree(E->d_hints); cudaFree(E->d_prejs); cudaFree(E->d_pu); cudaFree(E->d_mbcost);
    for (int k = 0; k < 2; ++k) { cudaFree(E->d_units_inf[k]); cudaFree(E->d_pu_inf[k]); }
    cudaFree(E->d_err_inf);
    if (E->st_inf) { cudaStreamSynchronize(E->st_inf); cudaStreamDestroy(E->st_inf); }
    for (cudaEvent_t e : {E->ev_inf, E->ev_main, E->ev_hfree[0], E->ev_hfree[1]}) if (e) cudaEventDestroy(e);
    for (auto &sl : E->slot) {
        for (auto &e : sl.ev) if (e) cudaEventDestroy(e);
        if (sl.stage) cudaFreeHost(sl.stage);
        if (sl.err_h) cudaFreeHost(sl.err_h);
    }
    cudaFree(E->key_src);
    if (E->key_stage) cudaFreeHost(E->key_stage);
    if (E->st) cudaStreamDestroy(E->st);
    delete E;
}

extern "C" int fdvb_engine_units(const fdvb_engine *E) { return E ? (int)E->units.size() : 0; }

// Parse a compacted output region: uint32 len[n] then the streams.  Returns
// the bytes the device wrote.
static size_t parse_streams(const uint8_t *p, int n, fdvb_streams *s) {
    const uint32_t *len = reinterpret_cast<const uint32_t *>(p);
    const uint8_t *d = p + 4 * n;
    for (int k = 0; k < 16; ++k) { s->s[k] = nullptr; s->n[k] = 0; }
    for (int k = 0; k < n; ++k) { s->s[k] = d; s->n[k] = len[k]; d += len[k]; }
    return (size_t)(d - p);
}

// Enqueue the reference preparation of units `which` from lane 0's deblocked
// reconstruction (or the lookahead lane's, key_lane) into ring slot
// seq % kRefSlots (the caller then advances seq); the task array is staged
// in `stage` (pinned, slot-owned) when given, else copied from the stack
// (callers that synchronise before returning).
static int prep_refs(fdvb_engine *E, const std::vector<int> &which, uint8_t *stage = nullptr, bool key_lane = false) {
    std::vector<PrepTaskH> pt;
    int maxw = 0, maxh = 0;
    for (int i : which) {
        Unit &u = E->units[i];
        RefSlot &s = u.slot_of(u.seq);
        PrepTaskH t;
        const uint8_t *src = key_lane ? u.krec : u.rec[0];
        t.rec[0] = src; t.rec[1] = src + (size_t)u.w * u.h; t.rec[2] = t.rec[1] + (size_t)u.cw * u.ch;
        t.G = s.G; t.B = s.B; t.H = s.H; t.J = s.J; t.U = s.U; t.V = s.V;
        t.w = u.w; t.h = u.h; t.ys = s.rp.ys; t.cs = s.rp.cs; t.border = E->border;
        pt.push_back(t);
        maxw = std::max(maxw, u.w); maxh = std::max(maxh, u.h);
    }
    if (pt.empty()) return 0;
    const void *src = pt.data();
    if (stage) { memcpy(stage, pt.data(), sizeof(PrepTaskH) * pt.size()); src = stage; }
    CK(cudaMemcpyAsync(E->d_prep, src, sizeof(PrepTaskH) * pt.size(), cudaMemcpyHostToDevice, E->st));
    launch_refprep(E->d_prep, (int)pt.size(), maxw, maxh, E->border, E->st);
    CK(cudaGetLastError());
    return 0;
}

// The units' lookahead lanes and the lookahead's source buffers, at first use.
static int alloc_key_lanes(fdvb_engine *E) {
    for (auto &u : E->units) {
        if (u.krec) continue;
        CK(cudaMalloc(&u.krec, (size_t)u.w * u.h * 3 / 2));
        int nrows = 0;
        for (int p = 0; p < 3; ++p) {
            CK(cudaMalloc(&u.kislots[p], (size_t)iframe_slot_bytes() * u.icols[p] * u.irows[p]));
            CK(cudaMalloc(&u.kmmap[p], (size_t)(u.pw[p] / 4) * (u.ph[p] / 4)));
            nrows += u.irows[p];
        }
        CK(cudaMalloc(&u.kprog, sizeof(int) * nrows));
    }
    if (!E->key_src) CK(cudaMalloc(&E->key_src, E->src_bytes));
    if (!E->key_stage) CK(cudaHostAlloc(&E->key_stage, E->src_bytes, cudaHostAllocDefault));
    return 0;
}

// Arm the key-frame lookahead: the next key-frame submission also analyses
// this frame (planes: 3 per unit, host or device as the engine's sources;
// qp: one per unit), and when this frame is itself submitted as a key frame,
// with the same plane pointers and quantisers, its analysis is reused.  The
// planes must stay valid and unchanged until then.  NULL planes disarm it and
// drop an analysed frame that was never submitted.
extern "C" int fdvb_engine_key_lookahead(fdvb_engine *E, const uint8_t *const *planes, const int *qp) {
    if (!E) return -1;
    if (!planes) { E->ka_armed = false; E->kr_ready = false; return 0; }
    const int nu = (int)E->units.size();
    if (!qp) { g_err = "bad arguments"; return -1; }
    for (int i = 0; i < nu; ++i) {
        if (qp[i] < 0 || qp[i] > 51) { g_err = "qp out of range"; return -1; }
        if (!planes[3 * i] || !planes[3 * i + 1] || !planes[3 * i + 2]) { g_err = "missing source frame"; return -1; }
    }
    CK(cudaSetDevice(E->device));
    if (alloc_key_lanes(E) != 0) return -3;
    E->ka_planes.assign(planes, planes + 3 * nu);
    E->ka_qp.assign(qp, qp + nu);
    E->ka_armed = true;
    return 0;
}

// Submit K frames (a batch, K <= kMaxBatch): arrays hold frame k's entries at
// k * nunits (planes: 3 per unit).  K > 1 needs every unit of every frame to
// be a P-frame, no learned proposals, no decision records and no deferred
// references; the frames go into one P-frame launch.
extern "C" int fdvb_engine_submit_batch(fdvb_engine *E, int K, const uint8_t *const *planes, const int *is_intra,
                                        const int *qp, const double *lscale, const int *force_skip) {
    if (!E) return -1;
    const int nu = (int)E->units.size();
    if (K < 1 || K > kMaxBatch) { g_err = "batch size out of range"; return -1; }
    if (E->inflight + K > kSlots) { g_err = "too many frames in flight"; return -1; }
    if (K > 1 && (E->d_mbcost || E->defer_refs)) {
        g_err = "batches of P-frames need decision records and deferred references off";
        return -1;
    }
    for (int k = 0; k < K; ++k)
        for (int i = 0; i < nu; ++i) {
            const int j = k * nu + i;
            if (qp[j] < 0 || qp[j] > 51) { g_err = "qp out of range"; return -1; }
            const bool fs = force_skip && force_skip[j];
            if (!fs && (!planes || !planes[3 * j] || !planes[3 * j + 1] || !planes[3 * j + 2])) {
                g_err = "missing source frame";
                return -1;
            }
            if (K > 1 && is_intra[j]) { g_err = "a batch of several frames holds P-frames only"; return -1; }
            const int nref = k == 0 ? E->units[i].nref : 1;
            if (fs && (is_intra[j] || nref == 0)) { g_err = "a held frame needs a reference"; return -1; }
            if (!is_intra[j] && nref == 0) { g_err = "a P-frame needs a reference"; return -1; }
        }
    // A key frame for every unit: either the lookahead analysed it already
    // (same planes and quantisers), or it is analysed now, with the armed
    // lookahead frame beside it in the same launch.
    bool all_key = K == 1;
    for (int i = 0; i < nu && all_key; ++i) if (!is_intra[i] || (force_skip && force_skip[i])) all_key = false;
    bool prefetched = false;
    if (all_key && E->kr_ready && !E->defer_refs) {
        prefetched = std::equal(E->kr_planes.begin(), E->kr_planes.end(), planes) &&
                     std::equal(E->kr_qp.begin(), E->kr_qp.end(), qp);
        E->kr_ready = false;
    }
    // (an armed frame that is this very frame is simply coded now)
    const bool joint = all_key && !prefetched && E->ka_armed && !E->defer_refs &&
                       !std::equal(E->ka_planes.begin(), E->ka_planes.end(), planes);
    CK(cudaSetDevice(E->device));
    if (ensure_lanes(E, K) != 0) return -3;
    int sis[kMaxBatch];
    for (int k = 0, s = 0; k < K; ++k) {
        while (E->busy[s]) ++s;
        sis[k] = s++;
        for (auto &u : E->units)
            if (unit_out(u, sis[k]) != 0) return -3;
        if (!E->slot[sis[k]].stage) CK(cudaHostAlloc(&E->slot[sis[k]].stage, E->stage_cap, cudaHostAllocDefault));
    }
    Slot &SL = E->slot[sis[K - 1]];   // the batch's last frame carries its timing
    CK(cudaEventRecord(SL.ev[0], E->st));
    // 1. sources: device sources are read where they are; host sources go
    // through each frame's pinned staging buffer, laid out as the lane buffer,
    // uploaded in chunks of at least 4 MB as units are staged, so the copies
    // overlap the staging while staying few (a held unit's part is left as
    // it is)
    // Pinned host sources whose caller keeps them unchanged until the frame
    // is collected (direct_upload), when a frame's planes tile one contiguous
    // span (the bands of one frame do), are copied in one piece straight from
    // the caller's memory, with no staging copy on the host; the units then
    // read their planes at their offsets in the span.
    auto pinned = [](const void *p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
        return a.type == cudaMemoryTypeHost;
    };
    std::vector<const uint8_t *> span_lo(K, nullptr);   // frame k copied as one span from here (else null)
    // this submission's source set: free once the kernels of the submission
    // before the last one (which read it) have run
    const int par = E->upar;
    if (!E->src_on_device) CK(cudaStreamWaitEvent(E->st_up, E->ev_srcfree[par], 0));
    if (!E->src_on_device && E->direct_upload && !force_skip)
        for (int k = 0; k < K; ++k) {
            const uint8_t *lo = nullptr, *hi = nullptr;
            size_t sum = 0;
            for (int i = 0; i < nu; ++i) {
                const Unit &u = E->units[i];
                const size_t sz[3] = {(size_t)u.w * u.h, (size_t)u.cw * u.ch, (size_t)u.cw * u.ch};
                for (int p = 0; p < 3; ++p) {
                    const uint8_t *q = planes[3 * (k * nu + i) + p];
                    if (!lo || q < lo) lo = q;
                    if (!hi || q + sz[p] > hi) hi = q + sz[p];
                    sum += sz[p];
                }
            }
            if ((size_t)(hi - lo) != sum || sum > E->src_bytes || !pinned(lo) || !pinned(hi - 1)) continue;
            if (cudaMemcpyAsync(E->lane_src[par][k], lo, sum, cudaMemcpyHostToDevice, E->st_up) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            span_lo[k] = lo;
        }
    if (!E->src_on_device)
        for (int k = 0; k < K; ++k) {
            if (span_lo[k]) continue;
            uint8_t *const stage0 = E->slot[sis[k]].stage;
            uint8_t *stage = stage0;
            size_t sent = 0;
            for (int i = 0; i < nu; ++i) {
                Unit &u = E->units[i];
                const int j = k * nu + i;
                const size_t ys = (size_t)u.w * u.h, cs = (size_t)u.cw * u.ch;
                if (!(force_skip && force_skip[j])) {
                    memcpy(stage, planes[3 * j], ys);
                    memcpy(stage + ys, planes[3 * j + 1], cs);
                    memcpy(stage + ys + cs, planes[3 * j + 2], cs);
                }
                stage += ys + 2 * cs;
                const size_t done = (size_t)(stage - stage0);
                if (done - sent >= ((size_t)4 << 20) || i == nu - 1) {
                    CK(cudaMemcpyAsync(E->lane_src[par][k] + sent, stage0 + sent, done - sent, cudaMemcpyHostToDevice,
                                       E->st_up));
                    sent = done;
                }
            }
        }
    if (!E->src_on_device) {
        // the kernels below read the sources once they are copied
        CK(cudaEventRecord(E->ev_up, E->st_up));
        CK(cudaStreamWaitEvent(E->st, E->ev_up, 0));
    }
    // the lookahead frame's sources: read in place, or staged and uploaded
    std::vector<const uint8_t *> kplanes;
    if (joint) {
        kplanes = E->ka_planes;
        if (!E->src_on_device) {
            size_t off = 0;
            for (int i = 0; i < nu; ++i) {
                Unit &u = E->units[i];
                const size_t ys = (size_t)u.w * u.h, cs = (size_t)u.cw * u.ch;
                memcpy(E->key_stage + off, kplanes[3 * i], ys);
                memcpy(E->key_stage + off + ys, kplanes[3 * i + 1], cs);
                memcpy(E->key_stage + off + ys + cs, kplanes[3 * i + 2], cs);
                kplanes[3 * i] = E->key_src + off;
                kplanes[3 * i + 1] = E->key_src + off + ys;
                kplanes[3 * i + 2] = E->key_src + off + ys + cs;
                off += ys + 2 * cs;
            }
            CK(cudaMemcpyAsync(E->key_src, E->key_stage, off, cudaMemcpyHostToDevice, E->st));
        }
    }
    // descriptors are staged after the first frame's sources
    uint8_t *stage = SL.stage + E->src_stage_bytes;
    auto staged = [&](const void *src, size_t n) -> const void * {
        memcpy(stage, src, n);
        const void *r = stage;
        stage += (n + 63) / 64 * 64;
        return r;
    };
    // 2. descriptors
    std::vector<UnitDev> ud(K * nu);
    std::vector<RowTask> rows;
    std::vector<IPlaneDevH> iplanes;
    std::vector<ITaskH> itasks;
    std::vector<CompactTaskH> cmp;
    std::vector<DbTaskH> db;
    // units deblocked and prepared after the frame by the whole-frame kernels:
    // key frames, and P-frames of the learned form (its confident macroblocks
    // take less time than a tile of the in-wavefront stage, which would then
    // lengthen the wavefront; the form runs one frame per launch anyway)
    std::vector<int> iunits;
    std::vector<int> kunits;  // key frames analysed by the lookahead: reference from its lane
    std::vector<char> iluma;  // per key-frame plane descriptor: a luma plane
    std::vector<int2> pu;     // P units and their first macroblock in the hint array
    int nhint = 0, npu0 = 0, nhint0 = 0;   // frame 0's share (its SKIP pre-analysis)
    // Inference ahead of the analysis (device sources, several frames, every
    // unit's previous frame known): frame 0 too infers against the previous
    // frame's source, so nothing of the batch before is needed.
    bool ahead = E->lnet && E->src_on_device && K > 1;
    for (int i = 0; i < nu && ahead; ++i) if (!E->prev_luma[i]) ahead = false;
    const int hpar = E->hpar;
    lrn::Hint *const hbase = E->d_hints ? E->d_hints + (size_t)hpar * kMaxBatch * E->total_mbs : nullptr;
    float *const pbase = E->d_prejs ? E->d_prejs + (size_t)hpar * kMaxBatch * E->total_mbs : nullptr;
    // One frame per launch whose P rows fill the SMs by themselves (many
    // streams in one engine): deblocking and reference preparation run as
    // whole-frame kernels after the analysis, at full width in a fraction of
    // a millisecond, instead of taking SM time from the rows.  Batches (the
    // next frame reads the reference while it is written) and frames whose
    // rows leave SMs idle use the in-wavefront stage.  The learned form's
    // single frames also use the whole-frame kernels (its confident
    // macroblocks are shorter than the stage's tiles).
    int p_rows = 0;
    for (int i = 0; i < nu; ++i) if (!is_intra[i]) p_rows += E->units[i].mbh;
    const bool whole_frame_refs = K == 1 && (E->lnet || p_rows >= E->nsm);
    for (int k = 0; k < K; ++k) {
        std::vector<RowTask> frows;
        E->slot[sis[k]].intra.assign(nu, 0);
        for (int i = 0; i < nu; ++i) {
            Unit &u = E->units[i];
            const int j = k * nu + i;
            UnitDev &d = ud[j];
            d.w = u.w; d.h = u.h; d.mbw = u.mbw; d.mbh = u.mbh;
            if (E->src_on_device && !(force_skip && force_skip[j])) {
                d.cur[0] = planes[3 * j]; d.cur[1] = planes[3 * j + 1]; d.cur[2] = planes[3 * j + 2];
            } else if (span_lo[k]) {
                for (int p = 0; p < 3; ++p) d.cur[p] = E->lane_src[par][k] + (planes[3 * j + p] - span_lo[k]);
            } else {
                d.cur[0] = E->lane_src[par][k] + u.src_off;
                d.cur[1] = d.cur[0] + (size_t)u.w * u.h;
                d.cur[2] = d.cur[1] + (size_t)u.cw * u.ch;
            }
            d.rec[0] = u.rec[k]; d.rec[1] = u.rec[k] + (size_t)u.w * u.h; d.rec[2] = d.rec[1] + (size_t)u.cw * u.ch;
            // frame k's references: the outputs of the two frames before it
            const int nref = k == 0 ? u.nref : std::min(2, u.nref + k);
            const int navail = nref >= 2 ? 2 : 1;
            d.ref[0] = u.slot_of(u.seq - 1 + k).rp;
            d.ref[1] = navail == 2 ? u.slot_of(u.seq - 2 + k).rp : d.ref[0];
            d.mbi = u.mbi[k]; d.progress = u.progress[k]; d.slots = u.slots[k];
            d.lambda = fdvb_lambda(qp[j], lscale ? lscale[j] : 1.0);
            d.qp = qp[j]; d.navail = navail; d.force_skip = force_skip ? force_skip[j] : 0; d.range = E->range;
            d.stall_row = (i == E->stall_unit && k == 0) ? E->stall_row : -1;
            d.prof = E->d_prof;
            d.hint = nullptr;
            d.prejs = nullptr;
            d.skip_gate = E->lgate;
            d.inter8 = E->linter8;
            d.mbcost = E->d_mbcost ? E->d_mbcost + u.mb_off : nullptr;
            d.tl = E->d_tl ? E->d_tl + 2 * (size_t)u.mb_off : nullptr;
            d.out = OutPlanes{};
            d.post_prog = nullptr;
            d.ref_prog = nullptr;
            d.lref = nullptr;
            d.lrs = 0;
            if (!is_intra[j] && E->lnet) {
                pu.push_back(make_int2(j, nhint));
                d.hint = hbase + nhint;
                // the SKIP pre-analysis needs the reference before the
                // launch: frame 0 of a batch only; later frames infer
                // against the previous frame's source
                d.prejs = k == 0 ? pbase + nhint : nullptr;
                if (k > 0) { d.lref = ud[j - nu].cur[0]; d.lrs = u.w; }
                else if (ahead) { d.lref = E->prev_luma[i]; d.lrs = u.w; }
                nhint += u.mbw * u.mbh;
                if (k == 0) { npu0 = (int)pu.size(); nhint0 = nhint; }
            }
            u.last_qp = qp[j];
            if (!is_intra[j]) {
                if (whole_frame_refs) {
                    iunits.push_back(i);
                    for (int p = 0; p < 3; ++p) db.push_back({d.rec[p], u.pw[p], u.ph[p], qp[j]});
                } else {
                    // the frame's reference is written inside the wavefront,
                    // into the ring slot after its own references
                    const RefSlot &o = u.slot_of(u.seq + k);
                    d.out = OutPlanes{o.G, o.B, o.H, o.J, o.U, o.V, o.rp.ys, o.rp.cs};
                    d.post_prog = u.progress[k] + 2 * u.mbh;
                    d.ref_prog = k > 0 ? u.progress[k - 1] + 2 * u.mbh : nullptr;
                }
                for (int r = 0; r < u.mbh; ++r) frows.push_back({j, r});
                CompactTaskH c{u.slots[k], u.mbw * u.mbh, kSlotBytes, 16, E->d_poff, u.out_d[sis[k]], u.out_cap,
                               u.hist_d[sis[k]], u.cout[k]};
                cmp.push_back(c);
            } else if (prefetched) {
                // analysed (and deblocked) in an earlier key frame's launch:
                // compact its symbols; its reference comes from the lookahead lane
                kunits.push_back(i);
                for (int p = 0; p < 3; ++p) {
                    CompactTaskH c{u.kislots[p], u.icols[p] * u.irows[p], iframe_slot_bytes(), 12, E->d_ioff,
                                   u.out_d[sis[k]] + u.out_off_i[p],
                                   (p < 2 ? u.out_off_i[p + 1] : u.out_cap) - u.out_off_i[p],
                                   u.hist_d[sis[k]] + p * 12 * 256, u.cout[k] + u.out_off_i[p]};
                    cmp.push_back(c);
                }
            } else {
                iunits.push_back(i);
                int prog = p_progress_words(u);
                for (int p = 0; p < 3; ++p) {
                    IPlaneDevH P;
                    P.src = d.cur[p]; P.rec = d.rec[p]; P.mmap = u.mmap[p]; P.progress = u.progress[0] + prog;
                    P.slots = u.islots[p]; P.w = u.pw[p]; P.h = u.ph[p]; P.cols = u.icols[p]; P.rows = u.irows[p];
                    P.qp = qp[j]; P.lambda = fdvb_lambda(qp[j], 1.0); P.prof = E->d_prof ? E->d_prof + 16 : nullptr;
                    int pid = (int)iplanes.size();
                    iplanes.push_back(P);
                    iluma.push_back(p == 0);
                    for (int r = 0; r < u.irows[p]; ++r) itasks.push_back({pid, r});
                    prog += u.irows[p];
                    CompactTaskH c{u.islots[p], u.icols[p] * u.irows[p], iframe_slot_bytes(), 12, E->d_ioff,
                                   u.out_d[sis[k]] + u.out_off_i[p],
                                   (p < 2 ? u.out_off_i[p + 1] : u.out_cap) - u.out_off_i[p],
                                   u.hist_d[sis[k]] + p * 12 * 256, u.cout[k] + u.out_off_i[p]};
                    cmp.push_back(c);
                }
                for (int p = 0; p < 3; ++p) db.push_back({d.rec[p], u.pw[p], u.ph[p], qp[j]});
                if (joint) {
                    // the lookahead frame: the same unit's planes into its lane
                    // (deblocked here too; compacted at its own submission)
                    const size_t ys = (size_t)u.w * u.h, cs = (size_t)u.cw * u.ch;
                    uint8_t *krec[3] = {u.krec, u.krec + ys, u.krec + ys + cs};
                    int kp = 0;
                    for (int p = 0; p < 3; ++p) {
                        IPlaneDevH P;
                        P.src = kplanes[3 * i + p]; P.rec = krec[p]; P.mmap = u.kmmap[p]; P.progress = u.kprog + kp;
                        P.slots = u.kislots[p]; P.w = u.pw[p]; P.h = u.ph[p]; P.cols = u.icols[p]; P.rows = u.irows[p];
                        P.qp = E->ka_qp[i]; P.lambda = fdvb_lambda(E->ka_qp[i], 1.0);
                        P.prof = E->d_prof ? E->d_prof + 16 : nullptr;
                        const int pid = (int)iplanes.size();
                        iplanes.push_back(P);
                        iluma.push_back(p == 0);
                        for (int r = 0; r < u.irows[p]; ++r) itasks.push_back({pid, r});
                        kp += u.irows[p];
                        db.push_back({krec[p], u.pw[p], u.ph[p], E->ka_qp[i]});
                    }
                    CK(cudaMemsetAsync(u.kprog, 0, sizeof(int) * kp, E->st));
                }
            }
            const int nprog = p_progress_words(u) + u.irows[0] + u.irows[1] + u.irows[2];
            CK(cudaMemsetAsync(u.progress[k], 0, sizeof(int) * nprog, E->st));
        }
        for (int i = 0; i < nu; ++i) E->slot[sis[k]].intra[i] = is_intra[k * nu + i];
        // Interleave the rows of different units so the early rows of every
        // unit start first; frames in order (a row only ever waits for rows
        // of its own frame above it and of the frame before: earlier tickets).
        int maxh = 0;
        for (auto &u : E->units) maxh = std::max(maxh, u.mbh);
        for (int r = 0; r < maxh; ++r)
            for (auto &t : frows) if (t.row == r) rows.push_back(t);
    }
    // Frames of a launch overlap: row r of frame k needs the frame before
    // only up to its row r + DR + 1 (the row that posts tile row r + DR,
    // DR the reference rows the window reaches), so a frame can start about
    // F macroblock steps after the one before, rows 2 steps apart.  Tickets
    // in that order (frame k, row r at k F + 2 r) hand an SM the row that
    // can run soonest: frame by frame, a tall frame's last rows, which start
    // long after the next frame's first ones, would hold SMs while they
    // wait.  F > 2 (DR + 1), so every row a task waits for still has an
    // earlier ticket (no deadlock); bands of a few rows keep frame order.
    if (K > 1 && !whole_frame_refs) {
        const bool win = E->range <= 32;
        const int dr = win ? (E->range + 19) / 16 : E->range / 16 + 2, dc = win ? 4 : E->range / 16 + 2;
        const int F = 2 * (dr + 1) + dc + 6;
        std::stable_sort(rows.begin(), rows.end(), [&](const RowTask &a, const RowTask &b) {
            return (a.unit / nu) * F + 2 * a.row < (b.unit / nu) * F + 2 * b.row;
        });
    }
    // Key-frame CTU rows in ticket order: by row, a row's luma planes (the
    // longest chains) before its chroma planes.  A row waits only for the row
    // above in its own plane, which comes earlier in this order.
    std::stable_sort(itasks.begin(), itasks.end(), [&](const ITaskH &a, const ITaskH &b) {
        return 2 * a.row + (iluma[a.plane] ? 0 : 1) < 2 * b.row + (iluma[b.plane] ? 0 : 1);
    });
    const void *ud_st = staged(ud.data(), sizeof(UnitDev) * K * nu);
    CK(cudaMemcpyAsync(E->d_units, ud_st, sizeof(UnitDev) * K * nu, cudaMemcpyHostToDevice, E->st));
    CK(cudaMemsetAsync(E->d_ticket, 0, sizeof(int) * 2, E->st));
    CK(cudaMemsetAsync(E->d_err, 0, sizeof(unsigned), E->st));
    // Frames streamed out of the P launch: every unit of every frame a
    // P-frame with its reference written inside the wavefront; the frame's
    // compaction tasks (one per unit, cmp[k * nu + i]) run inside the launch.
    bool all_p = true;
    for (int j = 0; j < K * nu; ++j) if (is_intra[j]) all_p = false;
    const bool streamable = E->stream_frames && !rows.empty() && itasks.empty() && all_p && !whole_frame_refs &&
                            (int)cmp.size() == K * nu;
    std::vector<unsigned> fs_val(K, 0u);
    if (streamable) {
        CK(cudaMemcpyAsync(E->d_cmp, staged(cmp.data(), sizeof(CompactTaskH) * cmp.size()),
                           sizeof(CompactTaskH) * cmp.size(), cudaMemcpyHostToDevice, E->st));
        std::vector<FrameSync> fsv(K);
        for (int k = 0; k < K; ++k) {
            if (++E->ready_seq == 0) ++E->ready_seq;
            fs_val[k] = E->ready_seq;
            E->ready_h[sis[k]] = 0u;
            fsv[k] = FrameSync{E->ready_d + sis[k], fs_val[k]};
        }
        CK(cudaMemcpyAsync(E->d_fsync, staged(fsv.data(), sizeof(FrameSync) * K), sizeof(FrameSync) * K,
                           cudaMemcpyHostToDevice, E->st));
        CK(cudaMemsetAsync(E->d_fdone, 0, sizeof(int) * K * (nu + 1), E->st));
    }
    if (!rows.empty()) {
        CK(cudaMemcpyAsync(E->d_rows, staged(rows.data(), sizeof(RowTask) * rows.size()), sizeof(RowTask) * rows.size(),
                           cudaMemcpyHostToDevice, E->st));
        // every SM: the next batch's inference (its own stream) takes the SMs
        // this launch leaves while it ramps up and drains; reserving 16 or 40
        // SMs for it made the learned P-frame slower (0.46 / 0.52 against
        // 0.39 ms on the learned 720p workload)
        const int grid = std::min((int)rows.size(), E->tune_pgrid > 0 ? std::min(E->tune_pgrid, E->nsm) : E->nsm);
        const void *pu_st = nullptr;
        if (!pu.empty()) {
            pu_st = staged(pu.data(), sizeof(int2) * pu.size());
            CK(cudaMemcpyAsync(E->d_pu, pu_st, sizeof(int2) * pu.size(), cudaMemcpyHostToDevice, E->st));
        }
        CK(cudaEventRecord(SL.ev[1], E->st));
        if (!pu.empty()) {
            // the inference stream: not before the analysis that last read
            // this hint buffer; ahead of this batch's analysis when it can
            // be, else after this batch's uploads
            const UnitDev *iu = E->d_units;
            const int2 *ip = E->d_pu;
            CK(cudaStreamWaitEvent(E->st_inf, E->ev_hfree[hpar], 0));
            if (ahead) {
                CK(cudaMemcpyAsync(E->d_units_inf[hpar], ud_st, sizeof(UnitDev) * K * nu, cudaMemcpyHostToDevice,
                                   E->st_inf));
                CK(cudaMemcpyAsync(E->d_pu_inf[hpar], pu_st, sizeof(int2) * pu.size(), cudaMemcpyHostToDevice,
                                   E->st_inf));
                iu = E->d_units_inf[hpar];
                ip = E->d_pu_inf[hpar];
            } else {
                CK(cudaEventRecord(E->ev_main, E->st));
                CK(cudaStreamWaitEvent(E->st_inf, E->ev_main, 0));
            }
            CK(cudaMemsetAsync(E->d_err_inf + hpar, 0, sizeof(unsigned), E->st_inf));
            if (lrn_infer_units(E->lnet, iu, ip, (int)pu.size(), nhint, E->lconf, 4 * E->range, hbase,
                                E->d_err_inf + hpar, E->st_inf) != 0) {
                g_err = std::string("learned inference: ") + fdvl_last_error();
                return -3;
            }
            CK(cudaEventRecord(E->ev_inf, E->st_inf));
            CK(cudaStreamWaitEvent(E->st, E->ev_inf, 0));
            if (npu0 > 0) launch_lrn_preskip(E->d_units, E->d_pu, npu0, nhint0, E->st);
            E->launches += 2;
        }
        launch_pframe(E->d_units, E->d_rows, (int)rows.size(), E->d_ticket, E->d_err, E->wait_ns, grid, E->range,
                      !pu.empty(), E->st, streamable ? E->d_fsync : nullptr, E->d_cmp, E->d_fdone, nu, K * nu);
        CK(cudaGetLastError());
        CK(cudaEventRecord(SL.ev[2], E->st));
        if (!pu.empty()) {
            CK(cudaEventRecord(E->ev_hfree[hpar], E->st));   // this hint buffer is free again
            E->hpar ^= 1;
        }
        E->launches += 1;
    }
    if (!itasks.empty()) {
        CK(cudaMemcpyAsync(E->d_planes, staged(iplanes.data(), sizeof(IPlaneDevH) * iplanes.size()),
                           sizeof(IPlaneDevH) * iplanes.size(), cudaMemcpyHostToDevice, E->st));
        CK(cudaMemcpyAsync(E->d_itasks, staged(itasks.data(), sizeof(ITaskH) * itasks.size()),
                           sizeof(ITaskH) * itasks.size(), cudaMemcpyHostToDevice, E->st));
        CK(cudaEventRecord(SL.ev[3], E->st));
        launch_iframe(E->d_planes, E->d_itasks, (int)itasks.size(), E->d_ticket + 1, E->d_err, E->wait_ns, E->nsm, E->st);
        CK(cudaGetLastError());
        CK(cudaEventRecord(SL.ev[4], E->st));
        E->launches += 1;
    }
    // 3. deblock (key frames), 4. compact
    if (!db.empty()) {
        CK(cudaMemcpyAsync(E->d_db, staged(db.data(), sizeof(DbTaskH) * db.size()), sizeof(DbTaskH) * db.size(),
                           cudaMemcpyHostToDevice, E->st));
        launch_deblock(E->d_db, (int)db.size(), E->st);
        CK(cudaGetLastError());
        E->launches += 2;
    }
    if (!streamable) {
        CK(cudaMemcpyAsync(E->d_cmp, staged(cmp.data(), sizeof(CompactTaskH) * cmp.size()),
                           sizeof(CompactTaskH) * cmp.size(), cudaMemcpyHostToDevice, E->st));
        launch_compact(E->d_cmp, (int)cmp.size(), E->d_err, E->st);
        CK(cudaGetLastError());
        E->launches += 1;
    }
    // 5. the new references (deferred: the caller may code this frame again)
    if (E->defer_refs) {
        E->pending_intra.assign(is_intra, is_intra + nu);
        E->pending_prep.assign(nu, 0);
        for (int i : iunits) E->pending_prep[i] = 1;
        E->pending = true;
        for (int i = 0; i < nu; ++i) {
            Unit &u = E->units[i];
            u.recon_slot = E->pending_prep[i] ? -1 : (int)(u.seq % kRefSlots);
        }
    } else {
        if (!iunits.empty()) {
            if (prep_refs(E, iunits, stage) != 0) return -3;
            stage += (sizeof(PrepTaskH) * iunits.size() + 63) / 64 * 64;
            E->launches += 2;
        }
        if (!kunits.empty()) {
            if (prep_refs(E, kunits, stage, true) != 0) return -3;
            E->launches += 2;
        }
        for (int i = 0; i < nu; ++i) {
            Unit &u = E->units[i];
            for (int k = 0; k < K; ++k) u.nref = is_intra[k * nu + i] ? 1 : (u.nref < 2 ? u.nref + 1 : 2);
            u.recon_slot = (int)((u.seq + K - 1) % kRefSlots);
            u.seq += K;
        }
    }
    for (int i = 0; i < nu; ++i) {
        const int j = (K - 1) * nu + i;
        E->prev_luma[i] = (E->src_on_device && !(force_skip && force_skip[j])) ? ud[j].cur[0] : nullptr;
    }
    for (int k = 0; k < K; ++k) {
        Slot &S = E->slot[sis[k]];
        CK(cudaMemcpyAsync(S.err_h, E->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, E->st));
        if (!pu.empty())   // the inference's error word (the main stream has waited for it)
            CK(cudaMemcpyAsync(S.err_h + 1, E->d_err_inf + hpar, sizeof(unsigned), cudaMemcpyDeviceToHost, E->st));
        else
            S.err_h[1] = 0;
        CK(cudaEventRecord(S.ev[5], E->st));
        S.has_p = !rows.empty();
        S.has_i = !itasks.empty();
        S.batch = k == K - 1 ? K : 0;
        S.streamed = streamable;
        S.ready_val = streamable ? fs_val[k] : 0u;
    }
    if (!E->src_on_device) {
        // this source set is free again once the kernels enqueued above have run
        CK(cudaEventRecord(E->ev_srcfree[par], E->st));
        E->upar ^= 1;
    }
    if (joint) {   // the lookahead frame waits in its lane for its own submission
        E->kr_ready = true;
        E->kr_planes = E->ka_planes;
        E->kr_qp = E->ka_qp;
        E->ka_armed = false;
    }
    E->stall_unit = E->stall_row = -1;     // an injected stall lasts one step
    for (int k = 0; k < K; ++k) {
        E->busy[sis[k]] = true;
        E->order.push_back(sis[k]);
    }
    E->inflight += K;
    return 0;
}

extern "C" int fdvb_engine_submit(fdvb_engine *E, const uint8_t *const *planes, const int *is_intra, const int *qp,
                                  const double *lscale, const int *force_skip) {
    return fdvb_engine_submit_batch(E, 1, planes, is_intra, qp, lscale, force_skip);
}

// The largest batch the engine takes in its present mode (1 with learned
// proposals, decision records or deferred references).
extern "C" int fdvb_engine_max_batch(const fdvb_engine *E) {
    if (!E) return 0;
    return (E->d_mbcost || E->defer_refs) ? 1 : E->tune_k;
}

// The launch shape: P-frames per launch at most (1..kMaxBatch) and blocks of
// the P-frame wavefront kernel (0: one per SM; at most the SM count).
extern "C" int fdvb_engine_set_tuning(fdvb_engine *E, int max_batch, int p_grid) {
    if (!E) return -1;
    if (max_batch < 1 || max_batch > kMaxBatch || p_grid < 0) { g_err = "tuning out of range"; return -1; }
    E->tune_k = max_batch;
    E->tune_pgrid = p_grid > E->nsm ? E->nsm : p_grid;
    return 0;
}
extern "C" void fdvb_engine_get_tuning(const fdvb_engine *E, int *max_batch, int *p_grid, int *nsm) {
    if (!E) return;
    if (max_batch) *max_batch = E->tune_k;
    if (p_grid) *p_grid = E->tune_pgrid > 0 ? E->tune_pgrid : E->nsm;
    if (nsm) *nsm = E->nsm;
}

// Wait for the oldest submitted frame; on success the stream views
// (fdvb_engine_pstreams / _istreams) describe it.
extern "C" int fdvb_engine_collect(fdvb_engine *E) {
    if (!E) return -1;
    if (E->inflight == 0) { g_err = "no frame in flight"; return -1; }
    const int si = E->order.front();
    Slot &SL = E->slot[si];
    E->order.pop_front();
    E->busy[si] = false;
    E->inflight -= 1;
    // A streamed frame that is not its batch's last is ready once its word is
    // set (the batch's errors are reported at its last frame); otherwise, or
    // when the batch ended without setting it, wait for the batch.
    bool early = false;
    if (SL.streamed && !SL.batch) {
        for (unsigned i = 0;; ++i) {
            if (*(volatile unsigned *)&E->ready_h[si] == SL.ready_val) { early = true; break; }
            const cudaError_t q = cudaEventQuery(SL.ev[5]);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) CK(q);
            if (i > 64) std::this_thread::yield();
        }
        std::atomic_thread_fence(std::memory_order_acquire);
    }
    if (!early) CK(cudaEventSynchronize(SL.ev[5]));
    E->steps += 1;
    if (SL.batch) {
        // the batch's last frame carries its timing: whole step, and the
        // P-frame kernel time counted per P-frame
        float ms = 0;
        cudaEventElapsedTime(&ms, SL.ev[0], SL.ev[5]);
        E->step_ms += ms;
        if (SL.has_p) { cudaEventElapsedTime(&ms, SL.ev[1], SL.ev[2]); E->pk_ms += ms; E->pk_n += SL.batch; }
        if (SL.has_i) { cudaEventElapsedTime(&ms, SL.ev[3], SL.ev[4]); E->ik_ms += ms; E->ik_n += 1; }
    }
    const unsigned err = early ? 0u : (SL.err_h[0] | SL.err_h[1]);
    if (err) {
        g_err = status_text(err);
        return -4;
    }
    for (int i = 0; i < (int)E->units.size(); ++i) {
        Unit &u = E->units[i];
        u.last_intra = SL.intra[i];
        if (!u.last_intra) {
            E->d2h += (long long)parse_streams(u.out_h[si], 16, &u.ps) + 16 * 256 * 4;
            u.ps.hist = u.hist_h[si];
        } else {
            for (int p = 0; p < 3; ++p) {
                E->d2h += (long long)parse_streams(u.out_h[si] + u.out_off_i[p], 12, &u.is[p]) + 12 * 256 * 4;
                u.is[p].hist = u.hist_h[si] + p * 12 * 256;
            }
        }
    }
    return 0;
}

extern "C" int fdvb_engine_step(fdvb_engine *E, const uint8_t *const *planes, const int *is_intra, const int *qp,
                                const double *lscale, const int *force_skip) {
    if (!E) return -1;
    if (E->inflight) { g_err = "a frame is still in flight"; return -1; }
    const int rc = fdvb_engine_submit(E, planes, is_intra, qp, lscale, force_skip);
    if (rc != 0) return rc;
    return fdvb_engine_collect(E);
}

extern "C" const fdvb_streams *fdvb_engine_pstreams(fdvb_engine *E, int unit) {
    if (!E || unit < 0 || unit >= (int)E->units.size() || E->units[unit].last_intra) return nullptr;
    return &E->units[unit].ps;
}
extern "C" const fdvb_streams *fdvb_engine_istreams(fdvb_engine *E, int unit, int plane) {
    if (!E || unit < 0 || unit >= (int)E->units.size() || !E->units[unit].last_intra || plane < 0 || plane > 2)
        return nullptr;
    return &E->units[unit].is[plane];
}
extern "C" int fdvb_engine_recon(fdvb_engine *E, int unit, uint8_t *i420) {
    if (!E || unit < 0 || unit >= (int)E->units.size() || !i420) return -1;
    Unit &u = E->units[unit];
    CK(cudaStreamSynchronize(E->st));
    if (u.recon_slot < 0) {
        CK(cudaMemcpy(i420, u.rec[0], (size_t)u.w * u.h * 3 / 2, cudaMemcpyDeviceToHost));
        return 0;
    }
    // the interior of the reference planes
    const RefSlot &r = u.ref[u.recon_slot];
    uint8_t *uo = i420 + (size_t)u.w * u.h, *vo = uo + (size_t)u.cw * u.ch;
    CK(cudaMemcpy2D(i420, u.w, r.G, r.rp.ys, u.w, u.h, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy2D(uo, u.cw, r.U, r.rp.cs, u.cw, u.ch, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy2D(vo, u.cw, r.V, r.rp.cs, u.cw, u.ch, cudaMemcpyDeviceToHost));
    return 0;
}
// Seed a unit's reference pool from host frames (tight I420): nearest, and the
// second one (NULL = none).  The next step then codes a P-frame against them.
extern "C" int fdvb_engine_set_refs(fdvb_engine *E, int unit, const uint8_t *near_i420, const uint8_t *far_i420) {
    if (!E || unit < 0 || unit >= (int)E->units.size() || !near_i420) return -1;
    if (E->inflight) { g_err = "a frame is still in flight"; return -1; }
    Unit &u = E->units[unit];
    const size_t fs = (size_t)u.w * u.h * 3 / 2;
    std::vector<int> one{unit};
    if (far_i420) {
        // far first: it becomes the second-nearest reference
        CK(cudaMemcpyAsync(u.rec[0], far_i420, fs, cudaMemcpyHostToDevice, E->st));
        if (prep_refs(E, one) != 0) return -3;
        CK(cudaStreamSynchronize(E->st));
        u.seq += 1;
    }
    CK(cudaMemcpyAsync(u.rec[0], near_i420, fs, cudaMemcpyHostToDevice, E->st));
    if (prep_refs(E, one) != 0) return -3;
    CK(cudaStreamSynchronize(E->st));
    u.recon_slot = (int)(u.seq % kRefSlots);
    u.seq += 1;
    u.nref = far_i420 ? 2 : 1;
    return 0;
}

// Sources of the next steps are device pointers (already resident in HBM).
extern "C" void fdvb_engine_src_on_device(fdvb_engine *E, int on) { if (E) E->src_on_device = on; }
// Host sources of the next steps stay valid and unchanged until their frames
// are collected: pinned ones are then copied without host staging.
extern "C" void fdvb_engine_direct_upload(fdvb_engine *E, int on) { if (E) E->direct_upload = on; }
// P-frames of the next submissions are streamed out of their launch: a frame
// can be collected as soon as its own rows are done (the errors of a batch are
// reported when its last frame is collected).
extern "C" void fdvb_engine_stream_frames(fdvb_engine *E, int on) { if (E) E->stream_frames = on; }
// Whether the oldest frame in flight can be collected without waiting:
// 1 yes, 0 not yet, -1 no frame in flight.
extern "C" int fdvb_engine_ready(fdvb_engine *E) {
    if (!E || E->inflight == 0) return -1;
    const int si = E->order.front();
    const Slot &SL = E->slot[si];
    if (SL.streamed && !SL.batch && *(volatile unsigned *)&E->ready_h[si] == SL.ready_val) return 1;
    return cudaEventQuery(SL.ev[5]) == cudaSuccess ? 1 : 0;
}

// Accumulated device time (CUDA events on the engine stream) of the steps, of
// the P-frame analysis kernel and of the key-frame kernel, with their counts,
// and the number of kernel launches.
extern "C" void fdvb_engine_stats(const fdvb_engine *E, double *step_ms, double *pk_ms, long long *pk_n,
                                  double *ik_ms, long long *ik_n, long long *launches, long long *steps,
                                  long long *d2h_bytes) {
    if (!E) return;
    if (d2h_bytes) *d2h_bytes = E->d2h;
    if (step_ms) *step_ms = E->step_ms;
    if (pk_ms) *pk_ms = E->pk_ms;
    if (pk_n) *pk_n = E->pk_n;
    if (ik_ms) *ik_ms = E->ik_ms;
    if (ik_n) *ik_n = E->ik_n;
    if (launches) *launches = E->launches;
    if (steps) *steps = E->steps;
}
extern "C" void fdvb_engine_stats_reset(fdvb_engine *E) {
    if (!E) return;
    E->step_ms = E->pk_ms = E->ik_ms = 0;
    E->steps = E->pk_n = E->ik_n = E->launches = E->d2h = 0;
}
// Bound on a wavefront wait before the kernel reports a timeout.
extern "C" void fdvb_engine_set_wait_ns(fdvb_engine *E, unsigned long long ns) { if (E) E->wait_ns = ns; }

// Fault injection for tests: in the next step, macroblock row `row` of unit
// `unit` is skipped, so the rows below it wait on a progress flag that nothing
// sets; their bounded waits expire and the step returns a timeout error.
extern "C" void fdvb_engine_inject_stall(fdvb_engine *E, int unit, int row) {
    if (!E) return;
    E->stall_unit = unit;
    E->stall_row = row;
}

// Per-phase cycle profile (thread 0 of each block adds clock64 deltas).
// Entries 0..15, P-frame kernel: wait, load, SKIP, searches, residuals, region
// decisions, commit, output, macroblock count, SKIP early-out count.  Entries
// 16..31, key-frame kernel: wait, 4x4 leaves, 8/16/32/64 leaves, CTU total,
// CTU count, 4x4 leaf count.  Enabling it allocates the accumulators; reading
// returns and clears them.
extern "C" int fdvb_engine_profile(fdvb_engine *E, int enable, unsigned long long *out32) {
    if (!E) return -1;
    if (enable && !E->d_prof) {
        if (cudaMalloc(&E->d_prof, 32 * sizeof(unsigned long long)) != cudaSuccess) return -3;
        cudaMemset(E->d_prof, 0, 32 * sizeof(unsigned long long));
        if (cudaMalloc(&E->d_tl, 2 * sizeof(unsigned long long) * E->total_mbs) != cudaSuccess) return -3;
        cudaMemset(E->d_tl, 0, 2 * sizeof(unsigned long long) * E->total_mbs);
    }
    if (out32 && E->d_prof) {
        cudaMemcpy(out32, E->d_prof, 32 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        cudaMemset(E->d_prof, 0, 32 * sizeof(unsigned long long));
    }
    if (!enable && E->d_prof) {
        cudaFree(E->d_prof); E->d_prof = nullptr;
        cudaFree(E->d_tl); E->d_tl = nullptr;
    }
    return 0;
}

// The last P-frame's per-macroblock timeline of unit u (phase profile on):
// out[2 m] the end of macroblock m's wait, out[2 m + 1] its publication,
// %globaltimer nanoseconds.
extern "C" int fdvb_engine_timeline(fdvb_engine *E, int u, unsigned long long *out) {
    if (!E || !E->d_tl || u < 0 || u >= (int)E->units.size() || !out) return -1;
    const Unit &U = E->units[u];
    if (cudaStreamSynchronize(E->st) != cudaSuccess) return -3;
    return cudaMemcpy(out, E->d_tl + 2 * (size_t)U.mb_off, 2 * sizeof(unsigned long long) * U.mbw * U.mbh,
                      cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -3;
}

// Re-coding support (average-bitrate control codes a frame again, coarser,
// when it overshoots): while deferral is on, a step leaves the reference pool
// untouched, so the same frame can be stepped again against the same
// references; commit then makes the last step's reconstruction the nearest
// reference.  Only one frame may be in flight while deferring.
extern "C" void fdvb_engine_defer_refs(fdvb_engine *E, int on) { if (E) E->defer_refs = on; }
extern "C" int fdvb_engine_commit_refs(fdvb_engine *E) {
    if (!E) return -1;
    if (!E->pending) return 0;
    if (E->inflight) { g_err = "a frame is still in flight"; return -1; }
    CK(cudaSetDevice(E->device));
    const int nu = (int)E->units.size();
    // key frames and learned-form P-frames: prepare the reference now; the
    // other P-frames wrote theirs inside the wavefront
    std::vector<int> iu;
    for (int i = 0; i < nu; ++i) if (E->pending_prep[i]) iu.push_back(i);
    if (!iu.empty()) {
        if (prep_refs(E, iu) != 0) return -3;
        E->launches += 2;
    }
    CK(cudaStreamSynchronize(E->st));
    for (int i = 0; i < nu; ++i) {
        Unit &u = E->units[i];
        u.nref = E->pending_intra[i] ? 1 : (u.nref < 2 ? u.nref + 1 : 2);
        u.recon_slot = (int)(u.seq % kRefSlots);
        u.seq += 1;
    }
    E->pending = false;
    return 0;
}

// Learned proposals for every later P-frame (params: fdvl_nparams() floats;
// NULL turns them off).  The engine owns a private inference network.
// Default SKIP gate, in units of lambda: static macroblocks' best merge
// candidate costs around 100-300 lambda, a wrongly predicted SKIP over moving
// content far more.
constexpr double kLearnSkipGate = 400.0;
extern "C" int fdvb_engine_set_learned(fdvb_engine *E, const float *params, float conf) {
    if (!E) return -1;
    CK(cudaSetDevice(E->device));
    if (!params) {
        if (E->lnet) { cudaStreamSynchronize(E->st); fdvl_destroy(E->lnet); E->lnet = nullptr; }
        return 0;
    }
    if (!E->lnet) {
        // sized for a batch: every P-frame of a launch is inferred in one pass
        E->lnet = lrn_create(E->device, kMaxBatch * E->total_mbs, 0, 16, 16);
        if (!E->lnet) { g_err = std::string("learned network: ") + fdvl_last_error(); return -3; }
        if (!E->d_hints) CK(cudaMalloc(&E->d_hints, sizeof(lrn::Hint) * 2 * kMaxBatch * E->total_mbs));
        if (!E->d_prejs) CK(cudaMalloc(&E->d_prejs, sizeof(float) * 2 * kMaxBatch * E->total_mbs));
        if (!E->d_pu) CK(cudaMalloc(&E->d_pu, sizeof(int2) * kMaxBatch * E->units.size()));
        for (int k = 0; k < 2; ++k) {
            if (!E->d_units_inf[k]) CK(cudaMalloc(&E->d_units_inf[k], sizeof(UnitDev) * kMaxBatch * E->units.size()));
            if (!E->d_pu_inf[k]) CK(cudaMalloc(&E->d_pu_inf[k], sizeof(int2) * kMaxBatch * E->units.size()));
        }
    }
    CK(cudaStreamSynchronize(E->st));
    if (fdvl_set_params(E->lnet, params) != 0) { g_err = std::string("learned network: ") + fdvl_last_error(); return -3; }
    // the product setting: every class narrowed at `conf` (SKIP behind the
    // RD-cost gate, inter keeping INTER8); every full search seeded with the
    // proposals
    E->lconf = make_float3(conf, conf, conf);
    E->lgate = kLearnSkipGate;
    E->linter8 = 1;
    return 0;
}

// Per-class confidence thresholds of the learned proposals (SKIP, inter,
// intra; a threshold above 1 turns that class's narrowed analysis off), the
// SKIP gate (a confident SKIP is taken only when the best merge candidate's
// RD cost is at most gate * lambda; gate <= 0: always) and whether the
// confident-inter path also tries INTER8.
extern "C" int fdvb_engine_learned_conf(fdvb_engine *E, const float *conf5) {
    if (!E || !conf5) return -1;
    E->lconf = make_float3(conf5[0], conf5[1], conf5[2]);
    E->lgate = conf5[3];
    E->linter8 = conf5[4] != 0.f;
    return 0;
}

// Per-macroblock decision records of the last collected P-frame: mode
// (0 SKIP, 1 INTER16, 2 INTRA16, 3 INTER8), MV (the neighbour-prediction
// vector: INTER8 keeps its last quadrant's), reference and RD cost (when
// enabled before the frame).  Any output may be NULL.
extern "C" int fdvb_engine_records(fdvb_engine *E, int enable) {
    if (!E) return -1;
    CK(cudaSetDevice(E->device));
    if (enable && !E->d_mbcost) {
        CK(cudaMalloc(&E->d_mbcost, sizeof(float) * E->total_mbs));
        CK(cudaMemset(E->d_mbcost, 0, sizeof(float) * E->total_mbs));
    } else if (!enable && E->d_mbcost) {
        cudaStreamSynchronize(E->st);
        cudaFree(E->d_mbcost);
        E->d_mbcost = nullptr;
    }
    return 0;
}

extern "C" int fdvb_engine_mb_records(fdvb_engine *E, int unit, uint8_t *mode, int16_t *mv, uint8_t *ref, float *cost) {
    if (!E || unit < 0 || unit >= (int)E->units.size()) { g_err = "bad unit"; return -1; }
    CK(cudaSetDevice(E->device));
    CK(cudaStreamSynchronize(E->st));
    Unit &u = E->units[unit];
    const int n = u.mbw * u.mbh;
    std::vector<MBInfo> mi(n);
    CK(cudaMemcpy(mi.data(), u.mbi[0], sizeof(MBInfo) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
        if (mode) mode[i] = mi[i].mode;
        if (mv) { mv[2 * i] = mi[i].x; mv[2 * i + 1] = mi[i].y; }
        if (ref) ref[i] = mi[i].ref;
    }
    if (cost) {
        if (!E->d_mbcost) { g_err = "cost records are off"; return -1; }
        CK(cudaMemcpy(cost, E->d_mbcost + u.mb_off, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    return 0;
}

// All analysis kernels in one translation unit, so the constant-memory tables
// (the H.264 quant tables, the scans, and the host-computed 8x8 DCT basis and
// quantiser steps) exist once, plus the host-callable launch wrappers the
// engine uses.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "frame_ops.cuh"
#include "iframe.cuh"
#include "pframe.cuh"

namespace fdvb {

int upload_tables(const int32_t c8[64], const int32_t q8[52]) {
    int32_t c8t[64];
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) c8t[j * 8 + i] = c8[i * 8 + j];
    if (cudaMemcpyToSymbol(g_C8, c8, sizeof(int32_t) * 64) != cudaSuccess ||
        cudaMemcpyToSymbol(g_C8T, c8t, sizeof(int32_t) * 64) != cudaSuccess ||
        cudaMemcpyToSymbol(c_QSTEP8, q8, sizeof(int32_t) * 52) != cudaSuccess)
        return -1;
    return 0;
}

void launch_iframe(const void *planes, const void *tasks, int ntasks, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, cudaStream_t st) {
    // the shared-memory opt-in is a per-device attribute: set once per device
    static std::mutex mu;
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = sizeof(IShared);
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64 && !attr[dev]) {
            cudaFuncSetAttribute(iframe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr[dev] = true;
        }
    }
    // clusters of ICL blocks, one CTU row each at a time; `grid` is the SM count
    const int ncl = std::max(1, std::min(ntasks, grid / ICL));
    iframe_kernel<<<ncl * ICL, INT, smem, st>>>(static_cast<const IPlaneDev *>(planes), static_cast<const ITask *>(tasks),
                                                ntasks, ticket, err, wait_ns);
}

// The P-frame kernel stages the references' luma in shared memory when the
// search range allows it (up to 32); a range of 64 reads them from global
// memory.  All units of one launch share the range.
void launch_pframe(const UnitDev *units, const RowTask *rows, int nrows, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, int range, bool learned, cudaStream_t st,
                   const FrameSync *fsync, const void *ctasks, int *fdone, int nu, int nunits) {
    static std::mutex mu;
    static bool attr[64][8] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const bool win = range <= 32;
    const int v = (win ? 1 : 0) + (learned ? 2 : 0) + (fsync ? 4 : 0);
    const size_t smem = win ? (size_t)kPWinOff + kPWinBytes : sizeof(PShared);
    void (*const k[8])(const UnitDev *, const RowTask *, int, int *, unsigned *, unsigned long long, const FrameSync *,
                       const CompactTask *, int *, int, int) = {
        pframe_kernel<false, false, false>, pframe_kernel<true, false, false>, pframe_kernel<false, true, false>,
        pframe_kernel<true, true, false>,   pframe_kernel<false, false, true>,  pframe_kernel<true, false, true>,
        pframe_kernel<false, true, true>,   pframe_kernel<true, true, true>};
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64 && !attr[dev][v]) {
            cudaFuncSetAttribute(k[v], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr[dev][v] = true;
        }
    }
    k[v]<<<grid, PNT, smem, st>>>(units, rows, nrows, ticket, err, wait_ns, fsync,
                                  static_cast<const CompactTask *>(ctasks), fdone, nu < 1 ? 1 : nu, nunits);
}

// The learned form's SKIP pre-analysis, one warp per macroblock of the P
// units (pu: {unit, first macroblock}), between the inference and the
// wavefront: a macroblock the network calls SKIP confidently gets the zero
// vector's SKIP analysed here -- prediction, SSD, RD cost, the gate -- and,
// when the gate passes, its reconstruction written and its cost kept in
// prejs; the wavefront commits it without analysis when its merge list turns
// out to be {zero vector on reference 0}, which gives the same SKIP
// (pframe_kernel).  Otherwise prejs is -1.
__global__ void __launch_bounds__(128) lrn_preskip_kernel(const UnitDev *__restrict__ units, const int2 *__restrict__ pu,
                                                          int np, int total) {
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (gw >= total) return;
    int k = 0;
    while (k + 1 < np && gw >= pu[k + 1].y) ++k;
    const UnitDev &U = units[pu[k].x];
    const int m = gw - pu[k].y;
    float *pj = const_cast<float *>(U.prejs) + m;
    if (U.hint[m].cls != 0) {
        if (lane == 0) *pj = -1.f;
        return;
    }
    const int w = U.w, bx = (m % U.mbw) * 16, by = (m / U.mbw) * 16;
    const RefPlanes &R = U.ref[0];
    const int r = lane >> 1, c = (lane & 1) * 8;   // a lane: 8 samples of one row
    const uint8_t *cp = U.cur[0] + (size_t)(by + r) * w + bx + c;
    const uint8_t *rp = R.G + (long)(by + r) * R.ys + bx + c;
    uint8_t pv[8];
    int s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        pv[i] = rp[i];
        const int d = (int)cp[i] - (int)pv[i];
        s += d * d;
    }
    s = __reduce_add_sync(FDVB_FULL, s);
    const double Js = rd_cost((double)s, U.lambda, kBitsMode);   // one merge candidate: no index bits
    if (!(U.skip_gate <= 0.0 || Js <= __dmul_rn(U.skip_gate, U.lambda))) {
        if (lane == 0) *pj = -1.f;
        return;
    }
    uint8_t *dr = U.rec[0] + (size_t)(by + r) * w + bx + c;
#pragma unroll
    for (int i = 0; i < 8; ++i) dr[i] = pv[i];
    const int cw = w / 2, cbx = bx / 2, cby = by / 2;
    for (int q = lane; q < 128; q += 32) {
        const int pl = q >> 6, p = q & 63;
        U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] =
            (uint8_t)mc_cpx(pl ? R.V : R.U, R.cs, cbx + (p & 7), cby + (p >> 3), 0, 0);
    }
    if (lane == 0) *pj = (float)Js;
}

void launch_lrn_preskip(const UnitDev *units, const int2 *pu, int np, int total, cudaStream_t st) {
    lrn_preskip_kernel<<<(total + 3) / 4, 128, 0, st>>>(units, pu, np, total);
}

void launch_refprep(const void *tasks, int ntasks, int maxw, int maxh, int border, cudaStream_t st) {
    if (border & 3) return;   // the kernels store 4 samples at a time from padded column 0
    dim3 blk(32, 8);
    dim3 gl((maxw + 2 * border + kRpTW - 1) / kRpTW, (maxh + 2 * border + kRpTH - 1) / kRpTH, ntasks);
    refprep_luma_kernel<<<gl, blk, 0, st>>>(static_cast<const PrepTask *>(tasks));
    dim3 gc((maxw / 2 + 2 * border + 127) / 128, (maxh / 2 + 2 * border + 7) / 8, ntasks);
    refprep_chroma_kernel<<<gc, blk, 0, st>>>(static_cast<const PrepTask *>(tasks));
}

void launch_deblock(const void *tasks, int ntasks, cudaStream_t st) {
    dim3 g(64, 1, ntasks);
    deblock_v_kernel<<<g, 256, 0, st>>>(static_cast<const DbTask *>(tasks));
    deblock_h_kernel<<<g, 256, 0, st>>>(static_cast<const DbTask *>(tasks));
}

void launch_compact(const void *tasks, int ntasks, unsigned *err, cudaStream_t st) {
    compact_kernel<<<ntasks, 1024, 0, st>>>(static_cast<const CompactTask *>(tasks), err);
}

}  // namespace fdvb

// ===================================================================
// Allocation-free P-frame analysis of one unit.
//
// Some callers cannot allocate device memory while they encode: a host that
// owns the GPU's memory itself (a media framework or inference server with its
// own pool, where a stray cudaMalloc competes with it or is forbidden), a
// real-time capture path that cannot take cudaMalloc's implicit device
// synchronisation in the middle of a frame, and code that must not grow the
// process's device footprint after start-up.  For them this entry point runs
// the whole P-frame analysis step -- reference preparation, the macroblock
// wavefront, deblocking and symbol compaction -- with every piece of scratch
// (padded reference planes, per-macroblock symbol slots, motion map, progress
// flags, launch descriptors) carved from one file-scope device array, so the
// call itself allocates nothing.  The caller passes its own device buffers for
// the inputs and outputs.
// ===================================================================
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../host/fdvb_internal.h"

namespace {

// 24 MiB: enough for one 1280x720 unit at any supported search range
// (padded reference planes for two references + one symbol slot per
// macroblock).  Every GPU that loads the library holds this array until the
// process exits.
constexpr size_t kStaticScratchBytes = (size_t)24 << 20;

}  // namespace

static __device__ __align__(256) uint8_t g_static_scratch[kStaticScratchBytes];

namespace {

struct StaticSetup {
    bool done = false;
    uint8_t *ptr = nullptr;     // device address of g_static_scratch on this device
    int nsm = 0;
};
StaticSetup g_static_setup[64];
std::mutex g_static_mu;
thread_local char g_static_err[256];

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

int static_fail(const char *msg) {
    snprintf(g_static_err, sizeof g_static_err, "%s", msg);
    return -1;
}

}  // namespace

extern "C" const char *fdvg_pframe_static_error(void) { return g_static_err; }

extern "C" size_t fdvg_pframe_static_capacity(void) { return kStaticScratchBytes; }

extern "C" int fdvg_pframe_static(const uint8_t *cur, const uint8_t *near_ref, const uint8_t *far_ref,
                                  uint8_t *rec, int w, int h, int qp, double lscale, int range,
                                  uint8_t *out, size_t out_cap, void *stream) {
    using namespace fdvb;
    g_static_err[0] = 0;
    if (!cur || !near_ref || !rec || !out) return static_fail("null buffer");
    // the kernels read and write these buffers in 4- to 16-byte words
    if ((reinterpret_cast<uintptr_t>(cur) | reinterpret_cast<uintptr_t>(near_ref) |
         reinterpret_cast<uintptr_t>(far_ref) | reinterpret_cast<uintptr_t>(rec) | reinterpret_cast<uintptr_t>(out)) & 15)
        return static_fail("cur, near_ref, far_ref, rec and out must be 16-byte aligned");
    if (w <= 0 || h <= 0 || (w & 15) || (h & 15) || w > 8192 || h > 8192)
        return static_fail("dimensions must be positive multiples of 16");
    if (qp < 0 || qp > 51) return static_fail("qp out of range");
    if (range != 16 && range != 32 && range != 64) return static_fail("search range must be 16, 32 or 64");
    if (out_cap < 64) return static_fail("output buffer too small");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return static_fail("no CUDA device");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        // Set-up, once per device, with that device current: the array's name
        // is only a host-side stand-in, so its device address is looked up here
        // and passed to the kernels.
        std::lock_guard<std::mutex> lk(g_static_mu);
        StaticSetup &S = g_static_setup[dev];
        if (!S.done) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess || !p) return static_fail("cudaGetSymbolAddress of the static scratch failed");
            int32_t c8[64], q8[52];
            fdvb_c8_tables(c8, q8);
            if (upload_tables(c8, q8) != 0) return static_fail("table upload failed");
            cudaDeviceGetAttribute(&S.nsm, cudaDevAttrMultiProcessorCount, dev);
            S.ptr = static_cast<uint8_t *>(p);
            S.done = true;
        }
    }
    const StaticSetup &S = g_static_setup[dev];

    // Carve the scratch.
    const int B = range + 16, cw = w / 2, ch = h / 2, mbw = w / 16, mbh = h / 16, nmb = mbw * mbh;
    const int ys = (w + 2 * B + 63) / 64 * 64, cs = (cw + 2 * B + 63) / 64 * 64;
    const size_t lsz = (size_t)ys * (h + 2 * B), csz = (size_t)cs * (ch + 2 * B);
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off = align256(off + n); return o; };
    size_t o_ref[2], o_mbi, o_slots, o_prog, o_misc, o_unit, o_rows, o_prep, o_db, o_cmp, o_off;
    for (int r = 0; r < 2; ++r) o_ref[r] = take(4 * lsz + 2 * csz);
    o_mbi = take(sizeof(MBInfo) * nmb);
    o_slots = take((size_t)kSlotBytes * nmb);
    o_prog = take(sizeof(unsigned long long) * mbh);
    o_misc = take(16);                       // ticket[2], error word
    o_unit = take(sizeof(UnitDev));
    o_rows = take(sizeof(RowTask) * mbh);
    o_prep = take(sizeof(PrepTask) * 2);
    o_db = take(sizeof(DbTask) * 3);
    o_cmp = take(sizeof(CompactTask));
    o_off = take(sizeof(int) * 16);
    if (off > kStaticScratchBytes) {
        snprintf(g_static_err, sizeof g_static_err,
                 "unit %dx%d at search range %d needs %zu bytes of scratch; the static scratch holds %zu "
                 "(about 1280x720 at most)", w, h, range, off, kStaticScratchBytes);
        return -1;
    }
    uint8_t *base = S.ptr;

    // Descriptors (host staging on the stack; the stream is synchronised
    // before they go out of scope).
    RefPlanes rp[2];
    PrepTask prep[2];
    const uint8_t *srcs[2] = {near_ref, far_ref ? far_ref : near_ref};
    for (int r = 0; r < 2; ++r) {
        uint8_t *m = base + o_ref[r];
        RefPlanes &R = rp[r];
        uint8_t *G = m + (size_t)B * ys + B, *Bp = G + lsz, *Hp = Bp + lsz, *Jp = Hp + lsz;
        uint8_t *U = m + 4 * lsz + (size_t)B * cs + B, *V = U + csz;
        R.G = G; R.B = Bp; R.H = Hp; R.J = Jp; R.U = U; R.V = V; R.ys = ys; R.cs = cs;
        PrepTask &t = prep[r];
        t.rec[0] = srcs[r]; t.rec[1] = srcs[r] + (size_t)w * h; t.rec[2] = t.rec[1] + (size_t)cw * ch;
        t.G = G; t.B = Bp; t.H = Hp; t.J = Jp; t.U = U; t.V = V;
        t.w = w; t.h = h; t.ys = ys; t.cs = cs; t.border = B;
    }
    UnitDev u;
    u.w = w; u.h = h; u.mbw = mbw; u.mbh = mbh;
    u.cur[0] = cur; u.cur[1] = cur + (size_t)w * h; u.cur[2] = u.cur[1] + (size_t)cw * ch;
    u.rec[0] = rec; u.rec[1] = rec + (size_t)w * h; u.rec[2] = u.rec[1] + (size_t)cw * ch;
    u.ref[0] = rp[0];
    u.ref[1] = far_ref ? rp[1] : rp[0];
    u.mbi = reinterpret_cast<MBInfo *>(base + o_mbi);
    u.progress = reinterpret_cast<int *>(base + o_prog);
    u.slots = base + o_slots;
    u.lambda = fdvb_lambda(qp, lscale);
    u.qp = qp; u.navail = far_ref ? 2 : 1; u.force_skip = 0; u.range = range; u.stall_row = -1; u.prof = nullptr;
    u.hint = nullptr; u.mbcost = nullptr; u.skip_gate = 0.0; u.inter8 = 0; u.prejs = nullptr; u.tl = nullptr;
    u.out = OutPlanes{}; u.post_prog = nullptr; u.ref_prog = nullptr; u.lref = nullptr; u.lrs = 0;
    RowTask rows[8192 / 16];
    for (int r = 0; r < mbh; ++r) rows[r] = {0, r};
    DbTask db[3] = {{rec, w, h, qp}, {rec + (size_t)w * h, cw, ch, qp}, {rec + (size_t)w * h + (size_t)cw * ch, cw, ch, qp}};
    int poff[16];
    for (int k = 0; k < 16; ++k) { int o = 0; for (int i = 0; i < k; ++i) o += kSlotCap[i]; poff[k] = o; }
    CompactTask cmp;
    cmp.slots = base + o_slots; cmp.nslots = nmb; cmp.slot_bytes = kSlotBytes; cmp.nstreams = 16;
    cmp.off = reinterpret_cast<const int *>(base + o_off); cmp.out = out; cmp.cap = out_cap; cmp.hist = nullptr;
    cmp.tmp = nullptr;   // the output is device memory: assembled in place

    int *ticket = reinterpret_cast<int *>(base + o_misc);
    unsigned *err = reinterpret_cast<unsigned *>(base + o_misc + 8);
    bool ok = cudaMemcpyAsync(base + o_prep, prep, sizeof prep, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(base + o_unit, &u, sizeof u, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(base + o_rows, rows, sizeof(RowTask) * mbh, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(base + o_db, db, sizeof db, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(base + o_cmp, &cmp, sizeof cmp, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(base + o_off, poff, sizeof poff, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              // what must start at zero: progress flags, row ticket, error word
              cudaMemsetAsync(base + o_prog, 0, sizeof(unsigned long long) * mbh, st) == cudaSuccess &&
              cudaMemsetAsync(base + o_misc, 0, 16, st) == cudaSuccess;
    if (!ok) return static_fail("descriptor upload failed");
    launch_refprep(base + o_prep, far_ref ? 2 : 1, w, h, B, st);
    launch_pframe(reinterpret_cast<const UnitDev *>(base + o_unit), reinterpret_cast<const RowTask *>(base + o_rows),
                  mbh, ticket, err, 4000000000ull, mbh < S.nsm ? mbh : S.nsm, range, false, st, nullptr, nullptr, nullptr, 1, 0);
    launch_deblock(base + o_db, 3, st);
    launch_compact(base + o_cmp, 1, err, st);
    if (cudaGetLastError() != cudaSuccess) return static_fail("kernel launch failed");
    unsigned herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return static_fail("device error");
    if (herr) return static_fail(status_text(herr));
    return 0;
}

// The P-frame analysis loop as one persistent wavefront kernel.
//
// Work unit: one macroblock row of one encoder unit (a band or a stream).
// Blocks take rows from an atomic ticket in (unit, row) order, so every row a
// block waits on was taken earlier by a block that is already running.  A row
// proceeds left to right; macroblock x of row y starts once row y-1 has
// finished macroblock x+1 -- exactly the samples and motion it reads: the
// reconstruction above and above-left for intra prediction, the above and
// above-right motion for merge candidates, and the above mode for the mode
// context.  The waits are bounded and report a timeout instead of hanging.
//
// A macroblock runs the reference's decision procedure (pframe_encode,
// fdv.h:5808-6162) on 512 threads in four phases:
//   0. SKIP: the merge candidates' predictions and squared errors; if SKIP
//      wins outright (Js <= lambda * 14) nothing else is evaluated.
//   1. Searches, concurrently on four groups of four warps: the 16x16 search
//      on the nearest reference, on the second reference, the chain of four
//      8x8 quadrant searches, and the SATD screen of the intra sub-modes.
//   2. Residuals of every candidate at once: up to three 16x16 residuals and
//      four 8x8 ones -- every 4x4 block on a warp (RDOQ candidates on lanes),
//      every 8x8 option on 64 threads -- then each candidate's per-region
//      transform-size decisions.
//   3. The reference's sequential mode decision replayed on those results:
//      reference break (lambda * 16), intra gate (lambda * 14), INTER8 gate
//      (lambda * 19 and the SAD ratio), strict-less selection in the order
//      SKIP, INTER16, INTRA, INTER8.  Candidates computed but not reached by
//      that flow are ignored, so the decisions are the reference's.  Then
//      chroma, reconstruction and the symbols of the chosen mode.
#include "common.cuh"
#include "engine_dev.cuh"
#include "frame_ops.cuh"
#include "inter.cuh"
#include "intra.cuh"
#include "post.cuh"
#include "residual.cuh"

namespace fdvb {

constexpr int PNT = 512;

struct PShared {
    QP4 q;
    uint8_t cur[256], curc[2][64];
    uint8_t top[16], left[16], ctop[2][8], cleft[2][8];
    int tl, ht, hl, ctl[2];
    MBInfo cand[3];
    int ncand, ssd3[3];
    uint8_t predS[3][256];
    // phase 1
    uint8_t pr[3][256];          // 16x16 predictions: nearest ref, second ref, selected intra
    uint8_t pred8[4][64];        // INTER8 quadrant predictions
    int mv[2][2], sad[2];
    int qmv[4][2], ssad;
    int isel;
    int satd[64];
    NNPred nn[4];
    int gsad[4][16];
    // phase 2: regions 0-3 nearest ref, 4-7 second ref, 8-11 intra, 12-15 INTER8 quadrants
    Blk4 blk[64];
    uint8_t recA[16][64];
    Reg8 reg[16];
    Reg8WScratch r8w[16];        // per warp: a region's 8x8 option
    Reg8Scratch r8[2];           // chroma 8x8 options (64 threads each)
    Blk4Scratch b4[32];          // per warp, two per warp for paired blocks
    RegDec dec[16];
    CoefSink sink[4];
    uint8_t sinkmem[4][kCsBytes];
    long long cD[4];
    int cB[4];
    // chroma
    uint8_t cpred[2][64], crec[2][64], cpred4[8][16];
    Blk4 cblk[8];
    Reg8 creg[2];
    RegDec cdec[2];
    long long ce;
    int cb;
    int task, row_ok, amode;
    // (appended last, so the members above keep their offsets)
    alignas(16) uint8_t pre[256];   // the next macroblock's source, prefetched by cp.async
    alignas(8) uint8_t prec[2][64];
    short2 lmv[lrn::kMvHyp];     // learned proposals of this macroblock
    short2 lmv2[lrn::kMvHyp];    // the same doubled, for the second reference (two frames back)
    int lcls;                    // their confident class, -1: none
    // learned form, indexed by macroblock parity (a fast macroblock has no
    // barrier after its reads, so thread 0 may already write the next one's)
    uint2 nbi[2][2];             // the above and above-right macroblock records
    float pjs[2];                // prejs of the macroblock
    int fast[2];                 // a pre-analysed zero-vector SKIP whose merge list is {0}
    int rok[2];                  // row_ok
    int amz[2];                  // the above macroblock's mode is not SKIP
    int pok;                     // the row's first reference wait succeeded
    // the reference output stage (post.cuh) while a row runs; a finished
    // frame's compaction (FrameSync launches) after the row's last tiles
    union {
        PostScratch post;
        CompactScratch<512> cmp;
    };
    int lastrow;                 // this block finished the frame's last row
};

__device__ __forceinline__ uint8_t ldcg8(const uint8_t *p) { return __ldcg(p); }

// A row's 64-bit progress word: bits 0-11 the macroblocks it has finished;
// bits 16-63 the record of the last of them (reference bit 16, inter bit 17,
// mode bits 18-19, vector x bits 32-47, y bits 48-63).
__device__ __forceinline__ unsigned long long prog_word(int count, const MBInfo &m) {
    return (unsigned long long)count | ((unsigned long long)(m.ref & 1u) << 16) |
           ((unsigned long long)(m.inter & 1u) << 17) | ((unsigned long long)(m.mode & 3u) << 18) |
           ((unsigned long long)(uint16_t)m.x << 32) | ((unsigned long long)(uint16_t)m.y << 48);
}
// The record in a progress word, packed as MBInfo is in memory ({x, y},
// {ref, inter, mode, 0}).
__device__ __forceinline__ uint2 prog_rec(unsigned long long v) {
    return make_uint2((uint32_t)(v >> 32), (uint32_t)((v >> 16) & 1u) | ((uint32_t)((v >> 17) & 1u) << 8) |
                                               ((uint32_t)((v >> 18) & 3u) << 16));
}

// Optional phase profile: thread 0 adds the cycles since the last mark.
struct PhaseClock {
    unsigned long long *acc;
    long long t;
    __device__ void start() { if (acc) t = clock64(); }
    __device__ void mark(int ph) {
        if (acc) { long long n = clock64(); atomicAdd(&acc[ph], (unsigned long long)(n - t)); t = n; }
    }
};

__device__ void write_slot_structs(uint8_t *slot, int k, const uint8_t *b, int n, unsigned *err) {
    uint16_t *len = slot_len(slot);
    if (len[k] + n > c_SlotCap[k]) { atomicOr(err, kErrSlotOverflow); return; }
    uint8_t *d = slot_data(slot, k) + len[k];
    for (int i = 0; i < n; ++i) d[i] = b[i];
    len[k] = (uint16_t)(len[k] + n);
}

// 16x16 prediction of a group of 128 threads (threads 0..63 one word each).
template <class Src>
__device__ __forceinline__ void mc16_group(const Src &R, int bx, int by, int mvx, int mvy, uint8_t *dst, int gt) {
    if (gt < 64) {
        const int row = gt >> 2, col = (gt & 3) * 4, ph = (mvy & 3) * 4 + (mvx & 3);
        reinterpret_cast<uint32_t *>(dst)[gt] = mc_word_nb(R, bx + col + (mvx >> 2), by + row + (mvy >> 2), ph);
    }
}

// ----------------------------------------------- reference window --
// With a search range up to 32 the luma planes of both references around the
// current macroblock are staged in shared memory: a ring of kWinRing columns
// (eight 16-column strips) by 2 * range + 23 rows per plane, which covers every
// sample a vector within the search range (plus the quarter-pel refinement
// and the interpolation taps) can touch.  Macroblock x reads strips x-3..x+3;
// while it runs, strip x+4 is copied in (cp.async) for macroblock x+1, into the
// ring slot of strip x-4, which is no longer read.
constexpr int kPWinOff = (int)((sizeof(PShared) + 127) / 128 * 128);
constexpr int kPWinBytes = 8 * kWinPlane;   // 2 references x 4 planes

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copy strips s0..s1 (clipped to the padded plane) of the window rows
// wy0 .. wy0 + wrows - 1 of nref references (all threads; one commit group).
__device__ void win_fill(uint8_t *win, const UnitDev &U, int nref, int s0, int s1, int wy0, int wrows, int tid) {
    const int B = U.range + 16, smin = -B / 16, smax = (U.w + B) / 16 - 1;
    s0 = s0 < smin ? smin : s0;
    s1 = s1 > smax ? smax : s1;
    if (s1 >= s0) {
        const int per = nref * 4 * wrows, total = (s1 - s0 + 1) * per;
        for (int i = tid; i < total; i += PNT) {
            const int si = i / per, rem = i - si * per, pr = rem / wrows, row = rem - pr * wrows;
            const int r = pr >> 2, p = pr & 3, x = 16 * (s0 + si);
            const RefPlanes &RP = U.ref[r];
            const uint8_t *pl = p == 0 ? RP.G : (p == 1 ? RP.B : (p == 2 ? RP.H : RP.J));
            cp_async16(win + (r * 4 + p) * kWinPlane + row * kWinStride + (x & (kWinRing - 1)),
                       pl + (long)(wy0 + row) * RP.ys + x);
        }
    }
    cp_async_commit();
}

template <bool WIN> struct LumaOf { using T = GlobalLumaCG; };
template <> struct LumaOf<true> { using T = WindowLuma; };
template <bool WIN>
__device__ __forceinline__ typename LumaOf<WIN>::T luma_src(const RefPlanes &R, const uint8_t *win, int r, int wy0, int wrows);
template <>
__device__ __forceinline__ GlobalLumaCG luma_src<false>(const RefPlanes &R, const uint8_t *, int, int, int) {
    return GlobalLumaCG(R);
}
template <>
__device__ __forceinline__ WindowLuma luma_src<true>(const RefPlanes &, const uint8_t *win, int r, int wy0, int wrows) {
    return WindowLuma{win + r * 4 * kWinPlane, wy0, wrows - 1};
}

// One residual warp task of region g (regions 4c..4c+3 belong to candidate c:
// 0, 1 INTER16 on the two references, 2 INTRA16, 3 INTER8): j = 0, 1 the 4x4
// block pairs 0-1 and 2-3 (one per half-warp), j = 2 the 8x8 option.
// Not inlined (nor group_decide below): one copy of their code serves every
// call site, which keeps the kernel's instruction footprint within the SM's
// instruction cache.
__device__ __noinline__ void resid_task(PShared &S, int g, int j, int qp, double lambda, int warp, int lane) {
    const uint8_t *cp, *pp;
    int pstr;
    if (g < 12) {
        const int c = g >> 2, rr = g & 3, rx = (rr & 1) * 8, ry = (rr >> 1) * 8;
        cp = S.cur + ry * 16 + rx; pp = S.pr[c] + ry * 16 + rx; pstr = 16;
    } else {
        const int q = g - 12, qx = (q & 1) * 8, qy = (q >> 1) * 8;
        cp = S.cur + qy * 16 + qx; pp = S.pred8[q]; pstr = 8;
    }
    if (j < 2) {
        const int s0 = 2 * j, sy = j * 4;
        warp_block4x2(cp + sy * 16, cp + sy * 16 + 4, 16, pp + sy * pstr, pp + sy * pstr + 4, pstr, &S.recA[g][sy * 8],
                      &S.recA[g][sy * 8 + 4], 8, S.q, lambda, true, &S.blk[4 * g + s0], &S.blk[4 * g + s0 + 1],
                      &S.b4[2 * warp], lane);
    } else {
        warp_region8(cp, 16, pp, pstr, qp, &S.reg[g], &S.r8w[warp], lane);
    }
}

// Candidate c's region decisions (fdv.h:5379-5411) on the four warps of a
// group (barrier `bar`): transform choices, stream offsets in region order,
// one warp per region copying its symbols; distortion and rate to cD/cB.
__device__ __noinline__ void group_decide(PShared &S, int c, double lambda, int gw, int gt, int lane, int bar,
                                             unsigned *err) {
    if (gt < 4) region_choice(&S.blk[4 * (4 * c + gt)], S.reg[4 * c + gt], lambda, S.dec[4 * c + gt]);
    gbar(bar, 128);
    if (gt == 0) {
        S.cD[c] = 0;
        S.cB[c] = 0;
        region_offsets(&S.dec[4 * c], 4, &S.sink[c], false, &S.cD[c], &S.cB[c], err);
    }
    gbar(bar, 128);
    region_symbols(S.dec[4 * c + gw], &S.blk[4 * (4 * c + gw)], S.reg[4 * c + gw], &S.sink[c], false, lane);
}

// Warp groups 0, 1 and 3 meet here after their searches (the pool of twelve
// warps that codes the INTER16 and INTRA16 residuals while group 2 still
// runs the INTER8 chain).
constexpr int BAR_POOL = 13;

// Large-diamond steps of the 16x16 search when it starts from learned proposals.
constexpr int kLearnLd = 4;

// LRN: the learned-proposal form (units carry hints); the plain instance has
// none of its code.
//
// FS: the streaming form.  fsync holds per frame of the launch (units j =
// frame * nu + i) its host-mapped ready word; the block that finishes unit
// j's last row compacts ctasks[j], and the last unit of a frame sets the
// frame's ready word (FrameSync).  fdone: per unit j its finished rows, then
// per frame its compacted units.  The other instances ignore the three and
// carry none of that code.
template <bool WIN, bool LRN, bool FS>
__global__ void __launch_bounds__(PNT, 1)
pframe_kernel(const UnitDev *__restrict__ units, const RowTask *__restrict__ rows, int nrows,
              int *ticket, unsigned *err, unsigned long long wait_ns, const FrameSync *__restrict__ fsync,
              const CompactTask *__restrict__ ctasks, int *fdone, int nu, int nunits) {
    extern __shared__ __align__(128) uint8_t psmem[];
    PShared &S = *reinterpret_cast<PShared *>(psmem);
    uint8_t *win = psmem + kPWinOff;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = warp >> 2, gw = warp & 3, gt = tid & 127;
    if (tid < 4) cs_init(&S.sink[tid], S.sinkmem[tid], c_CsCap);
    __syncthreads();
    for (;;) {
        if (tid == 0) S.task = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = S.task;
        __syncthreads();
        if (t >= nrows) {
            cp_async_wait_all();
            return;
        }
        const UnitDev &U = units[rows[t].unit];
        const int row = rows[t].row, w = U.w, cw = w / 2, mbw = U.mbw;
        unsigned long long *const prog64 = reinterpret_cast<unsigned long long *>(U.progress);
        if (row == U.stall_row) continue;   // injected stall: this row's progress flag is never set
        const double lambda = U.lambda;
        const int qp = U.qp, R = U.range, navail = U.navail;
        const double lam14 = __dmul_rn(lambda, 14.0), lam16 = __dmul_rn(lambda, 16.0), lam19 = __dmul_rn(lambda, 19.0);
        qp4_setup(&S.q, qp, tid);
        const int nref = navail > 1 ? 2 : 1, wy0 = row * 16 - R - 3, wrows = 2 * R + 23;
        // With the previous frame in the same launch: the reference rows this
        // row reads are its macroblock rows up to row + ref_dr, and macroblock
        // mbx reads its columns up to mbx + ref_dc (the window strip mbx + 4
        // filled at mbx, or +-(R + 3) samples read directly when R is 64).
        const int ref_dr = WIN ? (R + 19) / 16 : R / 16 + 2, ref_dc = WIN ? 4 : R / 16 + 2;
        const int ref_row = min(row + ref_dr, U.mbh - 1);
        cp_async_wait_all();   // this block's copies for an earlier row have landed
        if (tid == 0)
            S.pok = U.ref_prog ? wait_progress(U.ref_prog + ref_row, min(ref_dc, mbw - 1) + 1, err, wait_ns) : 1;
        __syncthreads();
        if (!S.pok) continue;
        if (WIN) win_fill(win, U, nref, -3, 4, wy0, wrows, tid);   // macroblock 0's strips and macroblock 1's
        // source prefetch: each macroblock's luma and chroma are copied into
        // S.pre while the one before it is analysed (aligned planes only)
        const bool pf = ((reinterpret_cast<uintptr_t>(U.cur[0]) | (uintptr_t)w) & 15) == 0 &&
                        ((reinterpret_cast<uintptr_t>(U.cur[1]) | reinterpret_cast<uintptr_t>(U.cur[2]) |
                          (uintptr_t)cw) & 7) == 0;
        auto prefetch = [&](int pbx, int pby) {
            if (tid < 16) {
                cp_async16(&S.pre[tid * 16], U.cur[0] + (size_t)(pby + tid) * w + pbx);
            } else if (tid < 32) {
                const int k = tid - 16, pl = k >> 3, r = k & 7;
                cp_async8(&S.prec[pl][r * 8], U.cur[1 + pl] + (size_t)(pby / 2 + r) * cw + pbx / 2);
            }
            cp_async_commit();
        };
        if (pf) prefetch(0, row * 16);
        const typename LumaOf<WIN>::T L0 = luma_src<WIN>(U.ref[0], win, 0, wy0, wrows);
        const typename LumaOf<WIN>::T L1 = luma_src<WIN>(U.ref[1], win, nref - 1, wy0, wrows);
        int pmvx = 0, pmvy = 0, prev_mode = 0;
        unsigned long long pword = 0;   // thread 0: the row above's progress word seen last
        PhaseClock pc{tid == 0 ? U.prof : nullptr, 0};
        // The post stage (post.cuh): this row posts the tiles of the row above
        // (and the last row its own) in runs of kPostRun once that many are
        // final, on threads 32..511 while thread 0 waits for the row above.
        int posted = 0;
        auto post_upto = [&](int ncols, bool all) {
            while (ncols - posted >= kPostRun || (all && posted < ncols)) {
                const int n = min(kPostRun, ncols - posted);
                for (int pr = row - 1; pr <= row; ++pr) {
                    if (pr < 0 || (pr == row && row != U.mbh - 1)) continue;
                    post_run(S.post, U, pr, posted, posted + n, tid - kPostT0);
                    if (tid == kPostT0) st_release_gpu(U.post_prog + pr, posted + n);
                }
                posted += n;
            }
        };
        int mbx = 0;
        for (; mbx < mbw; ++mbx) {
            const int bx = mbx * 16, by = row * 16, cbx = bx / 2, cby = by / 2;
            pc.start();
            cp_async_wait_all();   // this thread's strip and source copies; the barrier below publishes them
            const int par = mbx & 1;
            // Past the row's first macroblock, this one's neighbour samples
            // are final before its own wait: the row above's part was covered
            // by the previous macroblock's wait (which needed one macroblock
            // further), the left part is this block's own.  Threads 256-288
            // load them now, overlapping the wait; the load phase below then
            // skips them.
            const bool early = mbx > 0;
            if (early && tid >= 256 && tid < 256 + 33) {
                const int k = tid - 256;
                if (k < 16) {
                    S.top[k] = by > 0 ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx + k]) : 0;
                    S.left[k] = ldcg8(&U.rec[0][(size_t)(by + k) * w + bx - 1]);
                } else if (k < 32) {
                    const int pl = (k - 16) >> 3, q = k & 7;
                    S.ctop[pl][q] = cby > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx + q]) : 0;
                    S.cleft[pl][q] = ldcg8(&U.rec[1 + pl][(size_t)(cby + q) * cw + cbx - 1]);
                } else {
                    S.tl = by > 0 ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx - 1]) : 128;
                    for (int pl = 0; pl < 2; ++pl)
                        S.ctl[pl] = cby > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx - 1]) : 128;
                }
            }
            // tiles up to column mbx - 2: this row has finished macroblock mbx - 1
            if (U.post_prog && tid >= kPostT0) post_upto(mbx - 1, false);
            if (tid == 0) {
                // The row above: wait until it has finished macroblock mbx + 1
                // (the above-right neighbour), then the above and above-right
                // records for the merge candidates (fdv.h:5711-5729).  Its
                // progress word carries its last published macroblock's
                // record, so when the word seen here (or at the previous
                // macroblock) describes exactly the neighbour needed, no
                // record has to be loaded.
                const float pjs = (LRN && U.prejs) ? __ldcg(&U.prejs[row * mbw + mbx]) : -1.f;
                const int need = min(mbx + 2, mbw);
                int ok = 1;
                if (U.ref_prog && mbx > 0)
                    ok = wait_progress(U.ref_prog + ref_row, min(mbx + ref_dc, mbw - 1) + 1, err, wait_ns);
                uint2 nb[2] = {make_uint2(0, 0), make_uint2(0, 0)};
                if (row > 0 && ok) {
                    const unsigned long long v = wait_count64(prog64 + row - 1, need, err, wait_ns);
                    ok = v != ~0ull;
                    if (ok) {
                        const int c = (int)(v & 0xfffu);
                        bool h0 = false, h1 = mbx + 1 >= mbw;
                        if (need == mbx + 2 && c == need) {
                            nb[1] = prog_rec(v);
                            h1 = true;
                            if ((int)(pword & 0xfffu) == mbx + 1) { nb[0] = prog_rec(pword); h0 = true; }
                        } else if (mbx == mbw - 1 && c == mbw) {
                            nb[0] = prog_rec(v);
                            h0 = true;
                        }
                        if (!h0) nb[0] = __ldcg(reinterpret_cast<const uint2 *>(&U.mbi[(row - 1) * mbw + mbx]));
                        if (!h1) nb[1] = __ldcg(reinterpret_cast<const uint2 *>(&U.mbi[(row - 1) * mbw + mbx + 1]));
                        pword = v;
                    }
                }
                S.nbi[par][0] = nb[0];
                S.nbi[par][1] = nb[1];
                S.rok[par] = ok;
                if (LRN && U.prejs) {
                    // The learned form's pre-analysed SKIPs: the zero vector is
                    // what the merge list offers iff the left vector is zero
                    // and the above / above-right macroblocks are not inter or
                    // carry the zero vector on reference 0.
                    bool zero = pmvx == 0 && pmvy == 0;
                    for (int k = 0; k < 2; ++k)
                        if (((nb[k].y >> 8) & 0xffu) && (nb[k].x != 0 || (nb[k].y & 0xffu) != 0)) zero = false;
                    S.pjs[par] = pjs;
                    S.fast[par] = ok && pjs >= 0.f && zero;
                    S.amz[par] = ((nb[0].y >> 16) & 0xffu) != 0;
                }
            }
            __syncthreads();
            if (!S.rok[par]) break;
            const bool fast = LRN && U.prejs && S.fast[par];
            if (WIN && mbx >= 1 && !fast) win_fill(win, U, nref, mbx + 4, mbx + 4, wy0, wrows, tid);
            pc.mark(PP_WAIT);
            if (U.tl && tid == 0) U.tl[2 * (row * mbw + mbx)] = globaltimer();
            uint8_t *slot = U.slots + (size_t)(row * mbw + mbx) * kSlotBytes;
            if (tid < 16) slot_len(slot)[tid] = 0;
            if (fast) {
                // SKIP with the zero vector: reconstruction written ahead,
                // the symbols and the record here (as the commit below)
                __syncwarp();
                if (tid == 0) {
                    uint8_t m0 = 0;
                    write_slot_structs(slot, (prev_mode != 0 ? 2 : 0) + S.amz[par], &m0, 1, err);
                    MBInfo mi = {0, 0, 0, 1, 0, 0};
                    U.mbi[row * mbw + mbx] = mi;
                    if (U.mbcost) U.mbcost[row * mbw + mbx] = S.pjs[par];
                    if (pc.acc) { atomicAdd(&pc.acc[PP_NMB], 1ull); atomicAdd(&pc.acc[PP_NSKIP], 1ull); }
                    st_release_gpu64(prog64 + row, prog_word(mbx + 1, mi));
                    if (U.tl) U.tl[2 * (row * mbw + mbx) + 1] = globaltimer();
                }
                pmvx = 0; pmvy = 0;
                prev_mode = 0;
                // the reference window's next strip, after the publication
                if (WIN && mbx >= 1) win_fill(win, U, nref, mbx + 4, mbx + 4, wy0, wrows, tid);
                // this macroblock's source (landed: waited at the top) is not
                // needed; the next one's goes into the same buffer
                if (pf && mbx + 1 < mbw) prefetch(bx + 16, by);
                pc.mark(PP_OUT);
                continue;
            }
            // ---- the macroblock, its current-frame neighbours, merge candidates
            if (tid < 64) {
                const int r2 = tid >> 2, c2 = (tid & 3) * 4;
                *reinterpret_cast<uint32_t *>(&S.cur[tid * 4]) =
                    pf ? *reinterpret_cast<const uint32_t *>(&S.pre[tid * 4])
                       : *reinterpret_cast<const uint32_t *>(&U.cur[0][(size_t)(by + r2) * w + bx + c2]);
            } else if (tid < 96 && pf) {
                const int k = tid - 64, pl = k >> 4;
                *reinterpret_cast<uint32_t *>(&S.curc[pl][(k & 15) * 4]) =
                    *reinterpret_cast<const uint32_t *>(&S.prec[pl][(k & 15) * 4]);
            } else if (tid < 96) {
                const int k = tid - 64, pl = k >> 4, r2 = (k & 15) >> 1, c2 = (k & 1) * 4;
                *reinterpret_cast<uint32_t *>(&S.curc[pl][(k & 15) * 4]) =
                    *reinterpret_cast<const uint32_t *>(&U.cur[1 + pl][(size_t)(cby + r2) * cw + cbx + c2]);
            } else if (tid < 112) {
                if (!early) {
                    const int k = tid - 96;
                    S.top[k] = by > 0 ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx + k]) : 0;
                    S.left[k] = bx > 0 ? ldcg8(&U.rec[0][(size_t)(by + k) * w + bx - 1]) : 0;
                }
            } else if (tid < 128) {
                if (!early) {
                    const int k = tid - 112, pl = k >> 3, q = k & 7;
                    S.ctop[pl][q] = cby > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx + q]) : 0;
                    S.cleft[pl][q] = cbx > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby + q) * cw + cbx - 1]) : 0;
                }
            } else if (tid == 128) {
                // the above and above-right macroblock records (one 8-byte load
                // each, issued together with the corner samples)
                const uint2 nb[2] = {S.nbi[par][0], S.nbi[par][1]};
                S.ht = by > 0; S.hl = bx > 0;
                if (!early) {
                    S.tl = (by > 0 && bx > 0) ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx - 1]) : 128;
                    for (int pl = 0; pl < 2; ++pl)
                        S.ctl[pl] = (cby > 0 && cbx > 0) ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx - 1]) : 128;
                }
                // merge candidates (fdv.h:5711-5729)
                int n = 1;
                S.cand[0].x = (int16_t)pmvx; S.cand[0].y = (int16_t)pmvy; S.cand[0].ref = 0; S.cand[0].inter = 1;
                for (int k = 0; k < 2 && n < 3; ++k) {
                    if (row == 0 || mbx + k >= mbw) continue;
                    MBInfo m;
                    m.x = (int16_t)(nb[k].x & 0xffffu); m.y = (int16_t)(nb[k].x >> 16);
                    m.ref = (uint8_t)(nb[k].y & 0xffu); m.inter = (uint8_t)((nb[k].y >> 8) & 0xffu);
                    if (!m.inter) continue;
                    bool dup = false;
                    for (int j2 = 0; j2 < n; ++j2)
                        if (S.cand[j2].x == m.x && S.cand[j2].y == m.y && S.cand[j2].ref == m.ref) dup = true;
                    if (!dup) S.cand[n++] = m;
                }
                S.ncand = n;
                S.amode = row > 0 ? (int)((nb[0].y >> 16) & 0xffu) : 0;
                S.lcls = -1;
                if (LRN && U.hint) {
                    const lrn::Hint hh = U.hint[row * mbw + mbx];
                    S.lcls = hh.cls;
                    for (int k = 0; k < lrn::kMvHyp; ++k) {
                        S.lmv[k] = hh.mv[k];
                        S.lmv2[k] = make_short2((short)(2 * hh.mv[k].x), (short)(2 * hh.mv[k].y));
                    }
                }
            }
            __syncthreads();
            if (pf && mbx + 1 < mbw) prefetch(bx + 16, by);   // S.pre is consumed
            // mode context (fdv.h:4172): left / above macroblock skipped-ness;
            // the left one is this block's previous macroblock
            const int ctx = (prev_mode != 0 ? 2 : 0) + (S.amode != 0 ? 1 : 0);
            const RefPlanes &R0 = U.ref[0];
            if (U.force_skip) {
                // A held frame: SKIP with the zero vector everywhere (fdv.h:5820-5836).
                if (tid < 64) {
                    const int r2 = tid >> 2, c2 = (tid & 3) * 4;
                    *reinterpret_cast<uint32_t *>(&U.rec[0][(size_t)(by + r2) * w + bx + c2]) =
                        ld4u_cg(R0.G + (long)(by + r2) * R0.ys + bx + c2);
                } else if (tid < 192) {
                    const int k = tid - 64, pl = k >> 6, p = k & 63;
                    const uint8_t *P = pl ? R0.V : R0.U;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = __ldcg(&P[(long)(cby + (p >> 3)) * R0.cs + cbx + (p & 7)]);
                }
                if (tid == 0) {
                    uint8_t m0 = 0;
                    write_slot_structs(slot, ctx, &m0, 1, err);
                    MBInfo mi = {0, 0, 0, 1, 0, 0};
                    U.mbi[row * mbw + mbx] = mi;
                    if (U.mbcost) U.mbcost[row * mbw + mbx] = 0.f;
                }
                pmvx = 0; pmvy = 0;
                prev_mode = 0;
                __syncthreads();
                if (tid == 0) {
                    const MBInfo mz = {0, 0, 0, 1, 0, 0};
                    st_release_gpu64(prog64 + row, prog_word(mbx + 1, mz));
                }
                continue;
            }
            pc.mark(PP_LOAD);
            // ---- phase 0: SKIP (fdv.h:5843-5899)
            const int ncand = S.ncand;
            if (tid < ncand * 64) {
                const int mi = tid >> 6, k = tid & 63;
                const MBInfo &c = S.cand[mi];
                const int r2 = k >> 2, c2 = (k & 3) * 4, ph = (c.y & 3) * 4 + (c.x & 3);
                reinterpret_cast<uint32_t *>(S.predS[mi])[k] =
                    mc_word_nb(c.ref ? L1 : L0, bx + c2 + (c.x >> 2), by + r2 + (c.y >> 2), ph);
            }
            __syncthreads();
            if (warp < ncand) {
                int s = 0;
                for (int q = lane; q < 256; q += 32) { int d = (int)S.cur[q] - (int)S.predS[warp][q]; s += d * d; }
                s = __reduce_add_sync(FDVB_FULL, s);
                if (lane == 0) S.ssd3[warp] = s;
            }
            __syncthreads();
            int best_mi = 0, Ds = S.ssd3[0];
            for (int mi = 1; mi < ncand; ++mi) if (S.ssd3[mi] < Ds) { Ds = S.ssd3[mi]; best_mi = mi; }
            const int midx_bits = ncand > 1 ? kBitsMode : 0;
            const double Js = rd_cost((double)Ds, lambda, kBitsMode + midx_bits);
            // A confident learned proposal narrows the analysis: SKIP takes the
            // best merge candidate; inter searches only the nearest reference's
            // 16x16 vector, from the proposed vectors (a few diamond steps and
            // the sub-pel refinement), without the INTER8 chain and intra;
            // intra skips the motion searches.  Without a confident class the
            // full analysis runs, its nearest-reference 16x16 search seeded
            // with the proposed vectors as well.
            // (a SKIP the gate turns down was predicted wrongly: full analysis)
            const int lcls0 = LRN ? S.lcls : -1;
            const bool gate_ok = !LRN || U.skip_gate <= 0.0 || Js <= __dmul_rn(U.skip_gate, lambda);
            const int lcls = (lcls0 == 0 && !gate_ok) ? -1 : lcls0;
            const bool lfast = lcls >= 0, l_intra = lcls == 2;
            const bool l8 = !lfast || (LRN && lcls == 1 && U.inter8);   // INTER8 analysed
            const bool skip_wins = Js <= lam14 || (LRN && lcls == 0);
            double Jc = Js;   // RD cost of the chosen mode
            pc.mark(PP_SKIP);
            if (pc.acc) { atomicAdd(&pc.acc[PP_NMB], 1ull); if (skip_wins) atomicAdd(&pc.acc[PP_NSKIP], 1ull); }

            int chosen = 0, best_ref = 0, mvx = 0, mvy = 0, best_sub = 0;
            if (!skip_wins) {
                // ---- phase 1: searches on four warp groups
                const long long tg0 = (U.prof && gt == 0) ? clock64() : 0;
                if (tid < 4) cs_reset(&S.sink[tid]);
                if (grp < 2) {
                    // the 16x16 search on reference grp (one call site for both
                    // references keeps one copy of its code); with proposals
                    // it also starts from them (doubled for the second
                    // reference); a full search (not confident) still runs the
                    // diamond to the end
                    if (grp == 0 ? !l_intra : (navail > 1 && !lfast)) {
                        int mx, my;
                        const bool hinted = LRN && U.hint;
                        const typename LumaOf<WIN>::T &Lg = grp ? L1 : L0;
                        int sd = me_search_group<16>(S.cur, Lg, bx, by, R, pmvx, pmvy, &mx, &my, S.gsad[grp], gw, lane,
                                                     9 + grp, (grp == 0 && U.prof) ? &U.prof[PP_IT16] : nullptr,
                                                     hinted ? (grp ? S.lmv2 : S.lmv) : nullptr, hinted ? lrn::kMvHyp : 0,
                                                     lfast ? kLearnLd : 64);
                        if (gt == 0) { S.mv[grp][0] = mx; S.mv[grp][1] = my; S.sad[grp] = sd; }
                        mc16_group(Lg, bx, by, mx, my, S.pr[grp], gt);
                    }
                } else if (grp == 2) {
                    if (l8) {
                        int qpx = pmvx, qpy = pmvy, ssad = 0;
                        for (int q = 0; q < 4; ++q) {
                            const int qx = (q & 1) * 8, qy = (q >> 1) * 8;
                            int mx, my;
                            ssad += me_search_group<8>(S.cur + qy * 16 + qx, L0, bx + qx, by + qy, R, qpx, qpy, &mx, &my,
                                                       S.gsad[2], gw, lane, 11, U.prof ? &U.prof[PP_IT8] : nullptr,
                                                       (LRN && U.hint) ? S.lmv : nullptr,
                                                       (LRN && U.hint) ? lrn::kMvHyp : 0, lfast ? kLearnLd : 64);
                            if (gt == 0) { S.qmv[q][0] = mx; S.qmv[q][1] = my; }
                            qpx = mx; qpy = my;
                            if (gt < 16) {
                                const int r2 = gt >> 1, c2 = (gt & 1) * 4, ph = (my & 3) * 4 + (mx & 3);
                                reinterpret_cast<uint32_t *>(S.pred8[q])[gt] =
                                    mc_word_nb(L0, bx + qx + c2 + (mx >> 2), by + qy + r2 + (my >> 2), ph);
                            }
                        }
                        if (gt == 0) S.ssad = ssad;
                    }
                } else {
                    if (lfast && !l_intra) {
                        if (gt == 0) S.isel = -1;
                    } else {
                        // intra 16x16 sub-modes, SATD-screened (fdv.h:5961-5970)
                        if (gt < 4) S.nn[gt] = nn_setup(gt, S.top, S.left, S.tl, 16, S.ht, S.hl);
                        gbar(12, 128);
                        if (gt < 64) {
                            const int m = gt >> 4, b = gt & 15, oy = (b >> 2) * 4, ox = (b & 3) * 4;
                            uint8_t pk[16];
                            for (int p = 0; p < 16; ++p) pk[p] = (uint8_t)nn_px(S.nn[m], S.top, S.left, ox + (p & 3), oy + (p >> 2));
                            S.satd[gt] = satd4(S.cur + oy * 16 + ox, 16, pk, 4);
                        }
                        gbar(12, 128);
                        int sel = -1, sbest = 0;
                        for (int m = 0; m < 4; ++m) {
                            if (!nn_mode_ok(m, 16, S.ht, S.hl)) continue;
                            int sa = 0;
                            for (int b = 0; b < 16; ++b) sa += S.satd[m * 16 + b];
                            if (sel < 0 || sa < sbest) { sbest = sa; sel = m; }
                        }
                        if (gt == 0) S.isel = sel;
                        if (sel >= 0)
                            for (int p = gt; p < 256; p += 128) S.pr[2][p] = (uint8_t)nn_px(S.nn[sel], S.top, S.left, p & 15, p >> 4);
                    }
                }
                if (grp != 2) {
                    // the pool: residuals of candidates 0 (INTER16 nearest), 1
                    // (INTER16 second, with two references) and 2 (INTRA16, when
                    // a sub-mode is allowed), three warp tasks per region
                    team_bar(BAR_POOL, 384);
                    const int pw = warp < 8 ? warp : warp - 4;      // 0..11
                    const unsigned pmask = (l_intra ? 0u : 0xFu) | (navail > 1 && !lfast ? 0xF0u : 0u) |
                                           (S.isel >= 0 ? 0xF00u : 0u);
                    // every warp takes two 4x4 pair tasks and one 8x8 task
                    // (regions pw, pw + 4, pw + 8 mod 12): the warps finish
                    // together instead of a third of them doing the three
                    // shorter 8x8 tasks
#pragma unroll 1
                    for (int j = 0; j < 3; ++j) {
                        const int g = (pw + 4 * j) % 12;
                        if ((pmask >> g) & 1u) resid_task(S, g, j, qp, lambda, warp, lane);
                    }
                    team_bar(BAR_POOL, 384);
                    const int c = grp == 3 ? 2 : grp;
                    if ((pmask >> (4 * c)) & 1u) group_decide(S, c, lambda, gw, gt, lane, 9 + grp, err);
                }
                if (U.prof && gt == 0) atomicAdd(&U.prof[PP_G0 + grp], (unsigned long long)(clock64() - tg0));
                __syncthreads();
                pc.mark(PP_SEARCH);
                // ---- phase 3, first part: the reference's decision on the
                // INTER16 and INTRA16 results, which decides whether INTER8
                // is evaluated at all
                const int isel = S.isel, ssad = S.ssad;
                const bool haveI = isel >= 0;
                auto gate_skip = [&](int s16) { return s16 > 0 && ssad * 10 >= s16 * 9; };
                double Jbest = Js, Ji = 1e30, Jintra = 1e30, J8 = 1e30;
                int sad16 = 0;
                const int nsearch = l_intra ? 0 : (lfast ? 1 : navail);
                for (int r = 0; r < nsearch; ++r) {
                    if (r > 0 && Jbest <= lam16) break;
                    const int rmx = S.mv[r][0], rmy = S.mv[r][1];
                    const int bb = 2 * kBitsMode + bits_val(zz_enc(rmx - pmvx)) + bits_val(zz_enc(rmy - pmvy)) + S.cB[r];
                    const double J = rd_cost((double)S.cD[r], lambda, bb);
                    if (J < Jbest) Jbest = J;
                    if (J < Ji) { Ji = J; best_ref = r; mvx = rmx; mvy = rmy; sad16 = S.sad[r]; }
                }
                if (Jbest > lam14 && haveI) {
                    Jintra = rd_cost((double)S.cD[2], lambda, 2 * kBitsMode + S.cB[2]);
                    best_sub = isel;
                    if (Jintra < Jbest) Jbest = Jintra;
                }
                // ---- phase 2: the INTER8 residual, on every warp, only where
                // the reference evaluates INTER8 (the same condition as below;
                // every thread holds the same values)
                const bool need8 = l8 && Jbest > lam19 && !gate_skip(sad16);
                if (need8) {
                    if (warp < 12) resid_task(S, 12 + warp / 3, warp % 3, qp, lambda, warp, lane);
                    __syncthreads();
                    pc.mark(PP_RESID);
                    if (grp == 2) group_decide(S, 3, lambda, gw, gt, lane, 11, err);
                    __syncthreads();
                }
                pc.mark(PP_DECIDE);
                // ---- phase 3, second part: INTER8 and the final choice
                if (need8) {
                    int b8 = kBitsMode, px = pmvx, py = pmvy;
                    for (int q = 0; q < 4; ++q) {
                        b8 += bits_val(zz_enc(S.qmv[q][0] - px)) + bits_val(zz_enc(S.qmv[q][1] - py));
                        px = S.qmv[q][0]; py = S.qmv[q][1];
                    }
                    J8 = rd_cost((double)S.cD[3], lambda, b8 + S.cB[3]);
                }
                double Jmin = Js;
                if (Ji < Jmin) { Jmin = Ji; chosen = 1; }
                if (Jintra < Jmin) { Jmin = Jintra; chosen = 2; }
                if (J8 < Jmin) { Jmin = J8; chosen = 3; }
                Jc = Jmin;
            }

            // ---- commit (fdv.h:6049-6160)
            CoefSink *M = chosen == 1 ? &S.sink[best_ref] : &S.sink[chosen == 2 ? 2 : 3];
            MBInfo info = {0, 0, 0, 0, (uint8_t)chosen, 0};
            if (chosen == 0) {
                const int smvx = S.cand[best_mi].x, smvy = S.cand[best_mi].y, sref = S.cand[best_mi].ref;
                if (tid == 0) {
                    uint8_t m0 = 0, mi = (uint8_t)best_mi;
                    write_slot_structs(slot, ctx, &m0, 1, err);
                    if (ncand > 1) write_slot_structs(slot, PS_MERGE, &mi, 1, err);
                }
                if (tid < 64)
                    *reinterpret_cast<uint32_t *>(&U.rec[0][(size_t)(by + (tid >> 2)) * w + bx + (tid & 3) * 4]) =
                        reinterpret_cast<const uint32_t *>(S.predS[best_mi])[tid];
                else if (tid < 192) {
                    const int k = tid - 64, pl = k >> 6, p = k & 63;
                    const RefPlanes &Rs = U.ref[sref];
                    const int cmx = smvx / 2, cmy = smvy / 2;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] =
                        (uint8_t)mc_cpx_cg(pl ? Rs.V : Rs.U, Rs.cs, cbx + (p & 7) + (cmx >> 2), cby + (p >> 3) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                info.x = (int16_t)smvx; info.y = (int16_t)smvy; info.ref = (uint8_t)sref; info.inter = 1;
                pmvx = smvx; pmvy = smvy;
            } else if (chosen == 1) {
                if (tid == 0) {
                    uint8_t b[12];
                    int n = 0;
                    b[n++] = (uint8_t)best_ref;
                    n += leb_write(b + n, zz_enc(mvx - pmvx));
                    n += leb_write(b + n, zz_enc(mvy - pmvy));
                    uint8_t m1 = 1;
                    write_slot_structs(slot, ctx, &m1, 1, err);
                    write_slot_structs(slot, PS_REF, b, 1, err);
                    int part = 0;
                    for (int q = 1; q < n; ++q) {
                        write_slot_structs(slot, part ? PS_MVY : PS_MVX, b + q, 1, err);
                        if (!(b[q] & 0x80)) ++part;
                    }
                }
                {
                    const int rr = ((tid >> 4) >> 3) * 2 + ((tid & 15) >> 3), q = ((tid >> 4) & 7) * 8 + (tid & 7);
                    if (tid < 256) {
                        const int g = 4 * best_ref + rr;
                        U.rec[0][(size_t)(by + (tid >> 4)) * w + bx + (tid & 15)] =
                            S.dec[g].choice ? S.reg[g].rec[q] : S.recA[g][q];
                    }
                }
                // chroma INTER: prediction at mv/2, four 4x4 blocks per plane, no RDOQ (fdv.h:5576-5626)
                const RefPlanes &Rb = U.ref[best_ref];
                const int cmx = mvx / 2, cmy = mvy / 2;
                if (tid < 128) {
                    const int pl = tid >> 6, p = tid & 63;
                    S.cpred[pl][p] = (uint8_t)mc_cpx_cg(pl ? Rb.V : Rb.U, Rb.cs, cbx + (p & 7) + (cmx >> 2), cby + (p >> 3) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                __syncthreads();
                if (warp < 8) {
                    const int pl = warp >> 2, b = warp & 3, oy = (b >> 1) * 4, ox = (b & 1) * 4;
                    warp_block4(S.curc[pl] + oy * 8 + ox, 8, S.cpred[pl] + oy * 8 + ox, 8, S.crec[pl] + oy * 8 + ox, 8,
                                S.q, lambda, false, &S.cblk[warp], &S.b4[warp], lane);
                }
                __syncthreads();
                if (tid == 0) {
                    for (int pl = 0; pl < 2; ++pl) {
                        bool any = false;
                        for (int b = 0; b < 4; ++b) if (S.cblk[pl * 4 + b].count > 0) any = true;
                        cs_put1(M, CS_FL, any ? 1 : 0, err);
                        if (any)
                            for (int b = 0; b < 4; ++b) {
                                cs_put1(M, CS_NC, (uint8_t)S.cblk[pl * 4 + b].count, err);
                                cs_put(M, CS_LC, S.cblk[pl * 4 + b].bytes, S.cblk[pl * 4 + b].nbytes, err);
                            }
                    }
                }
                if (tid < 128) {
                    const int pl = tid >> 6, p = tid & 63;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = S.crec[pl][p];
                }
                info.x = (int16_t)mvx; info.y = (int16_t)mvy; info.ref = (uint8_t)best_ref; info.inter = 1;
                pmvx = mvx; pmvy = mvy;
            } else if (chosen == 2) {
                if (tid == 0) {
                    uint8_t m2 = 2, sb = (uint8_t)best_sub;
                    write_slot_structs(slot, ctx, &m2, 1, err);
                    write_slot_structs(slot, PS_SUB, &sb, 1, err);
                }
                if (tid < 256) {
                    const int rr = ((tid >> 4) >> 3) * 2 + ((tid & 15) >> 3), q = ((tid >> 4) & 7) * 8 + (tid & 7);
                    const int g = 8 + rr;
                    U.rec[0][(size_t)(by + (tid >> 4)) * w + bx + (tid & 15)] = S.dec[g].choice ? S.reg[g].rec[q] : S.recA[g][q];
                }
                // chroma intra with the same sub-mode through the residual coder, U then V (fdv.h:6104-6117)
                if (tid < 2) S.nn[tid] = nn_setup(best_sub, S.ctop[tid], S.cleft[tid], S.ctl[tid], 8, cby > 0, cbx > 0);
                __syncthreads();
                if (tid < 128) {
                    const int pl = tid >> 6, p = tid & 63;
                    S.cpred[pl][p] = (uint8_t)nn_px(S.nn[pl], S.ctop[pl], S.cleft[pl], p & 7, p >> 3);
                }
                __syncthreads();
                if (warp < 8) {
                    const int pl = warp >> 2, s = warp & 3, sx = (s & 1) * 4, sy = (s >> 1) * 4;
                    warp_block4(S.curc[pl] + sy * 8 + sx, 8, S.cpred[pl] + sy * 8 + sx, 8, &S.recA[pl][sy * 8 + sx], 8,
                                S.q, lambda, true, &S.blk[warp], &S.b4[warp], lane);
                } else if (tid >= 256 && tid < 384) {
                    const int pl = (tid - 256) >> 6;
                    region8(S.curc[pl], 8, S.cpred[pl], 8, qp, &S.creg[pl], &S.r8[pl], tid & 63, 1 + pl);
                }
                __syncthreads();
                for (int pl = 0; pl < 2; ++pl)
                    decide_regions<PNT>(1, &S.blk[4 * pl], &S.creg[pl], &S.cdec[pl], lambda, true, M, &S.ce, &S.cb, err);
                if (tid < 128) {
                    const int pl = tid >> 6, q = tid & 63;
                    U.rec[1 + pl][(size_t)(cby + (q >> 3)) * cw + cbx + (q & 7)] = S.cdec[pl].choice ? S.creg[pl].rec[q] : S.recA[pl][q];
                }
                info.inter = 0;
            } else {
                if (tid == 0) {
                    uint8_t b[20];
                    int n = 0, px = pmvx, py = pmvy;
                    for (int q = 0; q < 4; ++q) {
                        n += leb_write(b + n, zz_enc(S.qmv[q][0] - px));
                        n += leb_write(b + n, zz_enc(S.qmv[q][1] - py));
                        px = S.qmv[q][0]; py = S.qmv[q][1];
                    }
                    uint8_t m3 = 3;
                    write_slot_structs(slot, ctx, &m3, 1, err);
                    int part = 0;
                    for (int q = 0; q < n; ++q) {
                        write_slot_structs(slot, (part & 1) ? PS_MVY : PS_MVX, b + q, 1, err);
                        if (!(b[q] & 0x80)) ++part;
                    }
                }
                if (tid < 256) {
                    const int q = tid >> 6, p = tid & 63, qx = (q & 1) * 8, qy = (q >> 1) * 8, g = 12 + q;
                    U.rec[0][(size_t)(by + qy + (p >> 3)) * w + bx + qx + (p & 7)] = S.dec[g].choice ? S.reg[g].rec[p] : S.recA[g][p];
                }
                // chroma: 4x4 per quadrant at qmv/2 from the nearest reference, RDOQ'd (fdv.h:6143-6159)
                if (tid < 128) {
                    const int k = tid >> 4, p = tid & 15, pl = k >> 2, q = k & 3;
                    const int cmx = S.qmv[q][0] / 2, cmy = S.qmv[q][1] / 2, qcx = (q & 1) * 4, qcy = (q >> 1) * 4;
                    S.cpred4[k][p] = (uint8_t)mc_cpx_cg(pl ? R0.V : R0.U, R0.cs, cbx + qcx + (p & 3) + (cmx >> 2),
                                                     cby + qcy + (p >> 2) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                __syncthreads();
                if (warp < 8) {
                    const int pl = warp >> 2, q = warp & 3, qcx = (q & 1) * 4, qcy = (q >> 1) * 4;
                    warp_block4(S.curc[pl] + qcy * 8 + qcx, 8, S.cpred4[warp], 4, S.crec[pl] + qcy * 8 + qcx, 8,
                                S.q, lambda, true, &S.cblk[warp], &S.b4[warp], lane);
                }
                __syncthreads();
                if (tid == 0) {
                    for (int k = 0; k < 8; ++k) {
                        cs_put1(M, CS_NC, (uint8_t)S.cblk[k].count, err);
                        cs_put(M, CS_LC, S.cblk[k].bytes, S.cblk[k].nbytes, err);
                    }
                }
                if (tid < 128) {
                    const int pl = tid >> 6, p = tid & 63;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = S.crec[pl][p];
                }
                info.x = (int16_t)S.qmv[3][0]; info.y = (int16_t)S.qmv[3][1]; info.ref = 0; info.inter = 1;
                pmvx = S.qmv[3][0]; pmvy = S.qmv[3][1];
            }
            __syncthreads();
            pc.mark(PP_COMMIT);
            prev_mode = chosen;
            if (tid == 0) {
                U.mbi[row * mbw + mbx] = info;
                if (U.mbcost) U.mbcost[row * mbw + mbx] = (float)Jc;
                // Publish now: the row below reads the reconstruction (ordered
                // before this release by the barrier above) and the record
                // (also carried in the word), never the symbol slot.
                st_release_gpu64(prog64 + row, prog_word(mbx + 1, info));
                if (U.tl) U.tl[2 * (row * mbw + mbx) + 1] = globaltimer();
            }
            // ---- coefficient streams of the chosen mode into the slot (read
            // after the kernel; the sinks are reset only after the next
            // macroblock's first barrier)
            // (warp k copies stream k: no stream waits for the one before)
            if (chosen != 0 && (tid >> 5) < CS_NUM) {
                const int k = tid >> 5, ln = tid & 31;
                int n = M->len[k];
                if (n > c_SlotCap[PS_CN + k]) { if (ln == 0) atomicOr(err, kErrSlotOverflow); n = 0; }
                uint8_t *d = slot_data(slot, PS_CN + k);
                const uint8_t *s = M->buf[k];
                for (int i = ln; i < n; i += 32) d[i] = s[i];
                if (ln == 0) slot_len(slot)[PS_CN + k] = (uint16_t)n;
            }
            pc.mark(PP_OUT);
        }
        // the row's last tiles (its last macroblock is finished)
        if (U.post_prog && mbx == mbw && tid >= kPostT0) post_upto(mbw, true);
        __syncthreads();
        if (FS) {
            // the frame's rows done: the block that finishes the last one
            // compacts the frame (every row's slots were published by the
            // fence before its count) and tells the host
            const int j = rows[t].unit, fk = j / nu;
            __threadfence();
            __syncthreads();
            if (tid == 0) {
                S.lastrow = atomicAdd(&fdone[j], 1) + 1 == U.mbh;
                __threadfence();
            }
            __syncthreads();
            if (S.lastrow) {
                compact_block<PNT>(ctasks[j], err, S.cmp, tid);
                __threadfence_system();
                __syncthreads();
                if (tid == 0 && atomicAdd(&fdone[nunits + fk], 1) + 1 == nu) {
                    __threadfence_system();
                    *(volatile unsigned *)fsync[fk].ready = fsync[fk].ready_val;
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace fdvb

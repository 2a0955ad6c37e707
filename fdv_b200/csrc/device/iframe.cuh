// Key-frame analysis: the intra quadtree of the image codec as a persistent
// wavefront kernel over coding tree units, run by clusters of three blocks.
//
// Work unit: one 64x64 CTU row of one plane of one encoder unit; clusters take
// rows from an atomic ticket in plane order.  The reference's wavefront
// (intra_ctu_row, fdv.h:4698-4725) starts CTU (c, r) once row r-1 has
// finished CTU c+1, whose bottom-left samples the CTU's top-right 4x4 leaf
// may read (above-right).  On planes of more than two CTU rows, CTU (c, r)
// here starts once CTU (c, r-1) is done and waits for CTU (c+1, r-1) only at
// its top-right quadrant, a quarter of the way through its quadtree walk,
// reloading those four samples: rows follow each other about 1.75 CTUs apart
// instead of 2 (one 1280x720 plane: 32.4 -> 30.5 ms), and every sample is
// read final, as in the reference's order.  Every wait is bounded.
//
// The quadtree (intra_node, fdv.h:4494-4582) tries, at every node inside the
// plane, the split (four children, recursively) and the leaf, and keeps the
// leaf only if it is not more expensive.  A node's leaf trial reads nothing
// but the samples above and left of the node, which are final when the node
// starts, so it runs concurrently with the node's split trial:
//   * block 0, warps 0-3 ("the chain"): the walk in the reference's order, the
//     4x4 leaves (intra_leaf4, fdv.h:3907-4111), the split/leaf decisions and
//     the CTU's symbols; it holds the CTU's reconstruction and mode map;
//   * block 0, warps 4-11: the 8x8 leaf trials; block 1 (all 16 warps): the
//     16x16 leaf trials; block 2: the 32x32 and the 64x64 leaf trials
//     (intra_leafn, fdv.h:4442-4484), every allowed mode at once.  A CTU
//     has one 64x64 node and four 32x32 ones, whose trials keep a block busy
//     a fifth of the time or less, so they share one: each size has its own
//     job slot and result area, and the block codes whichever job is posted
//     (a 32x32 one first).  Three blocks per cluster let more CTU rows run at
//     once (the two key frames of a lookahead launch: 49 rows instead of 37).
// When the chain enters a node it posts the node's neighbours to the team of
// that size through distributed shared memory; the team codes the leaf and
// posts back its cost; the chain reads the winner's reconstruction and symbols
// from the team's shared memory only if the leaf wins.  Every wait is bounded.
#include <cooperative_groups.h>
#include "common.cuh"
#include "intra.cuh"
#include "pred4_table.h"
#include "residual.cuh"

namespace fdvb {

namespace cg = cooperative_groups;

__device__ const P4Tab g_p4tab = make_p4tab();

constexpr int INT = 512;              // threads per block
constexpr int ICL = 3;                // blocks per cluster
constexpr int kTileW = 129;           // tile columns: x in [-1, 127] relative to the CTU
constexpr int kChainNT = 128;         // chain threads (block 0, warps 0-3)
// 8x8 leaf team (block 0, warps 4-11).  Warps 12-15 of block 0 stay idle:
// the chain shares its SM with the team, and fewer team warps leave it more
// issue slots (the team still finishes a job before the chain needs it).
constexpr int kH8NT = 256;
enum { BAR_CHAIN = 1, BAR_H8 = 2, BAR_TEAM = 3 };

// Stream ids of the intra path (fdv.h:4273-4289).
enum { IS_SPLIT0 = 0, IS_MODEB = 4, IS_MODE0 = 5, IS_MODE1 = 6, IS_NS = 7 };

// Symbols of one node's trial: seven structure streams plus coefficients.
struct ISink {
    int slen[IS_NS], scap[IS_NS];
    uint8_t *sbuf[IS_NS];
    CoefSink c;
};

// Output slot of one CTU: uint16 len[12] at offset 0, stream k at 32 + off(k).
constexpr int kIStreamCap[12] = {1, 4, 16, 64, 85, 256, 256, 256, 8192, 64, 8192, 64};
__constant__ int c_IStreamCap[12] = {1, 4, 16, 64, 85, 256, 256, 256, 8192, 64, 8192, 64};
__constant__ int c_IStreamOff[12] = {0, 1, 5, 21, 85, 170, 426, 682, 938, 9130, 9194, 17386};
constexpr int islot_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += kIStreamCap[i]; return o; }
constexpr int kISlotBytes = ((32 + islot_off(12) + 127) / 128) * 128;

struct IPlaneDev {
    const uint8_t *src;     // plane source, tight (stride w)
    uint8_t *rec;           // plane reconstruction, tight
    uint8_t *mmap;          // 4x4-cell mode map, (w/4) x (h/4)
    int *progress;          // per CTU row
    uint8_t *slots;         // per CTU output slot
    int w, h, cols, rows, qp;
    double lambda;
    unsigned long long *prof;   // optional cycle profile (NULL: off)
};
// Profile entries of the key-frame kernel (relative to prof): chain waits for
// the row above, chain 4x4 leaves, team busy time per leaf size, CTU time,
// CTU count, 4x4 leaf count, chain waits for team results.
enum { IP_WAIT = 0, IP_LEAF4, IP_LEAF8, IP_LEAF16, IP_LEAF32, IP_LEAF64, IP_CTU, IP_NCTU, IP_NLEAF4, IP_HWAIT,
       IP_L4SCREEN, IP_L4SELECT, IP_L4TRIAL, IP_L4COMMIT, IP_L4RUN1, IP_L4RUN2 };
struct ITask { int plane, row; };

// Per-depth split-trial sink capacities (node of side n = 64 >> d, see
// nd_struct/nd_cnt/nd_lvl fdv.h:4312-4314).
__host__ __device__ constexpr int isink_scap(int d, int k) {
    return k < 4 ? (k >= d ? (1 << (2 * (k - d))) : 0)
                 : (k == 4 ? (d <= 0 ? 85 : (d == 1 ? 21 : (d == 2 ? 5 : 1))) : ((64 >> d) / 4) * ((64 >> d) / 4));
}
__host__ __device__ constexpr int isink_ccap(int d, int k) {
    return k == CS_N ? ((64 >> d) / 4) * ((64 >> d) / 4)
         : (k == CS_L || k == CS_L8) ? (64 >> d) * (64 >> d) * 2
         : (k == CS_N8 || k == CS_FL) ? ((64 >> d) / 8) * ((64 >> d) / 8) : 0;
}
__host__ __device__ constexpr int isink_bytes(int d) {
    int t = 0;
    for (int k = 0; k < IS_NS; ++k) t += isink_scap(d, k);
    for (int k = 0; k < CS_NUM; ++k) t += isink_ccap(d, k);
    return t;
}
// A team's per-mode coefficient sink: the capacities of a 64x64 leaf, stream
// k at a fixed offset so that the chain can address it in another block.
__host__ __device__ constexpr int leaf_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += isink_ccap(0, i); return o; }
constexpr int kLeafSinkBytes = leaf_off(CS_NUM);
// The same for a 32x32 leaf (the merged block's second result area).
__host__ __device__ constexpr int leaf32_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += isink_ccap(1, i); return o; }
constexpr int kLeaf32SinkBytes = leaf32_off(CS_NUM);

// A leaf-trial job (written by the chain) and its result (read by the chain).
struct HJob {
    int seq;                 // job sequence number, release-stored last
    int kind;                // 0: code the node's leaf; 1: end of the CTU row
    int bx, by, ht, hl, tl;
    uint8_t top[64], left[64];
};
struct HelperArea {
    HJob job;
    HJob job64;              // block 2: the 64x64 node's job (job: the 32x32 ones)
    int ok, sel, nm, ml[4];
    NNPred nn[4];
    long long e[4];
    int b[4];
    CoefSink sink[4];
    __align__(16) uint8_t src[64 * 64];
    __align__(16) uint8_t pred[4][64 * 64];
    __align__(16) uint8_t rec[4][64 * 64];
    __align__(16) uint8_t sinkmem[4][kLeafSinkBytes];
    TeamResidScratch<INT / 32> ts;
    // block 2: the 32x32 trials' results (the 64x64 trial's go to rec / sink
    // above), so that neither job overwrites a result the chain has not read
    CoefSink sink32[4];
    __align__(16) uint8_t rec32[4][32 * 32];
    __align__(16) uint8_t sinkmem32[4][kLeaf32SinkBytes];
};
struct ChainArea {
    uint8_t tile[65 * kTileW];            // reconstruction: rows -1..63, cols -1..127
    __align__(16) uint8_t src[64 * 64];
    uint8_t mm[17 * 17];                  // mode map: cells -1..15 x -1..15
    ISink ss[4];                          // split trial sinks per depth
    uint8_t ssmem[isink_bytes(0) + isink_bytes(1) + isink_bytes(2) + isink_bytes(3)];
    ISink out;                            // the CTU's output (global)
    // 4x4 leaf scratch
    int T9w[4][9], L5w[4][5];             // per warp: T(-1..7), L(-1..3)
    uint8_t cp[9][16];
    int csat[9], cs[9], cm[9], run, best_c;
    Blk4 trial[9];
    Blk4 fin[2];
    uint8_t frec[2][16], junk[4][16];
    Blk4Scratch b4[4];
    double retJ;
    int done[4];                          // per leaf size: last finished job (written by the teams)
    int issued[4];                        // per leaf size: last posted job
    double res_J[4];                      // per leaf size: the team's result (written by the team)
    int res_idx[4], res_mode[4];
    int abort, task, row_ok;
    uint16_t p4[9 * 16];                  // the 4x4 prediction table (pred4_table.h)
    int N4[3][14];                        // per screening warp: the neighbour vector
};
struct IShared {
    QP4 q;
    ChainArea C;
    HelperArea H;
};

struct CCtx {
    IShared *S;
    const IPlaneDev *P;
    int bx0, by0, w, h, qp;
    double lambda;
    unsigned *err;
    unsigned long long *prof;
    unsigned long long hlimit;
    unsigned long long wait_ns;   // limit of the waits for the CTU row above
    bool early;                   // CTUs start once the CTU above is done (planes of more than two CTU rows)
};

// --------------------------------------------------- cluster plumbing --
__device__ __forceinline__ void fence_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
__device__ __forceinline__ void st_release_cluster(int *p, int v) {
    asm volatile("st.release.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire_cluster(const int *p) {
    int v;
    asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Bounded wait (one thread) until *p >= need; false on timeout (reported) or
// when another block has already raised an error.
__device__ bool wait_cluster_flag(const int *p, int need, unsigned *err, unsigned long long limit_ns) {
    if (ld_acquire_cluster(p) >= need) return true;
    const unsigned long long t0 = globaltimer();
    for (;;) {
        if (ld_acquire_cluster(p) >= need) return true;
        if (*(volatile unsigned *)err) return false;
        if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrWaitTimeout); return false; }
        __nanosleep(32);
    }
}
// The leaf trials of nodes of side 64 >> L run in cluster block 3 - L, the
// 64x64 ones (L = 0) in block 2 beside the 32x32 ones.
__device__ __forceinline__ int level_rank(int L) { return L == 0 ? 2 : 3 - L; }
// The job slot of level L in its block's helper area (a local address).
__device__ __forceinline__ HJob *job_slot(HelperArea *H, int L) { return L == 0 ? &H->job64 : &H->job; }

__device__ __forceinline__ void cbar() { team_bar(BAR_CHAIN, kChainNT); }
__device__ __forceinline__ uint8_t &TL(ChainArea &C, int ty, int tx) { return C.tile[(ty + 1) * kTileW + tx + 1]; }
__device__ __forceinline__ uint8_t &MM(ChainArea &C, int cy, int cx) { return C.mm[(cy + 1) * 17 + cx + 1]; }
__device__ __forceinline__ long long prof_t0(const unsigned long long *prof, int t) { return (prof && t == 0) ? clock64() : 0; }
__device__ __forceinline__ void prof_add(unsigned long long *prof, int t, int k, long long t0) {
    if (prof && t == 0) atomicAdd(&prof[k], (unsigned long long)(clock64() - t0));
}

// ------------------------------------------------------------- sinks --
__device__ void isink_reset(ISink *s) {
    for (int k = 0; k < IS_NS; ++k) s->slen[k] = 0;
    cs_reset(&s->c);
}
__device__ void isink_put(ISink *s, int k, uint8_t v, unsigned *err) {
    if (s->slen[k] + 1 > s->scap[k]) { atomicOr(err, kErrSlotOverflow); return; }
    s->sbuf[k][s->slen[k]++] = v;
}
// Copy n bytes from src to dst by the 32 lanes of a warp, four loads in
// flight per lane.
__device__ __forceinline__ void warp_copy_bytes(uint8_t *dst, const uint8_t *src, int n, int lane) {
    int i = lane;
    for (; i + 96 < n; i += 128) {
        const uint8_t a = src[i], b = src[i + 32], c = src[i + 64], d = src[i + 96];
        dst[i] = a; dst[i + 32] = b; dst[i + 64] = c; dst[i + 96] = d;
    }
    for (; i < n; i += 32) dst[i] = src[i];
}
// dst += src, by the chain: lane s of every warp holds stream s's lengths
// (the seven structure streams, then the coefficient streams), warp w copies
// the w-th, (w + 4)-th, ... non-empty stream, and thread s updates stream s's
// length after a barrier.  A stream that would overflow is left out and
// reported.
constexpr int kChainNS = IS_NS + CS_NUM;
static_assert(kChainNS <= 32, "one lane per stream");
__device__ void chain_isink_append(ISink *dst, const ISink *src, unsigned *err) {
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    int n = 0, b = 0, cap = 0;
    if (lane < IS_NS) { n = src->slen[lane]; b = dst->slen[lane]; cap = dst->scap[lane]; }
    else if (lane < kChainNS) { n = src->c.len[lane - IS_NS]; b = dst->c.len[lane - IS_NS]; cap = dst->c.cap[lane - IS_NS]; }
    const bool fits = b + n <= cap;
    if (w == 0 && n > 0 && !fits) atomicOr(err, kErrSlotOverflow);
    unsigned todo = __ballot_sync(FDVB_FULL, n > 0 && fits);
    for (int r = 0; todo; ++r) {
        const int st = __ffs(todo) - 1;
        todo &= todo - 1;
        if ((r & 3) != w) continue;
        const int ns = __shfl_sync(FDVB_FULL, n, st), bs = __shfl_sync(FDVB_FULL, b, st);
        const uint8_t *sp = st < IS_NS ? src->sbuf[st] : src->c.buf[st - IS_NS];
        uint8_t *dp = (st < IS_NS ? dst->sbuf[st] : dst->c.buf[st - IS_NS]) + bs;
        warp_copy_bytes(dp, sp, ns, lane);
    }
    cbar();
    if (t < kChainNS && n > 0 && fits) {
        if (t < IS_NS) dst->slen[t] = b + n;
        else dst->c.len[t - IS_NS] = b + n;
    }
    cbar();
}
// dst += the level-L team's sink `idx` (in cluster block `rank`), by the
// chain, the same way (one lane per coefficient stream).
__device__ void chain_append_leaf(CoefSink *dst, IShared *S, int L, int rank, int idx, unsigned *err) {
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    cg::cluster_group cl = cg::this_cluster();
    const bool s32 = L == 1;
    const CoefSink *ls = s32 ? &S->H.sink32[idx] : &S->H.sink[idx];
    const uint8_t *lm = s32 ? &S->H.sinkmem32[idx][0] : &S->H.sinkmem[idx][0];
    const CoefSink *rs = rank ? cl.map_shared_rank(ls, rank) : ls;
    const uint8_t *rm = rank ? cl.map_shared_rank(lm, rank) : lm;
    int n = 0, b = 0, cap = 0;
    if (lane < CS_NUM) { n = rs->len[lane]; b = dst->len[lane]; cap = dst->cap[lane]; }
    const bool fits = b + n <= cap;
    if (w == 0 && n > 0 && !fits) atomicOr(err, kErrSlotOverflow);
    unsigned todo = __ballot_sync(FDVB_FULL, n > 0 && fits);
    for (int r = 0; todo; ++r) {
        const int k = __ffs(todo) - 1;
        todo &= todo - 1;
        if ((r & 3) != w) continue;
        const int ns = __shfl_sync(FDVB_FULL, n, k), bs = __shfl_sync(FDVB_FULL, b, k);
        warp_copy_bytes(dst->buf[k] + bs, rm + (s32 ? leaf32_off(k) : leaf_off(k)), ns, lane);
    }
    cbar();
    if (t < CS_NUM && n > 0 && fits) dst->len[t] = b + n;
    cbar();
}

// z-scan index of a 4x4 cell in its CTU (fdv.h:3659) and the availability of
// an above-right cell (fdv.h:3677).
__device__ __forceinline__ int zidx4(int lx, int ly) {
    int z = 0;
    for (int b = 8; b; b >>= 1) z = (z << 2) | ((ly & b) ? 2 : 0) | ((lx & b) ? 1 : 0);
    return z;
}
__device__ __forceinline__ bool cell_done(int x, int y, int bx, int by) {
    int cx0 = bx & ~63, cy0 = by & ~63;
    if (y < cy0) return true;
    if (x < cx0) return true;
    if (x >= cx0 + 64) return false;
    return zidx4((x - cx0) >> 2, (y - cy0) >> 2) < zidx4((bx - cx0) >> 2, (by - cy0) >> 2);
}
// The allowed 4x4 modes as a mask (bit m: mode m), the same as mode_ok4:
// lanes testing different modes take no divergent branch.
__device__ __forceinline__ unsigned mode_mask4(int ht, int htr, int hl, int htl) {
    const unsigned a = ht ? 1u : 0u, l = hl ? 1u : 0u, tr = (ht && htr) ? 1u : 0u, d = (ht && hl && htl) ? 1u : 0u;
    return 1u | (a << 1) | (l << 2) | (l << 8) | (tr << 3) | (tr << 7) | (d * 0x70u);
}
__device__ __forceinline__ bool mode_ok4(int m, int ht, int htr, int hl, int htl) {
    switch (m) {
    case 0: return true;
    case 1: return ht;
    case 2: case 8: return hl;
    case 3: case 7: return ht && htr;
    default: return ht && hl && htl;
    }
}

// ------------------------------------------------------- 4x4 leaf --
// One 4x4 leaf (fdv.h:3907-4111) on the chain's four warps.  Every warp reads
// the neighbours itself; half-warp h of warp w predicts and SATD-screens mode
// 2w + h (warp 0 also mode 8).  From QP 12 up the screen keeps at most two
// candidates: every warp derives the reference's selection-sort order and
// ratio prune with two warp minimums, and the trials run at once -- the RD
// trials without RDOQ on warps 0-1, the RDOQ re-codes of both candidates on
// warps 2-3 -- so one barrier separates the screen from the trials and one
// the trials from the commit, which every warp applies to its own view of the
// tile.  Below QP 12 every screened mode is tried in the sorted order and the
// winner re-coded after.
__device__ double leaf4(CCtx &c, int bx, int by, ISink *tgt) {
    ChainArea &C = c.S->C;
    const QP4 &Q = c.S->q;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const long long t0 = prof_t0(c.prof, t);
    const int tx = bx - c.bx0, ty = by - c.by0;
    const int ht = by > 0, hl = bx > 0, htl = ht && hl;
    const int htr = ht && (bx + 4 < c.w) && cell_done(bx + 4, by - 1, bx, by);
    // neighbours (gather_neighbors fdv.h:3689-3706), one copy per screening
    // warp: N = L(3..0) T(-1) T(0..7) DC (pred4_table.h)
    if (w < 3) {
        // one predicated load per lane -- lanes 0-7 the row above (4-7
        // repeat T(3) without the above-right samples), 8-11 the column to
        // the left, 12 the corner -- and one store at the lane's place in N:
        // lane-dependent if/else chains would diverge, several times slower
        int *N = C.N4[w];
        const int ry = lane < 8 ? ty - 1 : (lane < 12 ? ty + lane - 8 : ty - 1);
        const int rx = lane < 8 ? tx + ((lane < 4 || htr) ? lane : 3) : tx - 1;
        const bool ok = lane < 8 ? ht : (lane < 12 ? hl : (lane == 12 && htl));
        const int v = ok ? (int)TL(C, ry, rx) : (lane == 12 ? 128 : 0);
        const int sT = __reduce_add_sync(FDVB_FULL, lane < 4 ? v : 0);
        const int sL = __reduce_add_sync(FDVB_FULL, (lane >= 8 && lane < 12) ? v : 0);
        const int dc = (ht && hl) ? (sT + sL + 4) >> 3 : (ht ? (sT + 2) >> 2 : (hl ? (sL + 2) >> 2 : 128));
        const int ni = lane < 8 ? 5 + lane : (lane < 12 ? 11 - lane : (lane == 12 ? 4 : 13));
        if (lane < 14) N[ni] = lane == 13 ? dc : v;
        __syncwarp();
        // predictions and SATD (fdv.h:3803-3823): 8 lanes per mode, modes
        // 0-3 on warp 0, 4-7 on warp 1, 8 on warp 2; a lane holds two
        // samples (row i, columns 2h and 2h + 1)
        const int m = w < 2 ? 4 * w + (lane >> 3) : 8;
        const int q = lane & 7, i = q >> 1, h = q & 1, x0 = 2 * h;
        const uint16_t *op = &C.p4[m * 16 + i * 4 + x0];
        const int p0 = p4_eval(op[0], N), p1 = p4_eval(op[1], N);
        C.cp[m][i * 4 + x0] = (uint8_t)p0;       // warp 2's lanes 8-31 repeat lanes 0-7
        C.cp[m][i * 4 + x0 + 1] = (uint8_t)p1;
        const int d0 = C.src[(ty + i) * 64 + tx + x0] - p0, d1 = C.src[(ty + i) * 64 + tx + x0 + 1] - p1;
        // row transform: columns (0, 1) on h = 0, (2, 3) on h = 1
        const int s0 = d0 + d1, s1 = d0 - d1;
        const int o0 = __shfl_xor_sync(FDVB_FULL, s0, 1), o1 = __shfl_xor_sync(FDVB_FULL, s1, 1);
        int c0 = h ? o0 - s0 : s0 + o0, c1 = h ? o1 - s1 : s1 + o1;
        // column transform over the rows: lanes q ^ 2 (rows i ^ 1), q ^ 4 (rows i ^ 2)
        {
            const int u0 = __shfl_xor_sync(FDVB_FULL, c0, 2), u1 = __shfl_xor_sync(FDVB_FULL, c1, 2);
            c0 = (i & 1) ? u0 - c0 : c0 + u0;
            c1 = (i & 1) ? u1 - c1 : c1 + u1;
        }
        {
            const int u0 = __shfl_xor_sync(FDVB_FULL, c0, 4), u1 = __shfl_xor_sync(FDVB_FULL, c1, 4);
            c0 = (i & 2) ? u0 - c0 : c0 + u0;
            c1 = (i & 2) ? u1 - c1 : c1 + u1;
        }
        int sa = abs(c0) + abs(c1);
        sa += __shfl_xor_sync(FDVB_FULL, sa, 1);
        sa += __shfl_xor_sync(FDVB_FULL, sa, 2);
        sa += __shfl_xor_sync(FDVB_FULL, sa, 4);
        C.csat[m] = sa;                           // every lane of the mode's group holds the sum
    }
    cbar();
    long long tp = prof_t0(c.prof, t);
    prof_add(c.prof, t, IP_L4SCREEN, t0);
    const uint8_t *sblk = &C.src[ty * 64 + tx];
    int mode, fsel;
    if (c.qp >= 12) {
        // The selection sort (fdv.h:3962-3975) for two places: the first
        // minimum, then the first minimum of the rest in the order left by the
        // swap (the first candidate moved to the winner's place); the prune
        // keeps the second only if its SATD is within 5/4 of the first's.
        const unsigned vmask = mode_mask4(ht, htr, hl, htl);
        const bool vm = (vmask >> lane) & 1u;
        const unsigned sv = vm ? (unsigned)C.csat[lane] : 0u;
        const unsigned k0 = __reduce_min_sync(FDVB_FULL, vm ? (sv << 4) | lane : 0xffffffffu);
        const int m0 = k0 & 15, s0 = k0 >> 4;
        const int first = __ffs(vmask) - 1;
        const int p0 = __popc(vmask & ((1u << m0) - 1));
        const int pos = lane == first ? p0 : __popc(vmask & ((1u << lane) - 1));
        const unsigned k1 = __reduce_min_sync(FDVB_FULL, (vm && lane != m0) ? (sv << 8) | (pos << 4) | lane : 0xffffffffu);
        const int m1 = k1 & 15, s1 = k1 >> 8;
        const int run = (__popc(vmask) >= 2 && !((long long)s1 * 4 > (long long)s0 * 5)) ? 2 : 1;
        if (c.prof && t == 0) atomicAdd(&c.prof[run == 1 ? IP_L4RUN1 : IP_L4RUN2], 1ull);
        prof_add(c.prof, t, IP_L4SELECT, tp);
        tp = prof_t0(c.prof, t);
        if (run == 1) {
            if (w == 0) warp_block4(sblk, 64, C.cp[m0], 4, C.frec[0], 4, Q, c.lambda, true, &C.fin[0], &C.b4[0], lane);
        } else {
            const int k = w & 1, mk = k ? m1 : m0;
            if (w < 2) warp_block4(sblk, 64, C.cp[mk], 4, C.junk[w], 4, Q, c.lambda, false, &C.trial[k], &C.b4[w], lane);
            else       warp_block4(sblk, 64, C.cp[mk], 4, C.frec[k], 4, Q, c.lambda, true, &C.fin[k], &C.b4[w], lane);
        }
        cbar();
        fsel = 0;
        if (run == 2) {   // trial costs are positive: the second wins only if strictly cheaper
            const double J0 = rd_cost((double)C.trial[0].ssd, c.lambda, kBitsMode + C.trial[0].bits);
            const double J1 = rd_cost((double)C.trial[1].ssd, c.lambda, kBitsMode + C.trial[1].bits);
            fsel = J1 < J0 ? 1 : 0;
        }
        mode = fsel ? m1 : m0;
    } else {
        if (t == 0) {   // the reference's selection sort over every screened mode
            int nc = 0;
            for (int m = 0; m < 9; ++m)
                if (mode_ok4(m, ht, htr, hl, htl)) { C.cs[nc] = C.csat[m]; C.cm[nc] = m; ++nc; }
            for (int a = 0; a < nc; ++a) {
                int bst = a;
                for (int b2 = a + 1; b2 < nc; ++b2) if (C.cs[b2] < C.cs[bst]) bst = b2;
                if (bst != a) {
                    int v = C.cs[a]; C.cs[a] = C.cs[bst]; C.cs[bst] = v;
                    v = C.cm[a]; C.cm[a] = C.cm[bst]; C.cm[bst] = v;
                }
            }
            C.run = nc;
        }
        cbar();
        const int run = C.run;
        for (int k = w; k < run; k += 4)
            warp_block4(sblk, 64, C.cp[C.cm[k]], 4, C.junk[w], 4, Q, c.lambda, false, &C.trial[k], &C.b4[w], lane);
        cbar();
        double best = -1.0;
        int bc = 0;
        for (int k = 0; k < run; ++k) {
            const double J = rd_cost((double)C.trial[k].ssd, c.lambda, kBitsMode + C.trial[k].bits);
            if (best < 0.0 || J < best) { best = J; bc = k; }
        }
        mode = C.cm[bc];
        if (w == 0) warp_block4(sblk, 64, C.cp[mode], 4, C.frec[0], 4, Q, c.lambda, true, &C.fin[0], &C.b4[0], lane);
        cbar();
        fsel = 0;
    }
    prof_add(c.prof, t, IP_L4TRIAL, tp);
    tp = prof_t0(c.prof, t);
    // commit: every warp writes the winner into the tile (the next leaf's
    // neighbours come from this warp's own writes); warp 3, which does not
    // screen, the symbols, while warps 0-2 go on to the next leaf's screen
    // (it reaches the barrier after that screen before the next trials
    // rewrite C.fin)
    const Blk4 &F = C.fin[fsel];
    {
        const int l = lane & 15;                  // lanes 16-31 repeat lanes 0-15
        TL(C, ty + (l >> 2), tx + (l & 3)) = C.frec[fsel][l];
    }
    __syncwarp();
    if (t == 96) {
        cs_put1(&tgt->c, CS_N, (uint8_t)F.count, c.err);
        cs_put(&tgt->c, CS_L, F.bytes, F.nbytes, c.err);
        const int lcx = tx >> 2, lcy = ty >> 2;
        const int Lm = bx > 0 ? MM(C, lcy, lcx - 1) : 0;
        const int Am = by > 0 ? MM(C, lcy - 1, lcx) : 0;
        isink_put(tgt, Lm == Am ? IS_MODE0 : IS_MODE1, (uint8_t)mode, c.err);
        MM(C, lcy, lcx) = (uint8_t)mode;
        if (c.prof) atomicAdd(&c.prof[IP_NLEAF4], 1ull);
    }
    prof_add(c.prof, t, IP_L4COMMIT, tp);
    prof_add(c.prof, t, IP_LEAF4, t0);
    return rd_cost((double)F.ssd, c.lambda, kBitsMode + F.bits);
}

// ------------------------------------------------------ chain: nodes --
// Post the leaf trial of the node of side n = 64 >> L at (bx, by) to its team
// and clear the node's split-trial sink.
__device__ void post_leaf_job(CCtx &c, int L, int bx, int by, int n, ISink *ss) {
    ChainArea &C = c.S->C;
    const int t = threadIdx.x, tx = bx - c.bx0, ty = by - c.by0;
    const int ht = by > 0, hl = bx > 0;
    HJob *J = cg::this_cluster().map_shared_rank(job_slot(&c.S->H, L), level_rank(L));
    if (t < n) J->top[t] = ht ? TL(C, ty - 1, tx + t) : 0;
    if (t >= 64 && t - 64 < n) J->left[t - 64] = hl ? TL(C, ty + t - 64, tx - 1) : 0;
    if (t == 1) {
        J->bx = bx; J->by = by; J->ht = ht; J->hl = hl;
        J->tl = (ht && hl) ? TL(C, ty - 1, tx - 1) : 128;
        J->kind = 0;
    }
    if (t == 2) isink_reset(ss);
    if (L < 3) fence_cluster();
    cbar();
    if (t == 0) st_release_cluster(&J->seq, ++C.issued[L]);
}
// Tell every team that the CTU row is over.
__device__ void post_row_end(IShared *S) {
    ChainArea &C = S->C;
    if (threadIdx.x == 0) {
        for (int L = 0; L < 4; ++L) {
            HJob *J = cg::this_cluster().map_shared_rank(job_slot(&S->H, L), level_rank(L));
            J->kind = 1;
            st_release_cluster(&J->seq, ++C.issued[L]);
        }
    }
}

template <int D> struct CNode {
    static __device__ double run(CCtx &c, int bx, int by, ISink *tgt);
};
template <> struct CNode<4> {
    static __device__ double run(CCtx &c, int bx, int by, ISink *tgt) {
        if (c.S->C.abort) return 0.0;
        return leaf4(c, bx, by, tgt);
    }
};

template <int D>
__device__ double CNode<D>::run(CCtx &c, int bx, int by, ISink *tgt) {
    constexpr int n = 64 >> D, hn = n / 2;
    IShared *S = c.S;
    ChainArea &C = S->C;
    const int t = threadIdx.x;
    if (C.abort) return 0.0;
    // The CTU's top-right 4x4 leaf reads the four samples above-right of the
    // CTU, in the next CTU of the row above, which an early-started CTU did
    // not wait for (only for the CTU above it): entering the top-right
    // quadrant, wait for that CTU and load them.  Every other read of the row
    // above lies above the CTU itself.
    if (D == 1 && c.early && bx == c.bx0 + 32 && by == c.by0 && by > 0 && c.bx0 + 64 < c.w) {
        if (t == 0 && !wait_at_least(&c.P->progress[c.by0 / 64 - 1], min(c.bx0 / 64 + 2, c.P->cols), c.err, c.wait_ns))
            C.abort = 1;
        cbar();
        if (t < 4) TL(C, -1, 64 + t) = __ldcg(&c.P->rec[(size_t)(by - 1) * c.w + c.bx0 + 64 + t]);
        cbar();
        if (C.abort) return 0.0;
    }
    if (bx + n > c.w || by + n > c.h) {            // implicit split, no flag
        double J = 0.0;
        for (int k = 0; k < 4; ++k) {
            const int cx = bx + (k & 1) * hn, cy = by + (k >> 1) * hn;
            if (cx >= c.w || cy >= c.h) continue;
            J = __dadd_rn(J, CNode<D + 1>::run(c, cx, cy, tgt));
        }
        return J;
    }
    ISink *ss = &C.ss[D];
    post_leaf_job(c, D, bx, by, n, ss);
    double Js = 0.0;
    for (int k = 0; k < 4; ++k) Js = __dadd_rn(Js, CNode<D + 1>::run(c, bx + (k & 1) * hn, by + (k >> 1) * hn, ss));
    // the leaf trial's result
    const long long tw = prof_t0(c.prof, t);
    if (t == 0 && !C.abort && !wait_cluster_flag(&C.done[D], C.issued[D], c.err, c.hlimit)) C.abort = 1;
    cbar();
    prof_add(c.prof, t, IP_HWAIT, tw);
    if (C.abort) return 0.0;
    const int rank = level_rank(D);
    const double Jl = C.res_J[D];
    const int bi = C.res_idx[D], mode = C.res_mode[D];
    const bool split = Js < Jl;
    if (t == 0) isink_put(tgt, IS_SPLIT0 + D, (uint8_t)split, c.err);
    if (split) {
        chain_isink_append(tgt, ss, c.err);
        return Js;
    }
    if (t == 0) isink_put(tgt, IS_MODEB, (uint8_t)mode, c.err);
    const HelperArea *RH = &S->H;
    if (rank != 0) {
        fence_cluster();
        RH = cg::this_cluster().map_shared_rank(&S->H, rank);
    }
    const int tx = bx - c.bx0, ty = by - c.by0;
    const uint32_t *rw = reinterpret_cast<const uint32_t *>(D == 1 ? RH->rec32[bi] : RH->rec[bi]);
    for (int p = t; p < n * n / 4; p += kChainNT) {
        const uint32_t v = rw[p];
        const int y = (p * 4) / n, x = (p * 4) % n;
#pragma unroll
        for (int q = 0; q < 4; ++q) TL(C, ty + y, tx + x + q) = (uint8_t)(v >> (8 * q));
    }
    constexpr int cells = n / 4;
    const int m4 = mode == 1 ? 1 : (mode == 2 ? 2 : 0);   // nn_to_4x4_mode
    for (int p = t; p < cells * cells; p += kChainNT) MM(C, (ty >> 2) + p / cells, (tx >> 2) + p % cells) = (uint8_t)m4;
    chain_append_leaf(&tgt->c, S, D, rank, bi, c.err);
    return Jl;
}

// The chain's walk over one CTU row.
__device__ void chain_row(IShared *S, const IPlaneDev &P, int r, unsigned *err, unsigned long long wait_ns,
                          unsigned long long hlimit) {
    ChainArea &C = S->C;
    const int t = threadIdx.x;
    CCtx c;
    c.S = S; c.P = &P; c.w = P.w; c.h = P.h; c.qp = P.qp; c.lambda = P.lambda; c.err = err; c.prof = P.prof;
    c.hlimit = hlimit;
    c.wait_ns = wait_ns;
    c.early = P.rows > 2;
    const int mmw = P.w / 4, mmh = P.h / 4;
    if (t == 0) C.abort = 0;
    for (int col = 0; col < P.cols; ++col) {
        const long long tw = prof_t0(c.prof, t);
        // the CTU above finished, and on planes of more than two CTU rows
        // only that one (the one above-right is waited for at the CTU's
        // top-right 4x4 leaf, the only part of the CTU that reads it); on
        // shorter planes the row below has nothing to overlap and waits for
        // both at its start
        if (r > 0) {
            if (t == 0)
                C.row_ok = wait_at_least(&P.progress[r - 1], min(col + (c.early ? 1 : 2), P.cols), err, wait_ns);
        } else if (t == 0) C.row_ok = 1;
        cbar();
        if (!C.row_ok) break;
        prof_add(c.prof, t, IP_WAIT, tw);
        const long long tc = prof_t0(c.prof, t);
        const int bx0 = col * 64, by0 = r * 64;
        c.bx0 = bx0; c.by0 = by0;
        // the source block, the reconstruction above / left and their modes
        for (int p = t; p < 64 * 16; p += kChainNT) {
            const int y = by0 + p / 16, x = bx0 + (p % 16) * 4;
            uint32_t v = 0;
            if (y < P.h) {
#pragma unroll
                for (int q = 0; q < 4; ++q) if (x + q < P.w) v |= (uint32_t)P.src[(size_t)y * P.w + x + q] << (8 * q);
            }
            reinterpret_cast<uint32_t *>(C.src)[p] = v;
        }
        for (int p = t; p < kTileW; p += kChainNT) {
            const int x = bx0 - 1 + p, y = by0 - 1;
            C.tile[p] = (y >= 0 && x >= 0 && x < P.w) ? __ldcg(&P.rec[(size_t)y * P.w + x]) : 0;
        }
        if (t < 64) {
            const int x = bx0 - 1, y = by0 + t;
            TL(C, t, -1) = (x >= 0 && y < P.h) ? __ldcg(&P.rec[(size_t)y * P.w + x]) : 0;
        } else if (t < 64 + 17) {
            const int p = t - 64, cx = bx0 / 4 - 1 + p, cy = by0 / 4 - 1;
            C.mm[p] = (cy >= 0 && cx >= 0 && cx < mmw) ? __ldcg(&P.mmap[(size_t)cy * mmw + cx]) : 0;
        } else if (t < 64 + 17 + 16) {
            const int p = t - 81, cx = bx0 / 4 - 1, cy = by0 / 4 + p;
            MM(C, p, -1) = (cx >= 0 && cy < mmh) ? __ldcg(&P.mmap[(size_t)cy * mmw + cx]) : 0;
        }
        uint8_t *slot = P.slots + (size_t)(r * P.cols + col) * kISlotBytes;
        if (t == 0) {
            ISink *o = &C.out;
            for (int k = 0; k < IS_NS; ++k) { o->slen[k] = 0; o->scap[k] = c_IStreamCap[k]; o->sbuf[k] = slot + 32 + c_IStreamOff[k]; }
            int cc[CS_NUM] = {c_IStreamCap[7], c_IStreamCap[8], c_IStreamCap[9], c_IStreamCap[10], c_IStreamCap[11], 0, 0};
            cs_init(&o->c, slot + 32 + c_IStreamOff[7], cc);
        }
        cbar();
        CNode<0>::run(c, bx0, by0, &C.out);
        if (C.abort) break;
        // write back the reconstruction, the mode map and the slot lengths
        for (int p = t; p < 64 * 64; p += kChainNT) {
            const int y = by0 + p / 64, x = bx0 + p % 64;
            if (y < P.h && x < P.w) P.rec[(size_t)y * P.w + x] = TL(C, p / 64, p % 64);
        }
        for (int p = t; p < 256; p += kChainNT) {
            const int cy = by0 / 4 + p / 16, cx = bx0 / 4 + p % 16;
            if (cy < mmh && cx < mmw) P.mmap[(size_t)cy * mmw + cx] = MM(C, p / 16, p % 16);
        }
        if (t < 12) {
            const int len = t < IS_NS ? C.out.slen[t] : C.out.c.len[t - IS_NS];
            reinterpret_cast<uint16_t *>(slot)[t] = (uint16_t)len;
        }
        cbar();   // orders the chain's writes before thread 0's fence and flag
        if (t == 0) {
            __threadfence();
            atomicExch(&P.progress[r], col + 1);
        }
        prof_add(c.prof, t, IP_CTU, tc);
        if (c.prof && t == 0) atomicAdd(&c.prof[IP_NCTU], 1ull);
    }
    post_row_end(S);
}

// ------------------------------------------------------- leaf teams --
// A team codes the leaf trial of one node: every allowed mode
// (fdv_intra_nn_mode_ok) of the n x n leaf at once through team_residuals,
// then the reference's choice among them (the first strictly cheaper,
// fdv.h:4467-4471), into the result area (rec, sink), then posts the cost,
// the choice and job number `seq` of level L to the chain.
template <int NT, int BAR>
__device__ void team_code(IShared *S, const IPlaneDev &P, int L, const HJob &job, uint8_t *const *rec,
                          CoefSink *const *sink, int seq, unsigned *err, int tt) {
    HelperArea &H = S->H;
    const int n = 64 >> L;
    ChainArea *RC = cg::this_cluster().map_shared_rank(&S->C, 0);
    unsigned long long *prof = P.prof;
    const long long t0 = prof_t0(prof, tt);
    const int bx = job.bx, by = job.by, ht = job.ht, hl = job.hl, tl = job.tl;
    for (int p = tt; p < n * n; p += NT) {
        const int y = p / n, x = p % n;
        H.src[y * 64 + x] = P.src[(size_t)(by + y) * P.w + bx + x];
    }
    if (tt < 4) {
        H.nn[tt] = nn_setup(tt, job.top, job.left, tl, n, ht, hl);
        cs_reset(sink[tt]);
    }
    if (tt == 0) {
        int nm = 0;
        for (int m = 0; m < 4; ++m) if (nn_mode_ok(m, n, ht, hl)) H.ml[nm++] = m;
        H.nm = nm;
    }
    team_bar(BAR, NT);
    const int M = H.nm, nn2 = n * n;
    for (int p = tt; p < M * nn2; p += NT) {
        const int i = p / nn2, q = p - i * nn2;
        H.pred[i][q] = (uint8_t)nn_px(H.nn[H.ml[i]], job.top, job.left, q % n, q / n);
    }
    team_bar(BAR, NT);
    uint8_t *pr[4] = {H.pred[0], H.pred[1], H.pred[2], H.pred[3]};
    team_residuals<NT>(H.src, 64, pr, rec, sink, M, n, S->q, P.qp, P.lambda, H.e, H.b, &H.ts, err, tt, BAR);
    if (tt == 0) {
        double best = -1.0;
        int bi = 0;
        for (int i = 0; i < M; ++i) {
            const double J = rd_cost((double)H.e[i], P.lambda, kBitsMode + H.b[i]);
            if (best < 0.0 || J < best) { best = J; bi = i; }
        }
        RC->res_J[L] = best;
        RC->res_idx[L] = bi;
        RC->res_mode[L] = H.ml[bi];
    }
    if (L < 3) fence_cluster();
    team_bar(BAR, NT);
    if (tt == 0) st_release_cluster(&RC->done[L], seq);
    prof_add(prof, tt, IP_LEAF64 - L, t0);
}

// The team of one node size (block 0's 8x8 team, block 1's 16x16 team) until
// the chain ends the CTU row.  `seen` counts the jobs this team has taken.
template <int NT, int BAR>
__device__ void team_loop(IShared *S, const IPlaneDev &P, int L, unsigned *err, unsigned long long hlimit, int tt,
                          int &seen) {
    HelperArea &H = S->H;
    uint8_t *rec[4] = {H.rec[0], H.rec[1], H.rec[2], H.rec[3]};
    CoefSink *sink[4] = {&H.sink[0], &H.sink[1], &H.sink[2], &H.sink[3]};
    for (;;) {
        if (tt == 0) H.ok = wait_cluster_flag(&H.job.seq, seen + 1, err, hlimit);
        team_bar(BAR, NT);
        fence_cluster();
        if (!H.ok) break;
        ++seen;
        if (H.job.kind != 0) break;
        team_code<NT, BAR>(S, P, L, H.job, rec, sink, seen, err, tt);
    }
}

// Block 2: the 32x32 jobs (slot job, results in rec32 / sink32) and the
// 64x64 job (slot job64, results in rec / sink) until the chain has ended the
// CTU row on both.  seen32 / seen64 count the jobs taken from each slot.
template <int NT, int BAR>
__device__ void team_loop_3264(IShared *S, const IPlaneDev &P, unsigned *err, unsigned long long hlimit, int tt,
                               int &seen32, int &seen64) {
    HelperArea &H = S->H;
    uint8_t *rec64[4] = {H.rec[0], H.rec[1], H.rec[2], H.rec[3]};
    CoefSink *sink64[4] = {&H.sink[0], &H.sink[1], &H.sink[2], &H.sink[3]};
    uint8_t *rec32[4] = {H.rec32[0], H.rec32[1], H.rec32[2], H.rec32[3]};
    CoefSink *sink32[4] = {&H.sink32[0], &H.sink32[1], &H.sink32[2], &H.sink32[3]};
    bool end32 = false, end64 = false;
    while (!(end32 && end64)) {
        if (tt == 0) {
            // bounded wait for a job in either slot, a 32x32 one first
            int ok = 0, sel = 0;
            const unsigned long long t0 = globaltimer();
            for (;;) {
                if (!end32 && ld_acquire_cluster(&H.job.seq) >= seen32 + 1) { ok = 1; sel = 1; break; }
                if (!end64 && ld_acquire_cluster(&H.job64.seq) >= seen64 + 1) { ok = 1; sel = 0; break; }
                if (*(volatile unsigned *)err) break;
                if (globaltimer() - t0 > hlimit) { atomicOr(err, kErrWaitTimeout); break; }
                __nanosleep(32);
            }
            H.ok = ok;
            H.sel = sel;
        }
        team_bar(BAR, NT);
        fence_cluster();
        if (!H.ok) break;
        const int L = H.sel ? 1 : 0;
        const HJob &job = L ? H.job : H.job64;
        const int seq = L ? ++seen32 : ++seen64;
        if (job.kind != 0) {
            if (L) end32 = true;
            else end64 = true;
            team_bar(BAR, NT);   // every thread has read the slot before the next wait
            continue;
        }
        team_code<NT, BAR>(S, P, L, job, L ? rec32 : rec64, L ? sink32 : sink64, seq, err, tt);
    }
}

__global__ void __cluster_dims__(ICL, 1, 1) __launch_bounds__(INT, 1)
iframe_kernel(const IPlaneDev *__restrict__ planes, const ITask *__restrict__ tasks, int ntasks,
              int *ticket, unsigned *err, unsigned long long wait_ns) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    IShared *S = reinterpret_cast<IShared *>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x, rank = (int)cl.block_rank();
    // team waits may span a whole CTU row, including the chain's own waits
    const unsigned long long hlimit = 2 * wait_ns + 1000000000ull;
    if (tid == 0) {
        ChainArea &C = S->C;
        uint8_t *m = C.ssmem;
        for (int d = 0; d < 4; ++d) {
            ISink *s = &C.ss[d];
            for (int k = 0; k < IS_NS; ++k) { s->slen[k] = 0; s->scap[k] = isink_scap(d, k); s->sbuf[k] = m; m += s->scap[k]; }
            int cc[CS_NUM];
            for (int k = 0; k < CS_NUM; ++k) cc[k] = isink_ccap(d, k);
            cs_init(&s->c, m, cc);
            for (int k = 0; k < CS_NUM; ++k) m += cc[k];
        }
        int c0[CS_NUM];
        for (int k = 0; k < CS_NUM; ++k) c0[k] = isink_ccap(0, k);
        for (int i = 0; i < 4; ++i) cs_init(&S->H.sink[i], S->H.sinkmem[i], c0);
        int c1[CS_NUM];
        for (int k = 0; k < CS_NUM; ++k) c1[k] = isink_ccap(1, k);
        for (int i = 0; i < 4; ++i) cs_init(&S->H.sink32[i], S->H.sinkmem32[i], c1);
        for (int L = 0; L < 4; ++L) { C.done[L] = 0; C.issued[L] = 0; }
        for (int k = 0; k < 9 * 16; ++k) C.p4[k] = g_p4tab.op[k];
        S->H.job.seq = 0;
        S->H.job64.seq = 0;
    }
    int seen = 0, seen64 = 0;
    cl.sync();
    for (;;) {
        if (rank == 0 && tid == 0) S->C.task = atomicAdd(ticket, 1);
        cl.sync();
        const int t = *cl.map_shared_rank(&S->C.task, 0);
        cl.sync();
        if (t >= ntasks) break;
        const IPlaneDev &P = planes[tasks[t].plane];
        qp4_setup(&S->q, P.qp, tid);
        __syncthreads();
        if (rank == 0) {
            if (tid < kChainNT) chain_row(S, P, tasks[t].row, err, wait_ns, hlimit);
            else if (tid < kChainNT + kH8NT) team_loop<kH8NT, BAR_H8>(S, P, 3, err, hlimit, tid - kChainNT, seen);
        } else if (rank == 1) {
            team_loop<INT, BAR_TEAM>(S, P, 2, err, hlimit, tid, seen);
        } else {
            team_loop_3264<INT, BAR_TEAM>(S, P, err, hlimit, tid, seen, seen64);
        }
    }
}

size_t iframe_smem_bytes() { return sizeof(IShared); }
int iframe_slot_bytes() { return kISlotBytes; }
void iframe_slot_offsets(int off[12]) { for (int k = 0; k < 12; ++k) off[k] = islot_off(k); }

}  // namespace fdvb

// Key-frame analysis: the intra quadtree of the image codec as a persistent
// wavefront kernel over coding tree units.
//
// Work unit: one 64x64 CTU row of one plane of one encoder unit; rows are
// taken from an atomic ticket in plane order.  CTU (c, r) starts once row r-1
// has finished CTU c+1 -- the top-right samples a 4x4 leaf on the CTU's top
// edge may read -- exactly the reference's wavefront (intra_ctu_row,
// fdv.h:4698-4725), with bounded waits.
//
// Inside a CTU the 512 threads walk the quadtree in the reference's order
// (intra_node, fdv.h:4494-4582): at every node inside the plane the split trial
// (four children, recursively) and then the leaf trial, kept if strictly
// cheaper; nodes crossing the plane edge split with no flag; 4x4 leaves choose
// among the nine directions by SATD screen and RD trial and are re-coded with
// RDOQ (intra_leaf4, fdv.h:3907-4111).  The recursion is unrolled at compile
// time (inode<D>).  The CTU's reconstruction, its 4x4 mode map and every
// trial's symbols live in shared memory; the winner is appended to the CTU's
// output slot.  A 4x4 leaf runs on one warp; a larger leaf's four sub-modes and
// their 8x8 regions use all sixteen warps.
#include "common.cuh"
#include "intra.cuh"
#include "residual.cuh"

namespace fdvb {

constexpr int INT = 512;              // threads per block
constexpr int kTileW = 129;           // tile columns: x in [-1, 127] relative to the CTU

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
};
struct ITask { int plane, row; };

// Per-depth sink capacities (node of side n = 64 >> d, see nd_struct/nd_cnt/nd_lvl fdv.h:4312-4314).
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
constexpr int kLeafSinkBytes = isink_ccap(0, 0) + isink_ccap(0, 1) + isink_ccap(0, 2) + isink_ccap(0, 3) + isink_ccap(0, 4);

struct IShared {
    QP4 q;
    uint8_t tile[65 * kTileW];            // reconstruction: rows -1..63, cols -1..127
    uint8_t src[64 * 64];
    uint8_t mm[17 * 17];                  // mode map: cells -1..15 x -1..15
    uint8_t stash_rec[64 * 64 + 32 * 32 + 16 * 16 + 8 * 8];
    uint8_t stash_mm[16 * 16 + 8 * 8 + 4 * 4 + 2 * 2];
    uint8_t pred[4][16 * 16];             // leaf trial predictions (all four modes when n <= 16)
    uint8_t trec[4][64 * 64 / 4 > 256 ? 1024 : 1024];
    uint8_t bigpred[64 * 64];
    uint8_t bigrec[2][64 * 64];
    ISink ss[4];                          // split trial sinks per depth
    uint8_t ssmem[isink_bytes(0) + isink_bytes(1) + isink_bytes(2) + isink_bytes(3)];
    CoefSink lsink[4];                    // leaf trial sinks (parallel modes, or ping-pong)
    uint8_t lsmem[4][isink_ccap(2, 0) + isink_ccap(2, 1) + isink_ccap(2, 2) + isink_ccap(2, 3) + isink_ccap(2, 4)];
    CoefSink bsink[2];                    // ping-pong for n >= 32
    uint8_t bsmem[2][kLeafSinkBytes];
    ResidScratchT<INT> rs;
    ISink out;                            // the CTU's output (global)
    // 4x4 leaf scratch (warp 0)
    uint8_t cp[9][16];
    int csat[9], cmode[9], ncand, ntry;
    Blk4 trial[9];
    Blk4 fin;
    uint8_t trec4[16];
    Blk4Scratch b4;
    uint8_t nb_top[64], nb_left[64];
    int nb_tl, nb_ht, nb_hl;
    NNPred nn[4];
    double J[4];
    int jbits[4];
    long long jd[4];
    double retJ;
    int retMode;
    int task, row_ok;
};

struct ICtx {
    IShared *S;
    const IPlaneDev *P;
    int bx0, by0, w, h, qp;
    double lambda;
    unsigned *err;
};

__device__ __forceinline__ uint8_t &TL(IShared *S, int ty, int tx) { return S->tile[(ty + 1) * kTileW + tx + 1]; }
__device__ __forceinline__ uint8_t &MM(IShared *S, int cy, int cx) { return S->mm[(cy + 1) * 17 + cx + 1]; }

__device__ void isink_reset(ISink *s) {
    for (int k = 0; k < IS_NS; ++k) s->slen[k] = 0;
    cs_reset(&s->c);
}
__device__ void isink_put(ISink *s, int k, uint8_t v, unsigned *err) {
    if (s->slen[k] + 1 > s->scap[k]) { atomicOr(err, kErrSlotOverflow); return; }
    s->sbuf[k][s->slen[k]++] = v;
}
// dst += src (all threads; lengths updated after a barrier).
__device__ void isink_append(ISink *dst, const ISink *src, unsigned *err) {
    const int tid = threadIdx.x;
    for (int k = 0; k < IS_NS; ++k) {
        int n = src->slen[k], b = dst->slen[k];
        if (b + n > dst->scap[k]) { if (tid == 0) atomicOr(err, kErrSlotOverflow); continue; }
        for (int i = tid; i < n; i += INT) dst->sbuf[k][b + i] = src->sbuf[k][i];
    }
    for (int k = 0; k < CS_NUM; ++k) {
        int n = src->c.len[k], b = dst->c.len[k];
        if (b + n > dst->c.cap[k]) { if (tid == 0) atomicOr(err, kErrSlotOverflow); continue; }
        for (int i = tid; i < n; i += INT) dst->c.buf[k][b + i] = src->c.buf[k][i];
    }
    __syncthreads();
    if (tid == 0) {
        for (int k = 0; k < IS_NS; ++k) if (dst->slen[k] + src->slen[k] <= dst->scap[k]) dst->slen[k] += src->slen[k];
        for (int k = 0; k < CS_NUM; ++k) if (dst->c.len[k] + src->c.len[k] <= dst->c.cap[k]) dst->c.len[k] += src->c.len[k];
    }
    __syncthreads();
}
__device__ void csink_append(CoefSink *dst, const CoefSink *src, unsigned *err) {
    const int tid = threadIdx.x;
    for (int k = 0; k < CS_NUM; ++k) {
        int n = src->len[k], b = dst->len[k];
        if (b + n > dst->cap[k]) { if (tid == 0) atomicOr(err, kErrSlotOverflow); continue; }
        for (int i = tid; i < n; i += INT) dst->buf[k][b + i] = src->buf[k][i];
    }
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < CS_NUM; ++k) if (dst->len[k] + src->len[k] <= dst->cap[k]) dst->len[k] += src->len[k];
    __syncthreads();
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
__device__ __forceinline__ bool mode_ok4(int m, int ht, int htr, int hl, int htl) {
    switch (m) {
    case 0: return true;
    case 1: return ht;
    case 2: case 8: return hl;
    case 3: case 7: return ht && htr;
    default: return ht && hl && htl;
    }
}

// One 4x4 leaf (fdv.h:3907-4111) on warp 0; all threads call, the result is
// returned uniformly.
__device__ double leaf4(ICtx &c, int bx, int by, ISink *tgt) {
    IShared *S = c.S;
    const int tid = threadIdx.x, lane = tid & 31;
    const int tx = bx - c.bx0, ty = by - c.by0;
    if (tid < 32) {
        const int ht = by > 0, hl = bx > 0, htl = ht && hl;
        const int htr = ht && (bx + 4 < c.w) && cell_done(bx + 4, by - 1, bx, by);
        // neighbours (gather_neighbors fdv.h:3689-3706)
        __shared__ uint8_t top[8], left[4];
        __shared__ int tlv;
        if (lane < 8) {
            int v = 0;
            if (ht) v = (lane < 4 || htr) ? TL(S, ty - 1, tx + lane) : TL(S, ty - 1, tx + 3);
            top[lane] = (uint8_t)v;
        } else if (lane < 12) {
            left[lane - 8] = hl ? TL(S, ty + lane - 8, tx - 1) : 0;
        } else if (lane == 12) {
            tlv = htl ? TL(S, ty - 1, tx - 1) : 128;
        }
        __syncwarp();
        // predict the allowed modes and SATD-screen them
        if (lane < 9) {
            int m = lane;
            if (mode_ok4(m, ht, htr, hl, htl)) {
                int Tn[9], Ln[5];
                Tn[0] = tlv; for (int k = 0; k < 8; ++k) Tn[k + 1] = top[k];
                Ln[0] = tlv; for (int k = 0; k < 4; ++k) Ln[k + 1] = left[k];
                for (int p = 0; p < 16; ++p) S->cp[m][p] = (uint8_t)pred4_px(m, Tn, Ln, top, left, ht, hl, p & 3, p >> 2);
                S->csat[m] = satd4(&S->src[ty * 64 + tx], 64, S->cp[m], 4);
            }
        }
        __syncwarp();
        if (lane == 0) {
            int cs[9], cm[9], nc = 0;
            for (int m = 0; m < 9; ++m) if (mode_ok4(m, ht, htr, hl, htl)) { cs[nc] = S->csat[m]; cm[nc] = m; ++nc; }
            int ntry = c.qp < 12 ? nc : (nc < 2 ? nc : 2);
            for (int a = 0; a < ntry; ++a) {
                int bst = a;
                for (int b2 = a + 1; b2 < nc; ++b2) if (cs[b2] < cs[bst]) bst = b2;
                if (bst != a) { int t = cs[a]; cs[a] = cs[bst]; cs[bst] = t; t = cm[a]; cm[a] = cm[bst]; cm[bst] = t; }
            }
            // how many trials run before the SATD prune breaks the loop (fdv.h:3987-3990)
            int run = 0;
            for (int k = 0; k < ntry; ++k) {
                if (k > 0 && c.qp >= 12 && (long long)cs[k] * 4 > (long long)cs[0] * 5) break;
                ++run;
            }
            for (int k = 0; k < run; ++k) S->cmode[k] = cm[k];
            S->ntry = run;
        }
        __syncwarp();
        const int run = S->ntry;
        double best_cost = -1.0;
        int best_c = 0;
        for (int k = 0; k < run; ++k) {
            warp_block4(&S->src[ty * 64 + tx], 64, S->cp[S->cmode[k]], 4, S->trec4, 4, S->q, c.lambda, false,
                        &S->trial[k], &S->b4, lane);
            double J = rd_cost((double)S->trial[k].ssd, c.lambda, kBitsMode + S->trial[k].bits);
            if (best_cost < 0.0 || J < best_cost) { best_cost = J; best_c = k; }
        }
        const int mode = S->cmode[best_c];
        // re-code the winner with RDOQ straight into the reconstruction tile
        warp_block4(&S->src[ty * 64 + tx], 64, S->cp[mode], 4, &TL(S, ty, tx), kTileW, S->q, c.lambda, true,
                    &S->fin, &S->b4, lane);
        if (lane == 0) {
            cs_put1(&tgt->c, CS_N, (uint8_t)S->fin.count, c.err);
            cs_put(&tgt->c, CS_L, S->fin.bytes, S->fin.nbytes, c.err);
            int lcx = tx >> 2, lcy = ty >> 2;
            int Lm = bx > 0 ? MM(S, lcy, lcx - 1) : 0;
            int Am = by > 0 ? MM(S, lcy - 1, lcx) : 0;
            isink_put(tgt, Lm == Am ? IS_MODE0 : IS_MODE1, (uint8_t)mode, c.err);
            MM(S, lcy, lcx) = (uint8_t)mode;
            S->retJ = rd_cost((double)S->fin.ssd, c.lambda, kBitsMode + S->fin.bits);
        }
    }
    __syncthreads();
    double J = S->retJ;
    __syncthreads();
    return J;
}

// Gather a leaf's n top / n left neighbours from the tile (gather_nb fdv.h:5201).
__device__ void gather_leaf_nb(ICtx &c, int bx, int by, int n) {
    IShared *S = c.S;
    const int tid = threadIdx.x, tx = bx - c.bx0, ty = by - c.by0;
    const int ht = by > 0, hl = bx > 0;
    if (tid < n) S->nb_top[tid] = ht ? TL(S, ty - 1, tx + tid) : 0;
    else if (tid >= 64 && tid < 64 + n) S->nb_left[tid - 64] = hl ? TL(S, ty + tid - 64, tx - 1) : 0;
    if (tid == 0) { S->nb_ht = ht; S->nb_hl = hl; S->nb_tl = (ht && hl) ? TL(S, ty - 1, tx - 1) : 128; }
    __syncthreads();
    if (tid < 4) S->nn[tid] = nn_setup(tid, S->nb_top, S->nb_left, S->nb_tl, n, S->nb_ht, S->nb_hl);
    __syncthreads();
}

// An n x n leaf (intra_leafn fdv.h:4442-4484): the allowed sub-modes coded
// through the residual coder, the cheapest (first strictly better) kept.
// Leaves the winner's reconstruction in the tile and returns its cost; the
// winner's coefficient sink is *best_sink.
template <int n>
__device__ double leafn(ICtx &c, int bx, int by, int *mode_out, CoefSink **best_sink) {
    IShared *S = c.S;
    const int tid = threadIdx.x, tx = bx - c.bx0, ty = by - c.by0;
    gather_leaf_nb(c, bx, by, n);
    const int ht = S->nb_ht, hl = S->nb_hl;
    double best = -1.0;
    int bmode = 0, bidx = 0;
    if (n <= 16) {
        // all allowed modes at once: each mode's regions are independent work
        if (tid < 4) cs_reset(&S->lsink[tid]);
        for (int p = tid; p < 4 * n * n; p += INT) {
            int m = p / (n * n), q = p % (n * n);
            S->pred[m][q] = (uint8_t)nn_px(S->nn[m], S->nb_top, S->nb_left, q % n, q / n);
        }
        __syncthreads();
        for (int m = 0; m < 4; ++m) {
            if (!nn_mode_ok(m, n, ht, hl)) continue;
            int bits = kBitsMode;
            long long D = code_residual_t<INT>(&S->src[ty * 64 + tx], 64, S->pred[m], n, n, S->q, c.qp, c.lambda, false,
                                               S->trec[m], n, &S->lsink[m], &bits, &S->rs, c.err);
            double J = rd_cost((double)D, c.lambda, bits);
            if (best < 0.0 || J < best) { best = J; bmode = m; bidx = m; }
        }
        for (int p = tid; p < n * n; p += INT) TL(S, ty + p / n, tx + p % n) = S->trec[bidx][p];
        *best_sink = &S->lsink[bidx];
    } else {
        int cur = 0;
        bidx = -1;
        for (int m = 0; m < 4; ++m) {
            if (!nn_mode_ok(m, n, ht, hl)) continue;
            const int t = bidx == 0 ? 1 : 0;
            if (tid == 0) cs_reset(&S->bsink[t]);
            for (int p = tid; p < n * n; p += INT) S->bigpred[p] = (uint8_t)nn_px(S->nn[m], S->nb_top, S->nb_left, p % n, p / n);
            __syncthreads();
            int bits = kBitsMode;
            long long D = code_residual_t<INT>(&S->src[ty * 64 + tx], 64, S->bigpred, n, n, S->q, c.qp, c.lambda, false,
                                               S->bigrec[t], n, &S->bsink[t], &bits, &S->rs, c.err);
            double J = rd_cost((double)D, c.lambda, bits);
            if (best < 0.0 || J < best) { best = J; bmode = m; bidx = t; }
            cur = t;
        }
        (void)cur;
        for (int p = tid; p < n * n; p += INT) TL(S, ty + p / n, tx + p % n) = S->bigrec[bidx][p];
        *best_sink = &S->bsink[bidx];
    }
    __syncthreads();
    *mode_out = bmode;
    return best;
}

__device__ __forceinline__ int nn_to_4x4(int m) { return m == 1 ? 1 : (m == 2 ? 2 : 0); }

template <int D> struct INode {
    static __device__ double run(ICtx &c, int bx, int by, ISink *tgt);
};

template <> struct INode<4> {
    static __device__ double run(ICtx &c, int bx, int by, ISink *tgt) { return leaf4(c, bx, by, tgt); }
};

template <int D>
__device__ double INode<D>::run(ICtx &c, int bx, int by, ISink *tgt) {
    constexpr int n = 64 >> D, hn = n / 2;
    IShared *S = c.S;
    const int tid = threadIdx.x;
    if (bx + n > c.w || by + n > c.h) {
        double J = 0.0;
        for (int k = 0; k < 4; ++k) {
            int cx = bx + (k & 1) * hn, cy = by + (k >> 1) * hn;
            if (cx >= c.w || cy >= c.h) continue;
            J = __dadd_rn(J, INode<D + 1>::run(c, cx, cy, tgt));
        }
        return J;
    }
    ISink *ss = &S->ss[D];
    if (tid == 0) isink_reset(ss);
    __syncthreads();
    double Jsplit = 0.0;
    for (int k = 0; k < 4; ++k)
        Jsplit = __dadd_rn(Jsplit, INode<D + 1>::run(c, bx + (k & 1) * hn, by + (k >> 1) * hn, ss));
    // stash the split trial's reconstruction and mode map
    constexpr int rs_off = D == 0 ? 0 : (D == 1 ? 4096 : (D == 2 ? 5120 : 5376));
    constexpr int ms_off = D == 0 ? 0 : (D == 1 ? 256 : (D == 2 ? 320 : 336));
    constexpr int cells = n / 4;
    const int tx = bx - c.bx0, ty = by - c.by0;
    for (int p = tid; p < n * n; p += INT) S->stash_rec[rs_off + p] = TL(S, ty + p / n, tx + p % n);
    for (int p = tid; p < cells * cells; p += INT) S->stash_mm[ms_off + p] = MM(S, (ty >> 2) + p / cells, (tx >> 2) + p % cells);
    __syncthreads();
    int mode = 0;
    CoefSink *lbest = nullptr;
    double Jleaf = leafn<n>(c, bx, by, &mode, &lbest);
    const bool split = Jsplit < Jleaf;
    if (tid == 0) isink_put(tgt, IS_SPLIT0 + D, (uint8_t)split, c.err);
    if (split) {
        for (int p = tid; p < n * n; p += INT) TL(S, ty + p / n, tx + p % n) = S->stash_rec[rs_off + p];
        for (int p = tid; p < cells * cells; p += INT) MM(S, (ty >> 2) + p / cells, (tx >> 2) + p % cells) = S->stash_mm[ms_off + p];
        __syncthreads();
        isink_append(tgt, ss, c.err);
        return Jsplit;
    }
    if (tid == 0) isink_put(tgt, IS_MODEB, (uint8_t)mode, c.err);
    for (int p = tid; p < cells * cells; p += INT) MM(S, (ty >> 2) + p / cells, (tx >> 2) + p % cells) = (uint8_t)nn_to_4x4(mode);
    __syncthreads();
    csink_append(&tgt->c, lbest, c.err);
    return Jleaf;
}

__global__ void __launch_bounds__(INT, 1)
iframe_kernel(const IPlaneDev *__restrict__ planes, const ITask *__restrict__ tasks, int ntasks,
              int *ticket, unsigned *err, unsigned long long wait_ns) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    IShared *S = reinterpret_cast<IShared *>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) {
        uint8_t *m = S->ssmem;
        for (int d = 0; d < 4; ++d) {
            ISink *s = &S->ss[d];
            for (int k = 0; k < IS_NS; ++k) { s->slen[k] = 0; s->scap[k] = isink_scap(d, k); s->sbuf[k] = m; m += s->scap[k]; }
            int cc[CS_NUM];
            for (int k = 0; k < CS_NUM; ++k) cc[k] = isink_ccap(d, k);
            cs_init(&s->c, m, cc);
            for (int k = 0; k < CS_NUM; ++k) m += cc[k];
        }
        int c2[CS_NUM], c0[CS_NUM];
        for (int k = 0; k < CS_NUM; ++k) { c2[k] = isink_ccap(2, k); c0[k] = isink_ccap(0, k); }
        for (int i = 0; i < 4; ++i) cs_init(&S->lsink[i], S->lsmem[i], c2);
        for (int i = 0; i < 2; ++i) cs_init(&S->bsink[i], S->bsmem[i], c0);
    }
    __syncthreads();
    for (;;) {
        if (tid == 0) S->task = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = S->task;
        __syncthreads();
        if (t >= ntasks) return;
        const IPlaneDev &P = planes[tasks[t].plane];
        const int r = tasks[t].row;
        ICtx c;
        c.S = S; c.P = &P; c.w = P.w; c.h = P.h; c.qp = P.qp; c.lambda = P.lambda; c.err = err;
        qp4_setup(&S->q, P.qp, tid);
        const int mmw = P.w / 4, mmh = P.h / 4;
        for (int col = 0; col < P.cols; ++col) {
            if (r > 0) {
                if (tid == 0) S->row_ok = wait_at_least(&P.progress[r - 1], min(col + 2, P.cols), err, wait_ns);
            } else if (tid == 0) S->row_ok = 1;
            __syncthreads();
            if (!S->row_ok) break;
            const int bx0 = col * 64, by0 = r * 64;
            c.bx0 = bx0; c.by0 = by0;
            // load the source block, the reconstruction above / left and their modes
            for (int p = tid; p < 64 * 64; p += INT) {
                int y = by0 + p / 64, x = bx0 + p % 64;
                S->src[p] = (y < P.h && x < P.w) ? P.src[(size_t)y * P.w + x] : 0;
            }
            for (int p = tid; p < kTileW; p += INT) {
                int x = bx0 - 1 + p, y = by0 - 1;
                S->tile[p] = (y >= 0 && x >= 0 && x < P.w) ? __ldcg(&P.rec[(size_t)y * P.w + x]) : 0;
            }
            for (int p = tid; p < 64; p += INT) {
                int x = bx0 - 1, y = by0 + p;
                TL(S, p, -1) = (x >= 0 && y < P.h) ? __ldcg(&P.rec[(size_t)y * P.w + x]) : 0;
            }
            for (int p = tid; p < 17; p += INT) {
                int cx = bx0 / 4 - 1 + p, cy = by0 / 4 - 1;
                S->mm[p] = (cy >= 0 && cx >= 0 && cx < mmw) ? __ldcg(&P.mmap[(size_t)cy * mmw + cx]) : 0;
            }
            for (int p = tid; p < 16; p += INT) {
                int cx = bx0 / 4 - 1, cy = by0 / 4 + p;
                MM(S, p, -1) = (cx >= 0 && cy < mmh) ? __ldcg(&P.mmap[(size_t)cy * mmw + cx]) : 0;
            }
            uint8_t *slot = P.slots + (size_t)(r * P.cols + col) * kISlotBytes;
            if (tid == 0) {
                ISink *o = &S->out;
                for (int k = 0; k < IS_NS; ++k) { o->slen[k] = 0; o->scap[k] = c_IStreamCap[k]; o->sbuf[k] = slot + 32 + c_IStreamOff[k]; }
                int cc[CS_NUM] = {c_IStreamCap[7], c_IStreamCap[8], c_IStreamCap[9], c_IStreamCap[10], c_IStreamCap[11], 0, 0};
                cs_init(&o->c, slot + 32 + c_IStreamOff[7], cc);
            }
            __syncthreads();
            INode<0>::run(c, bx0, by0, &S->out);
            // write back the reconstruction, the mode map and the slot lengths
            for (int p = tid; p < 64 * 64; p += INT) {
                int y = by0 + p / 64, x = bx0 + p % 64;
                if (y < P.h && x < P.w) P.rec[(size_t)y * P.w + x] = TL(S, p / 64, p % 64);
            }
            for (int p = tid; p < 256; p += INT) {
                int cy = by0 / 4 + p / 16, cx = bx0 / 4 + p % 16;
                if (cy < mmh && cx < mmw) P.mmap[(size_t)cy * mmw + cx] = MM(S, p / 16, p % 16);
            }
            if (tid < 12) {
                int len = tid < IS_NS ? S->out.slen[tid] : S->out.c.len[tid - IS_NS];
                reinterpret_cast<uint16_t *>(slot)[tid] = (uint16_t)len;
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) atomicExch(&P.progress[r], col + 1);
        }
        __syncthreads();
    }
}

size_t iframe_smem_bytes() { return sizeof(IShared); }
int iframe_slot_bytes() { return kISlotBytes; }
void iframe_slot_offsets(int off[12]) { for (int k = 0; k < 12; ++k) off[k] = islot_off(k); }

}  // namespace fdvb

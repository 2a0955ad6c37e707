// Residual coding on the GPU: the 4x4 block coder with RDOQ (one warp per
// block, or two blocks per warp on half-warps; one lane per truncation
// candidate), the 8x8 transform option (one warp, or 64 threads), the
// per-8x8-region transform-size decision and its stream offsets, and the
// team-level coder of whole n x n residuals.
//
//   code_block4        fdv.h:5214-5278   (+ fdv_rdoq4x4_inner fdv.h:2493-2536)
//   8x8 option         fdv.h:5324-5377   (fdv_fdct8x8/quant8x8/dequant8x8/idct8x8 :2614-2685)
//   region decision    fdv.h:5379-5411
//   chroma_block       fdv.h:5576-5637
#pragma once
#include "common.cuh"

namespace fdvb {

// The seven coefficient streams of one candidate (fdv_cw, fdv.h:618-627):
// lengths, capacities and buffers (shared or global memory).
enum { CS_N = 0, CS_L, CS_N8, CS_L8, CS_FL, CS_NC, CS_LC, CS_NUM };
// Capacities of one P-frame macroblock candidate (luma + chroma of one MB).
constexpr int kCsCap[CS_NUM] = {16, 768, 8, 1152, 8, 8, 384};
__constant__ int c_CsCap[CS_NUM] = {16, 768, 8, 1152, 8, 8, 384};
constexpr int cs_off(int k) { int o = 0; for (int i = 0; i < k; ++i) o += kCsCap[i]; return o; }
constexpr int kCsBytes = cs_off(CS_NUM);
struct CoefSink {
    int len[CS_NUM];
    int cap[CS_NUM];
    uint8_t *buf[CS_NUM];
};
__device__ __forceinline__ uint8_t *cs_buf(const CoefSink *s, int k) { return s->buf[k]; }
__device__ __forceinline__ void cs_reset(CoefSink *s) {
    for (int k = 0; k < CS_NUM; ++k) s->len[k] = 0;
}
// Lay a sink over `mem` with the given capacities (single thread).
__device__ __forceinline__ void cs_init(CoefSink *s, uint8_t *mem, const int *caps) {
    for (int k = 0; k < CS_NUM; ++k) { s->len[k] = 0; s->cap[k] = caps[k]; s->buf[k] = mem; mem += caps[k]; }
}
// Append n bytes to stream k (single thread).
__device__ __forceinline__ void cs_put(CoefSink *s, int k, const uint8_t *b, int n, unsigned *err) {
    if (s->len[k] + n > s->cap[k]) { atomicOr(err, kErrSlotOverflow); return; }
    uint8_t *d = s->buf[k] + s->len[k];
    for (int i = 0; i < n; ++i) d[i] = b[i];
    s->len[k] += n;
}
__device__ __forceinline__ void cs_put1(CoefSink *s, int k, uint8_t v, unsigned *err) { cs_put(s, k, &v, 1, err); }

// ----------------------------------------------------- 4x4 block coder --
// Per-QP constants of the 4x4 quantiser and dequantiser (fdv.h:2430-2444,
// :2546-2555), per coefficient position, set up once per block of threads.
struct QP4 {
    int mf[16];       // MF[qp % 6][class(p)]
    int dq[16];       // DEQUANT_V[qp % 6][class(p)] << (qp / 6)
    int f, qbits;
};
__device__ __forceinline__ void qp4_setup(QP4 *q, int qp, int t) {
    if (t < 16) {
        q->mf[t] = c_MF[qp % 6][pos_class(t)];
        q->dq[t] = c_DQV[qp % 6][pos_class(t)] << (qp / 6);
    }
    if (t == 0) { q->qbits = 15 + qp / 6; q->f = (1 << (15 + qp / 6)) / 3; }
}

// Result of one 4x4 block: its end-of-block count, level bytes, squared error
// against the source after clipping, and its rate in fdv_bits_val units.
struct Blk4 {
    int count, nbytes, ssd, bits;
    uint8_t bytes[48];
};
// Per-warp scratch.
// Sixteen ints of 16-byte aligned shared scratch, four vector loads.
__device__ __forceinline__ void load16(const int *src, int v[16]) {
    const int4 *s4 = reinterpret_cast<const int4 *>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int4 a = s4[q];
        v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
    }
}
struct __align__(16) Blk4Scratch {
    int res[16];
    int lev[16];
};


// One warp codes one 4x4 block: forward transform, quantisation, optional RDOQ
// (fdv.h:2493-2536), dequantisation, inverse transform, reconstruction.  Lane
// l < 16 owns raster position l and zigzag position l; lanes 0..16 evaluate
// the RDOQ truncation candidate L = lane - 1 in parallel, their rates come
// from a suffix sum over the zigzag scan.  The reference's sequential
// selection (bestJ < 0.0 || J < bestJ, in the order L = last .. -1) is a
// warp minimum when no cost is negative and is replayed step by step
// otherwise (a rate can go negative).  Level bytes are packed in
// parallel at offsets counted from ballots of their LEB lengths.  Writes rec
// (stride rs).
// Not inlined: the key-frame quadtree reaches it from many inlined node
// levels, and one copy of its code keeps the kernels' instruction footprint
// small (key frame 26.7 -> 22.6 ms on the hd720 bands).
__device__ __noinline__ void warp_block4(const uint8_t *cur, int cs, const uint8_t *pred, int ps,
                            uint8_t *rec, int rs, const QP4 &Q, double lambda, bool rdoq,
                            Blk4 *out, Blk4Scratch *sc, int lane) {
    // Lanes 16-31 compute the same values as lanes 0-15 (every shuffle reads
    // lanes 0-15), so their stores repeat those of lanes 0-15 and no store
    // needs a lane-dependent branch.
    const int l = lane & 15, i = l >> 2, j = l & 3;
    const int cv = cur[i * cs + j], pv = pred[i * ps + j];
    const int res = cv - pv;
    int x0 = __shfl_sync(FDVB_FULL, res, i * 4 + 0), x1 = __shfl_sync(FDVB_FULL, res, i * 4 + 1);
    int x2 = __shfl_sync(FDVB_FULL, res, i * 4 + 2), x3 = __shfl_sync(FDVB_FULL, res, i * 4 + 3);
    const int t = fwd1(x0, x1, x2, x3, j);
    int y0 = __shfl_sync(FDVB_FULL, t, 0 * 4 + j), y1 = __shfl_sync(FDVB_FULL, t, 1 * 4 + j);
    int y2 = __shfl_sync(FDVB_FULL, t, 2 * 4 + j), y3 = __shfl_sync(FDVB_FULL, t, 3 * 4 + j);
    const int coef = fwd1(y0, y1, y2, y3, i);
    const int dql = Q.dq[l];
    int lev;
    {
        int sign = coef < 0 ? -1 : 1;
        long long aw = coef < 0 ? -(long long)coef : (long long)coef;
        lev = (int16_t)(sign * (int)((aw * Q.mf[l] + Q.f) >> Q.qbits));
    }
    // zigzag view: lane k holds the level at zigzag position k
    const int kz = l;
    int levz = __shfl_sync(FDVB_FULL, lev, zz4(kz));
    unsigned nzm = __ballot_sync(FDVB_FULL, lane < 16 && levz != 0);
    int last = nzm ? 31 - __clz(nzm) : -1;
    if (rdoq && last >= 0) {
        // candidate c = lane (0..16): the levels at zigzag positions < c
        // kept, the rate bits0 less 8 bits per byte of the dropped ones
        const uint32_t z = zz_enc(levz);
        const bool in = lane < 16 && kz <= last;
        const int bits0 = bits_val((uint32_t)(last + 1)) + __reduce_add_sync(FDVB_FULL, in ? bits_val(z) : 0);
        int tlen;
        const int ex = ballot_prefix(in ? leb_size(z) : 0, lane, FDVB_FULL, tlen);
        const int bitsL = bits0 - 8 * (tlen - ex);
        const unsigned vmask = 1u | (nzm << 1);
        const bool valid = lane <= 16 && ((vmask >> lane) & 1u);
        sc->res[l] = res;
        sc->lev[l] = lev * dql;          // the dequantised level
        __syncwarp();
        double J;
        {
            const int L = lane - 1;
            int d[16], r[16], rv[16];
            load16(sc->lev, d);
            load16(sc->res, rv);
#pragma unroll
            for (int p = 0; p < 16; ++p) d[p] = izz4(p) <= L ? d[p] : 0;
            idct4_thread(d, r);
            int D = 0;
#pragma unroll
            for (int p = 0; p < 16; ++p) { int e = rv[p] - r[p]; D += e * e; }
            J = valid ? rd_cost((double)D, lambda, bitsL) : 0.0;
        }
        int bestL = last;
        if (!__any_sync(FDVB_FULL, valid && J < 0.0)) {
            // every cost non-negative: the sequential rule is the minimum, ties
            // going to the first candidate in its order (the highest c).  The
            // bit patterns of non-negative doubles order like their values, so
            // the minimum is taken on the high word, then the low word.
            const unsigned long long jb = (unsigned long long)__double_as_longlong(J);
            const unsigned hi = valid ? (unsigned)(jb >> 32) : 0xffffffffu;
            const unsigned mh = __reduce_min_sync(FDVB_FULL, hi);
            const unsigned lo = (valid && hi == mh) ? (unsigned)jb : 0xffffffffu;
            const unsigned ml = __reduce_min_sync(FDVB_FULL, lo);
            const unsigned bc = 32u - __clz(__ballot_sync(FDVB_FULL, valid && hi == mh && lo == ml));
            bestL = (int)bc - 2;
        } else {
            double bestJ = -1.0;
            unsigned m = vmask;
            while (m) {                                    // uniform across the warp
                const int c = 31 - __clz(m);
                m &= ~(1u << c);
                const double Jc = __shfl_sync(FDVB_FULL, J, c);
                if (bestJ < 0.0 || Jc < bestJ) { bestJ = Jc; bestL = c - 1; }
            }
        }
        if (kz > bestL) levz = 0;
        if (izz4(l) > bestL) lev = 0;
        last = bestL;
        __syncwarp();
    }
    // reconstruct from the final levels
    const int dq = (lane < 16 ? lev : 0) * dql;
    int d0 = __shfl_sync(FDVB_FULL, dq, i * 4 + 0), d1 = __shfl_sync(FDVB_FULL, dq, i * 4 + 1);
    int d2 = __shfl_sync(FDVB_FULL, dq, i * 4 + 2), d3 = __shfl_sync(FDVB_FULL, dq, i * 4 + 3);
    int u = inv1(d0, d1, d2, d3, j);
    int e0 = __shfl_sync(FDVB_FULL, u, 0 * 4 + j), e1 = __shfl_sync(FDVB_FULL, u, 1 * 4 + j);
    int e2 = __shfl_sync(FDVB_FULL, u, 2 * 4 + j), e3 = __shfl_sync(FDVB_FULL, u, 3 * 4 + j);
    const int rr = (int16_t)((inv1(e0, e1, e2, e3, i) + 32) >> 6);
    const int r = clipb(pv + rr);
    rec[i * rs + j] = (uint8_t)r;
    const int dd = cv - r;
    // rate and level bytes, zigzag order
    const uint32_t z = zz_enc(levz);
    const bool in = lane < 16 && kz <= last;
    const int len = in ? leb_size(z) : 0;
    int nbytes;
    const int ex = ballot_prefix(len, lane, FDVB_FULL, nbytes);
    leb_put(out->bytes + ex, reinterpret_cast<uint8_t *>(sc->res) + lane, z, len);
    const int ssd = __reduce_add_sync(FDVB_FULL, lane < 16 ? dd * dd : 0);
    const int bits = bits_val((uint32_t)(last + 1)) + __reduce_add_sync(FDVB_FULL, in ? bits_val(z) : 0);
    out->count = last + 1;               // warp-uniform values
    out->nbytes = nbytes;
    out->ssd = ssd;
    out->bits = bits;
    __syncwarp();
}

// Sum of v over the 16 lanes of this lane's half-warp (two predicated warp
// reductions, independent of each other).
__device__ __forceinline__ int half_sum(int v, int lane) {
    const int lo = __reduce_add_sync(FDVB_FULL, lane < 16 ? v : 0);
    const int hi = __reduce_add_sync(FDVB_FULL, lane < 16 ? 0 : v);
    return lane < 16 ? lo : hi;
}

// Two 4x4 blocks on one warp, block h on half-warp h (lanes 16h..16h+15),
// with the same results as warp_block4 on each (fdv.h:5214-5278, RDOQ
// fdv.h:2493-2536).  In a half, lane l owns raster position l and zigzag
// position l; the RDOQ truncation candidates L = -1..14 sit on lanes 0..15 of
// the half, the candidate that keeps every level (L = 15, possible only when
// the last level is at 15) is scored from the half's lane-parallel inverse.
// The reference's choice (bestJ < 0.0 || J < bestJ over L = last .. -1) is a
// per-half minimum, ties to the highest L, when no cost is negative, and is
// replayed step by step otherwise.  sc holds two scratch entries.
__device__ void warp_block4x2(const uint8_t *cur0, const uint8_t *cur1, int cs, const uint8_t *pred0,
                              const uint8_t *pred1, int ps, uint8_t *rec0, uint8_t *rec1, int rs, const QP4 &Q,
                              double lambda, bool rdoq, Blk4 *out0, Blk4 *out1, Blk4Scratch *sc, int lane) {
    const int h = lane >> 4, hb = lane & 16, l = lane & 15, i = l >> 2, j = l & 3;
    const unsigned hmask = h ? 0xffff0000u : 0x0000ffffu;
    const uint8_t *cur = h ? cur1 : cur0, *pred = h ? pred1 : pred0;
    const int cv = cur[i * cs + j], pv = pred[i * ps + j];
    const int res = cv - pv;
    int x0 = __shfl_sync(FDVB_FULL, res, hb + i * 4 + 0), x1 = __shfl_sync(FDVB_FULL, res, hb + i * 4 + 1);
    int x2 = __shfl_sync(FDVB_FULL, res, hb + i * 4 + 2), x3 = __shfl_sync(FDVB_FULL, res, hb + i * 4 + 3);
    const int t = fwd1(x0, x1, x2, x3, j);
    int y0 = __shfl_sync(FDVB_FULL, t, hb + 0 * 4 + j), y1 = __shfl_sync(FDVB_FULL, t, hb + 1 * 4 + j);
    int y2 = __shfl_sync(FDVB_FULL, t, hb + 2 * 4 + j), y3 = __shfl_sync(FDVB_FULL, t, hb + 3 * 4 + j);
    const int coef = fwd1(y0, y1, y2, y3, i);
    int lev;
    {
        const int sign = coef < 0 ? -1 : 1;
        const long long aw = coef < 0 ? -(long long)coef : (long long)coef;
        lev = (int16_t)(sign * (int)((aw * Q.mf[l] + Q.f) >> Q.qbits));
    }
    int levz = __shfl_sync(FDVB_FULL, lev, hb + zz4(l));
    const unsigned nzm = (__ballot_sync(FDVB_FULL, levz != 0) >> hb) & 0xffffu;
    int last = nzm ? 31 - __clz(nzm) : -1;
    // the inverse of the levels as quantised (also the L = 15 candidate)
    auto inverse = [&](int lv) {
        const int dq = lv * Q.dq[l];
        const int d0 = __shfl_sync(FDVB_FULL, dq, hb + i * 4 + 0), d1 = __shfl_sync(FDVB_FULL, dq, hb + i * 4 + 1);
        const int d2 = __shfl_sync(FDVB_FULL, dq, hb + i * 4 + 2), d3 = __shfl_sync(FDVB_FULL, dq, hb + i * 4 + 3);
        const int u = inv1(d0, d1, d2, d3, j);
        const int e0 = __shfl_sync(FDVB_FULL, u, hb + 0 * 4 + j), e1 = __shfl_sync(FDVB_FULL, u, hb + 1 * 4 + j);
        const int e2 = __shfl_sync(FDVB_FULL, u, hb + 2 * 4 + j), e3 = __shfl_sync(FDVB_FULL, u, hb + 3 * 4 + j);
        return (int)(int16_t)((inv1(e0, e1, e2, e3, i) + 32) >> 6);
    };
    if (rdoq && __any_sync(FDVB_FULL, last >= 0)) {
        const uint32_t z = zz_enc(levz);
        const bool in = l <= last;
        const int bits0 = bits_val((uint32_t)(last + 1)) + half_sum(in ? bits_val(z) : 0, lane);
        int tlen;
        const int ex = ballot_prefix(in ? leb_size(z) : 0, lane, hmask, tlen);
        const int L = l - 1;
        const int bitsL = bits0 - 8 * (tlen - ex);    // the bytes of positions >= l dropped
        const unsigned vmask = 1u | (nzm << 1);           // candidate c = L + 1, c = 0..16
        const bool active = last >= 0;                      // this half truncates at all
        const bool valid = active && ((vmask >> l) & 1u);
        sc[h].res[l] = res;
        sc[h].lev[l] = lev * Q.dq[l];      // the dequantised level
        __syncwarp();
        double J;
        {   // every lane (no divergent branch); only valid candidates count
            int d[16], r[16], rv[16];
            load16(sc[h].lev, d);
            load16(sc[h].res, rv);
#pragma unroll
            for (int p = 0; p < 16; ++p) d[p] = izz4(p) <= L ? d[p] : 0;
            idct4_thread(d, r);
            int D = 0;
#pragma unroll
            for (int p = 0; p < 16; ++p) { const int e = rv[p] - r[p]; D += e * e; }
            J = valid ? rd_cost((double)D, lambda, bitsL) : 0.0;
        }
        // candidate L = 15: every level kept
        const bool v16 = active && ((vmask >> 16) & 1u);
        double J16 = 0.0;
        if (__any_sync(FDVB_FULL, v16)) {
            const int e = res - inverse(lev);
            const int D16 = half_sum(e * e, lane);
            J16 = rd_cost((double)D16, lambda, bits0);
        }
        int bestL = last;
        const bool neg = (valid && J < 0.0) || (v16 && J16 < 0.0);
        if (!__any_sync(FDVB_FULL, neg)) {
            // the minimum, ties to the highest candidate; non-negative doubles
            // order like their bit patterns
            const unsigned long long jb = (unsigned long long)__double_as_longlong(J);
            const unsigned hi = valid ? (unsigned)(jb >> 32) : 0xffffffffu;
            const unsigned mh0 = __reduce_min_sync(FDVB_FULL, h == 0 ? hi : 0xffffffffu);
            const unsigned mh1 = __reduce_min_sync(FDVB_FULL, h == 1 ? hi : 0xffffffffu);
            const unsigned mh = h ? mh1 : mh0;
            const unsigned lo = (valid && hi == mh) ? (unsigned)jb : 0xffffffffu;
            const unsigned ml0 = __reduce_min_sync(FDVB_FULL, h == 0 ? lo : 0xffffffffu);
            const unsigned ml1 = __reduce_min_sync(FDVB_FULL, h == 1 ? lo : 0xffffffffu);
            const unsigned ml = h ? ml1 : ml0;
            const unsigned ck = (valid && hi == mh && lo == ml) ? (unsigned)l + 1u : 0u;
            const unsigned bc0 = __reduce_max_sync(FDVB_FULL, h == 0 ? ck : 0u);
            const unsigned bc1 = __reduce_max_sync(FDVB_FULL, h == 1 ? ck : 0u);
            const unsigned bc = h ? bc1 : bc0;
            const double jmin = __longlong_as_double((long long)(((unsigned long long)mh << 32) | ml));
            bestL = (int)bc - 2;
            if (v16 && !(jmin < J16)) bestL = 15;
        } else {
            double bestJ = -1.0;
            for (int c = 16; c >= 0; --c) {                 // uniform across the warp
                const double Jc = c == 16 ? J16 : __shfl_sync(FDVB_FULL, J, hb + c);
                const bool vc = c == 16 ? v16 : (active && ((vmask >> c) & 1u));
                if (vc && (bestJ < 0.0 || Jc < bestJ)) { bestJ = Jc; bestL = c - 1; }
            }
        }
        if (!active) bestL = last;
        if (l > bestL) levz = 0;
        if (izz4(l) > bestL) lev = 0;
        last = bestL;
        __syncwarp();
    }
    const int rr = inverse(lev);
    const int r = clipb(pv + rr);
    (h ? rec1 : rec0)[i * rs + j] = (uint8_t)r;
    const int dd = cv - r;
    const int ssd = half_sum(dd * dd, lane);
    const uint32_t z = zz_enc(levz);
    const bool in = l <= last;
    const int bits = bits_val((uint32_t)(last + 1)) + half_sum(in ? bits_val(z) : 0, lane);
    const int len = in ? leb_size(z) : 0;
    int nbytes;
    const int ex = ballot_prefix(len, lane, hmask, nbytes);
    Blk4 *out = h ? out1 : out0;
    leb_put(out->bytes + ex, reinterpret_cast<uint8_t *>(sc[h].res) + l, z, len);
    out->count = last + 1;               // uniform over the half
    out->nbytes = nbytes;
    out->ssd = ssd;
    out->bits = bits;
    __syncwarp();
}

// ------------------------------------------------------ 8x8 transform --
struct Reg8Scratch {
    int32_t X[64];
    int32_t A[64];
    int32_t Y[64];
    int32_t L[64];
    long long B[64];
    int part[2][4];
};
struct Reg8 {
    int count, nbytes, bits;
    long long ssd;
    uint8_t rec[64];
    uint8_t bytes[192];
};

// 64 threads (t = 0..63) code one 8x8 region with the 8x8 transform: forward
// DCT in int32, quantise, dequantise (saturating to int32), inverse in int64
// with >> 36 normalisation, reconstruct; then count, rate and level bytes in
// zigzag order from ballots and prefix sums.  `bar` names a named barrier
// shared only by these 64 threads (two warps).
__device__ __forceinline__ void bar_sync64(int bar) { asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory"); }

__device__ void region8(const uint8_t *cur, int cs, const uint8_t *pred, int ps, int qp,
                        Reg8 *out, Reg8Scratch *sc, int t, int bar) {
    const int r = t >> 3, c = t & 7, lane = t & 31, w = t >> 5;
    const int cv = cur[r * cs + c], pv = pred[r * ps + c];
    sc->X[t] = cv - pv;
    bar_sync64(bar);
    {   // A[u][x] = sum_y C8[u][y] X[y][x]   (u = r, x = c)
        int32_t s = 0;
#pragma unroll
        for (int y = 0; y < 8; ++y) s += c8(r * 8 + y) * sc->X[y * 8 + c];
        sc->A[t] = s;
    }
    bar_sync64(bar);
    int32_t Yv;
    {   // Y[u][v] = sum_x A[u][x] C8[v][x]   (u = r, v = c)
        int32_t s = 0;
#pragma unroll
        for (int x = 0; x < 8; ++x) s += sc->A[r * 8 + x] * c8t(x * 8 + c);
        Yv = s;
    }
    const int32_t q = c_QSTEP8[qp], f = q / 3;
    int sign = Yv < 0 ? -1 : 1;
    int32_t a = Yv < 0 ? -Yv : Yv;
    int lev = (int16_t)(sign * ((a + f) / q));
    sc->L[t] = lev;
    long long dv = (long long)lev * q;
    sc->Y[t] = dv < INT32_MIN ? INT32_MIN : (dv > INT32_MAX ? INT32_MAX : (int32_t)dv);
    bar_sync64(bar);
    {   // B[y][v] = sum_u C8[u][y] Y[u][v]   (y = r, v = c)
        long long s = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) s += (long long)c8(u * 8 + r) * sc->Y[u * 8 + c];
        sc->B[t] = s;
    }
    bar_sync64(bar);
    int rr;
    {   // X[y][x] = (sum_v B[y][v] C8[v][x] + 2^35) >> 36   (y = r, x = c)
        long long s = 0;
#pragma unroll
        for (int v = 0; v < 8; ++v) s += sc->B[r * 8 + v] * (long long)c8(v * 8 + c);
        rr = (int16_t)((s + (1LL << 35)) >> 36);
    }
    const int rv = clipb(pv + rr);
    out->rec[t] = (uint8_t)rv;
    const int d = cv - rv;
    // zigzag view: thread k holds the level at zigzag position k
    const int lz = sc->L[zz8(t)];
    const unsigned b = __ballot_sync(FDVB_FULL, lz != 0);
    const int ssd = __reduce_add_sync(FDVB_FULL, d * d);
    if (lane == 0) { sc->part[w][0] = b ? 32 * w + 31 - __clz(b) : -1; sc->part[w][1] = ssd; }
    bar_sync64(bar);
    const int last = max(sc->part[0][0], sc->part[1][0]);
    const uint32_t z = zz_enc(lz);
    const bool in = t <= last;
    const int bsum = __reduce_add_sync(FDVB_FULL, in ? bits_val(z) : 0);
    const int len = in ? leb_size(z) : 0;
    int tot;
    const int ex = ballot_prefix(len, lane, FDVB_FULL, tot);
    if (lane == 31) { sc->part[w][2] = tot; sc->part[w][3] = bsum; }
    bar_sync64(bar);
    const int base = w ? sc->part[0][2] : 0;
    // the residual (sc->X) is no longer read: its bytes take the unused stores
    leb_put(out->bytes + base + ex, reinterpret_cast<uint8_t *>(sc->X) + t, z, len);
    if (t == 0) {
        out->count = last + 1;
        out->nbytes = sc->part[0][2] + sc->part[1][2];
        out->bits = kBitsFlag + bits_val((uint32_t)(last + 1)) + sc->part[0][3] + sc->part[1][3];
        out->ssd = (long long)sc->part[0][1] + sc->part[1][1];
    }
    bar_sync64(bar);
}

// One warp codes one 8x8 region with the 8x8 transform: the same arithmetic
// as region8 (int32 forward DCT, quantiser step QSTEP8[qp] with f = q / 3,
// dequantisation saturated to int32, int64 inverse with >> 36), lane l owning
// positions l and l + 32.  No barrier beyond the warp, so any number of warps
// of a block can run it concurrently.
struct Reg8WScratch {
    int32_t X[64];            // residual, later the dequantised coefficients
    int32_t A[64];
    int16_t L[64];
    long long B[64];
};
__device__ void warp_region8(const uint8_t *cur, int cs, const uint8_t *pred, int ps, int qp,
                             Reg8 *out, Reg8WScratch *sc, int lane) {
    const int c = lane & 7, r0 = lane >> 3, r1 = r0 + 4;
    const int cv0 = cur[r0 * cs + c], pv0 = pred[r0 * ps + c];
    const int cv1 = cur[r1 * cs + c], pv1 = pred[r1 * ps + c];
    sc->X[lane] = cv0 - pv0;
    sc->X[lane + 32] = cv1 - pv1;
    __syncwarp();
    {   // A[u][x] = sum_y C8[u][y] X[y][x]   (u = r0, r1; x = c)
        int32_t a0 = 0, a1 = 0;
#pragma unroll
        for (int y = 0; y < 8; ++y) {
            const int32_t xv = sc->X[y * 8 + c];
            a0 += c8(r0 * 8 + y) * xv;
            a1 += c8(r1 * 8 + y) * xv;
        }
        sc->A[lane] = a0;
        sc->A[lane + 32] = a1;
    }
    __syncwarp();
    {   // Y[u][v] = sum_x A[u][x] C8[v][x]   (u = r0, r1; v = c), quantise, dequantise
        int32_t y0 = 0, y1 = 0;
#pragma unroll
        for (int x = 0; x < 8; ++x) {
            const int32_t cx = c8t(x * 8 + c);
            y0 += sc->A[r0 * 8 + x] * cx;
            y1 += sc->A[r1 * 8 + x] * cx;
        }
        const int32_t q = c_QSTEP8[qp], f = q / 3;
        const int l0 = (int16_t)((y0 < 0 ? -1 : 1) * (((y0 < 0 ? -y0 : y0) + f) / q));
        const int l1 = (int16_t)((y1 < 0 ? -1 : 1) * (((y1 < 0 ? -y1 : y1) + f) / q));
        sc->L[lane] = (int16_t)l0;
        sc->L[lane + 32] = (int16_t)l1;
        const long long d0 = (long long)l0 * q, d1 = (long long)l1 * q;
        sc->X[lane] = d0 < INT32_MIN ? INT32_MIN : (d0 > INT32_MAX ? INT32_MAX : (int32_t)d0);
        sc->X[lane + 32] = d1 < INT32_MIN ? INT32_MIN : (d1 > INT32_MAX ? INT32_MAX : (int32_t)d1);
    }
    __syncwarp();
    {   // B[y][v] = sum_u C8[u][y] Yd[u][v]   (y = r0, r1; v = c)
        long long b0 = 0, b1 = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long yd = sc->X[u * 8 + c];
            b0 += (long long)c8(u * 8 + r0) * yd;
            b1 += (long long)c8(u * 8 + r1) * yd;
        }
        sc->B[lane] = b0;
        sc->B[lane + 32] = b1;
    }
    __syncwarp();
    int rv0, rv1;
    {   // X[y][x] = (sum_v B[y][v] C8[v][x] + 2^35) >> 36   (y = r0, r1; x = c)
        long long s0 = 0, s1 = 0;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const long long cc = c8(v * 8 + c);
            s0 += sc->B[r0 * 8 + v] * cc;
            s1 += sc->B[r1 * 8 + v] * cc;
        }
        rv0 = clipb(pv0 + (int16_t)((s0 + (1LL << 35)) >> 36));
        rv1 = clipb(pv1 + (int16_t)((s1 + (1LL << 35)) >> 36));
    }
    out->rec[lane] = (uint8_t)rv0;
    out->rec[lane + 32] = (uint8_t)rv1;
    const int e0 = cv0 - rv0, e1 = cv1 - rv1;
    const int ssd = __reduce_add_sync(FDVB_FULL, e0 * e0 + e1 * e1);
    // zigzag view: lane k holds zigzag positions k and k + 32
    const int lz0 = sc->L[zz8(lane)], lz1 = sc->L[zz8(lane + 32)];
    const unsigned m0 = __ballot_sync(FDVB_FULL, lz0 != 0), m1 = __ballot_sync(FDVB_FULL, lz1 != 0);
    const int last = m1 ? 63 - __clz(m1) : (m0 ? 31 - __clz(m0) : -1);
    const uint32_t z0 = zz_enc(lz0), z1 = zz_enc(lz1);
    const bool in0 = lane <= last, in1 = lane + 32 <= last;
    const int bsum = __reduce_add_sync(FDVB_FULL, (in0 ? bits_val(z0) : 0) + (in1 ? bits_val(z1) : 0));
    const int len0 = in0 ? leb_size(z0) : 0, len1 = in1 ? leb_size(z1) : 0;
    int tot0, tot1;
    const int ex0 = ballot_prefix(len0, lane, FDVB_FULL, tot0);
    const int ex1 = tot0 + ballot_prefix(len1, lane, FDVB_FULL, tot1);
    // every lane has read its levels (the ballots above): sc->L is junk now
    uint8_t *const junk = reinterpret_cast<uint8_t *>(sc->L);
    leb_put(out->bytes + ex0, junk + lane, z0, len0);
    leb_put(out->bytes + ex1, junk + 32 + lane, z1, len1);
    out->count = last + 1;               // warp-uniform values
    out->nbytes = tot0 + tot1;
    out->bits = kBitsFlag + bits_val((uint32_t)(last + 1)) + bsum;
    out->ssd = ssd;
    __syncwarp();
}

// --------------------------------------------------- residual (n x n) --
// The decision of one 8x8 region between its 4x4 option (A) and its 8x8
// option (B), with the region's byte counts in each stream.
struct RegDec {
    int choice, flv;          // 0 = four 4x4 (A), 1 = one 8x8 (B); flag byte value
    int nl, ol;               // level bytes and their offset in the level stream
    int oc, ofl;              // offsets in the count stream and the flag stream
    long long e;
    int b;
};

// The RD choice of one 8x8 region between its four 4x4 blocks (A) and its 8x8
// transform (B), with the empty-region flag value 0 (fdv.h:5379-5411).
__device__ __forceinline__ void region_choice(const Blk4 *b4, const Reg8 &R, double lambda, RegDec &D) {
    long long eA = 0;
    int bA = kBitsFlag, lpA = 0;
    for (int s = 0; s < 4; ++s) { eA += b4[s].ssd; bA += b4[s].bits; lpA += b4[s].nbytes; }
    long long eB = R.ssd;
    int bB = R.bits;
    const bool emptyA = lpA == 0, emptyB = R.count == 0;
    if (emptyA) bA = kBitsFlag;
    if (emptyB) bB = kBitsFlag;
    if (rd_cost((double)eA, lambda, bA) <= rd_cost((double)eB, lambda, bB)) {
        D.choice = 0; D.flv = emptyA ? 0 : 1; D.nl = emptyA ? 0 : lpA; D.e = eA; D.b = bA;
    } else {
        D.choice = 1; D.flv = emptyB ? 0 : 2; D.nl = emptyB ? 0 : R.nbytes; D.e = eB; D.b = bB;
    }
}

// Copy region rg's symbols (flag, counts, level bytes) to the offsets its
// decision reserved (one warp).  The four 4x4 blocks' level bytes are one
// copy over their concatenation, each byte's block found by comparing with
// the running offsets (no loop per block waiting on the previous one's size).
__device__ __forceinline__ void region_symbols(const RegDec &D, const Blk4 *b4, const Reg8 &R, CoefSink *sink,
                                               bool chroma, int lane) {
    const int flv = D.flv;
    if (flv < 0) return;
    if (lane == 0) sink->buf[CS_FL][D.ofl] = (uint8_t)flv;
    if (flv == 1) {
        uint8_t *cnt = sink->buf[chroma ? CS_NC : CS_N] + D.oc;
        uint8_t *lv = sink->buf[chroma ? CS_LC : CS_L] + D.ol;
        if (lane < 4) cnt[lane] = (uint8_t)b4[lane].count;
        const int o1 = b4[0].nbytes, o2 = o1 + b4[1].nbytes, o3 = o2 + b4[2].nbytes, tot = o3 + b4[3].nbytes;
        for (int i = lane; i < tot; i += 32) {
            const int s1 = i >= o1 ? 1 : 0, s2 = i >= o2 ? 1 : 0, s3 = i >= o3 ? 1 : 0;
            const int base = (o1 & -s1) + ((o2 - o1) & -s2) + ((o3 - o2) & -s3);
            lv[i] = b4[s1 + s2 + s3].bytes[i - base];
        }
    } else if (flv == 2) {
        if (lane == 0) sink->buf[CS_N8][D.oc] = (uint8_t)R.count;
        uint8_t *lv = sink->buf[CS_L8] + D.ol;
        for (int i = lane; i < D.nl; i += 32) lv[i] = R.bytes[i];
    }
}

// Reserve the stream offsets of regions dec[0..nreg) in order (one thread);
// on overflow report it, clamp the lengths and mark the regions unwritten.
// The five lengths a region can grow are kept in registers meanwhile.
__device__ __forceinline__ void region_offsets(RegDec *dec, int nreg, CoefSink *sink, bool chroma,
                                               long long *e, int *b, unsigned *err) {
    const int kc = chroma ? CS_NC : CS_N, kl = chroma ? CS_LC : CS_L;
    int lfl = sink->len[CS_FL], lc = sink->len[kc], ll = sink->len[kl], ln8 = sink->len[CS_N8], ll8 = sink->len[CS_L8];
    long long es = 0;
    int bs = 0;
#pragma unroll 4
    for (int rg = 0; rg < nreg; ++rg) {
        RegDec &D = dec[rg];
        const int flv = D.flv, nl = D.nl;
        D.ofl = lfl++;
        if (flv == 1) { D.oc = lc; lc += 4; D.ol = ll; ll += nl; }
        else if (flv == 2) { D.oc = ln8; ln8 += 1; D.ol = ll8; ll8 += nl; }
        es += D.e;
        bs += D.b;
    }
    const bool ovf = lfl > sink->cap[CS_FL] || lc > sink->cap[kc] || ll > sink->cap[kl] || ln8 > sink->cap[CS_N8] ||
                     ll8 > sink->cap[CS_L8];
    if (ovf) {
        atomicOr(err, kErrSlotOverflow);
        lfl = min(lfl, sink->cap[CS_FL]); lc = min(lc, sink->cap[kc]); ll = min(ll, sink->cap[kl]);
        ln8 = min(ln8, sink->cap[CS_N8]); ll8 = min(ll8, sink->cap[CS_L8]);
        for (int rg = 0; rg < nreg; ++rg) dec[rg].flv = -1;
    }
    sink->len[CS_FL] = lfl; sink->len[kc] = lc; sink->len[kl] = ll; sink->len[CS_N8] = ln8; sink->len[CS_L8] = ll8;
    *e += es;
    *b += bs;
}

// Decide regions [0, nreg) given their A results blk[4*rg..] and B results
// reg[rg], append their symbols to `sink` in region order, and leave the
// chunk's distortion and rate in e / b.  Called by all NT threads.
template <int NT>
__device__ void decide_regions(int nreg, Blk4 *blk, Reg8 *reg, RegDec *dec, double lambda, bool chroma,
                               CoefSink *sink, long long *e_out, int *b_out, unsigned *err) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < nreg) region_choice(&blk[tid * 4], reg[tid], lambda, dec[tid]);
    __syncthreads();
    if (tid == 0) {
        *e_out = 0;
        *b_out = 0;
        region_offsets(dec, nreg, sink, chroma, e_out, b_out, err);
    }
    __syncthreads();
    // one warp per region copies its flag, counts and level bytes
    for (int rg = warp; rg < nreg; rg += NT / 32) region_symbols(dec[rg], &blk[rg * 4], reg[rg], sink, chroma, lane);
}

// ---------------------------------------------- team residual coding --
// A team is NT threads (a multiple of 32) of one block that synchronise on
// their own named barrier, so several teams of a block run independently.
__device__ __forceinline__ void team_bar(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Scratch of a team: one chunk of up to TR regions, per-warp coder scratch.
template <int NW>
struct TeamResidScratch {
    static constexpr int TR = 16;
    Blk4 blk[4 * TR];
    __align__(16) uint8_t recA[TR][64];
    Reg8 reg[TR];
    RegDec dec[TR];
    Reg8WScratch r8[NW];
    Blk4Scratch b4[NW];
};

// M residuals of n x n (n in {8, 16, 32, 64}) coded at once against the same
// source cur (stride cs): prediction pred[i] (stride n), reconstruction rec[i]
// (stride n), symbols appended to sink[i], distortion e[i] and rate b[i]
// (region flags and coefficients; the caller charges the mode symbol).  Each
// residual follows code_residual (fdv.h:5300-5414): 8x8 regions in raster
// order, each the RD choice between four RDOQ'd 4x4 blocks and one 8x8
// transform.  Work goes out in chunks of TR regions, five warp tasks per
// region (four 4x4 blocks, the 8x8 option); TR is a multiple of (n/8)^2 or
// divides it, so a chunk never splits one residual's regions unevenly.
// Called by all NT threads of the team (tt = 0..NT-1) with barrier `bar`.
template <int NT, int NWS>
__device__ void team_residuals(const uint8_t *cur, int cs, uint8_t *const *pred, uint8_t *const *rec,
                               CoefSink *const *sink, int M, int n, const QP4 &Q, int qp, double lambda,
                               long long *e, int *b, TeamResidScratch<NWS> *sc, unsigned *err, int tt,
                               int bar) {
    constexpr int NW = NT / 32, TR = TeamResidScratch<NWS>::TR;
    static_assert(NW <= NWS, "scratch for every warp of the team");
    const int wt = tt >> 5, lane = tt & 31;
    const int rpl = n / 8, rpm = rpl * rpl, total = M * rpm;
    if (tt < M) { e[tt] = 0; b[tt] = 0; }
    for (int g0 = 0; g0 < total; g0 += TR) {
        const int R = min(TR, total - g0);
        for (int k = wt; k < 5 * R; k += NW) {
            const int i = k / 5, sub = k - 5 * i, g = g0 + i, m = g / rpm, rg = g - m * rpm;
            const int rx = (rg % rpl) * 8, ry = (rg / rpl) * 8;
            const uint8_t *cb = cur + ry * cs + rx, *pb = pred[m] + ry * n + rx;
            if (sub < 4) {
                const int sx = (sub & 1) * 4, sy = (sub >> 1) * 4;
                warp_block4(cb + sy * cs + sx, cs, pb + sy * n + sx, n, &sc->recA[i][sy * 8 + sx], 8, Q, lambda, true,
                            &sc->blk[4 * i + sub], &sc->b4[wt], lane);
            } else {
                warp_region8(cb, cs, pb, n, qp, &sc->reg[i], &sc->r8[wt], lane);
            }
        }
        team_bar(bar, NT);
        if (tt < R) region_choice(&sc->blk[4 * tt], sc->reg[tt], lambda, sc->dec[tt]);
        team_bar(bar, NT);
        const int seg = min(rpm, R), nseg = R / seg;
        if (tt < nseg) {
            const int m = (g0 + tt * seg) / rpm;
            region_offsets(&sc->dec[tt * seg], seg, sink[m], false, &e[m], &b[m], err);
        }
        team_bar(bar, NT);
        for (int i = wt; i < R; i += NW) {
            const int g = g0 + i, m = g / rpm, rg = g - m * rpm;
            const int rx = (rg % rpl) * 8, ry = (rg / rpl) * 8;
            const RegDec &D = sc->dec[i];
            region_symbols(D, &sc->blk[4 * i], sc->reg[i], sink[m], false, lane);
            for (int q = lane; q < 64; q += 32)
                rec[m][(ry + (q >> 3)) * n + rx + (q & 7)] = D.choice ? sc->reg[i].rec[q] : sc->recA[i][q];
        }
        team_bar(bar, NT);
    }
}

}  // namespace fdvb

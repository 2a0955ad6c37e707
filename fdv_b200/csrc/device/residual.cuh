// Residual coding on the GPU: the 4x4 block coder with RDOQ (one warp per
// block, one lane per truncation candidate), the 8x8 transform option (64
// threads per region), the per-8x8-region transform-size decision, and the
// chroma residual of SKIP/INTER macroblocks.
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
// Result of one 4x4 block: its end-of-block count, level bytes, squared error
// against the source after clipping, and its rate in fdv_bits_val units.
struct Blk4 {
    int count, nbytes, ssd, bits;
    uint8_t bytes[48];
};
// Per-warp scratch.
struct Blk4Scratch {
    int res[16];
    int lev[16];
    double J[17];
    int valid[17];
};

// One warp codes one 4x4 block: forward transform, quantisation, optional RDOQ
// (fdv.h:2493), dequantisation, inverse transform, reconstruction.  Lane l<16
// owns coefficient position l; lanes 0..16 evaluate the RDOQ truncation
// candidate L = lane-1 in parallel and lane 0 replays the reference's
// sequential selection over them.  Writes rec (uint8, stride rs) and `out`.
__device__ void warp_block4(const uint8_t *cur, int cs, const uint8_t *pred, int ps,
                            uint8_t *rec, int rs, int qp, double lambda, bool rdoq,
                            Blk4 *out, Blk4Scratch *sc, int lane) {
    const int l = lane & 15, i = l >> 2, j = l & 3;
    const int cv = cur[i * cs + j], pv = pred[i * ps + j];
    const int res = cv - pv;
    int x0 = __shfl_sync(FDVB_FULL, res, i * 4 + 0), x1 = __shfl_sync(FDVB_FULL, res, i * 4 + 1);
    int x2 = __shfl_sync(FDVB_FULL, res, i * 4 + 2), x3 = __shfl_sync(FDVB_FULL, res, i * 4 + 3);
    int t = fwd1(x0, x1, x2, x3, j);
    int y0 = __shfl_sync(FDVB_FULL, t, 0 * 4 + j), y1 = __shfl_sync(FDVB_FULL, t, 1 * 4 + j);
    int y2 = __shfl_sync(FDVB_FULL, t, 2 * 4 + j), y3 = __shfl_sync(FDVB_FULL, t, 3 * 4 + j);
    int coef = fwd1(y0, y1, y2, y3, i);
    int lev = quant4(coef, l, qp);
    const int iz = c_IZZ4[l];
    int last = __reduce_max_sync(FDVB_FULL, (lane < 16 && lev != 0) ? iz : -1);
    if (rdoq && last >= 0) {
        if (lane < 16) { sc->res[l] = res; sc->lev[l] = lev; }
        __syncwarp();
        int bv = (lane < 16 && iz <= last) ? bits_val(zz_enc(lev)) : 0;
        int bits0 = bits_val((uint32_t)(last + 1)) + __reduce_add_sync(FDVB_FULL, bv);
        const int L = lane - 1;
        bool valid = lane <= 16 && L <= last && (L < 0 || sc->lev[c_ZZ4[L]] != 0);
        if (valid) {
            int bits = bits0;
            for (int k = L + 1; k <= last; ++k) bits -= 8 * leb_size(zz_enc(sc->lev[c_ZZ4[k]]));
            int d[16], r[16];
#pragma unroll
            for (int p = 0; p < 16; ++p) d[p] = dequant4(c_IZZ4[p] <= L ? sc->lev[p] : 0, p, qp);
            idct4_thread(d, r);
            long long D = 0;
#pragma unroll
            for (int p = 0; p < 16; ++p) { int e = sc->res[p] - r[p]; D += (long long)e * e; }
            sc->J[lane] = rd_cost((double)D, lambda, bits);
        }
        if (lane <= 16) sc->valid[lane] = valid;
        __syncwarp();
        int bestL = last;
        if (lane == 0) {
            double bestJ = -1.0;
            for (int Lc = last; Lc >= -1; --Lc) {
                if (!sc->valid[Lc + 1]) continue;
                double J = sc->J[Lc + 1];
                if (bestJ < 0.0 || J < bestJ) { bestJ = J; bestL = Lc; }
            }
        }
        bestL = __shfl_sync(FDVB_FULL, bestL, 0);
        if (iz > bestL) lev = 0;
        last = bestL;
        __syncwarp();
    }
    // Reconstruct from the final levels.
    int dq = dequant4(lane < 16 ? lev : 0, l, qp);
    int d0 = __shfl_sync(FDVB_FULL, dq, i * 4 + 0), d1 = __shfl_sync(FDVB_FULL, dq, i * 4 + 1);
    int d2 = __shfl_sync(FDVB_FULL, dq, i * 4 + 2), d3 = __shfl_sync(FDVB_FULL, dq, i * 4 + 3);
    int u = inv1(d0, d1, d2, d3, j);
    int e0 = __shfl_sync(FDVB_FULL, u, 0 * 4 + j), e1 = __shfl_sync(FDVB_FULL, u, 1 * 4 + j);
    int e2 = __shfl_sync(FDVB_FULL, u, 2 * 4 + j), e3 = __shfl_sync(FDVB_FULL, u, 3 * 4 + j);
    int rr = (int16_t)((inv1(e0, e1, e2, e3, i) + 32) >> 6);
    int r = clipb(pv + rr);
    if (lane < 16) rec[i * rs + j] = (uint8_t)r;
    int dd = cv - r;
    int ssd = __reduce_add_sync(FDVB_FULL, lane < 16 ? dd * dd : 0);
    uint32_t z = zz_enc(lev);
    int bl = (lane < 16 && iz <= last) ? bits_val(z) : 0;
    int bits = bits_val((uint32_t)(last + 1)) + __reduce_add_sync(FDVB_FULL, bl);
    // Level bytes in zigzag order: each lane knows its LEB length; lane 0 packs.
    if (lane < 16) sc->lev[l] = lev;
    __syncwarp();
    if (lane == 0) {
        int nb = 0;
        for (int k = 0; k <= last; ++k) nb += leb_write(out->bytes + nb, zz_enc(sc->lev[c_ZZ4[k]]));
        out->count = last + 1;
        out->nbytes = nb;
        out->ssd = ssd;
        out->bits = bits;
    }
    __syncwarp();
}

// ------------------------------------------------------ 8x8 transform --
struct Reg8Scratch {
    int32_t X[64];
    int32_t A[64];
    int32_t Y[64];
    int32_t L[64];
    long long B[64];
    int ssd_part[2];
};
struct Reg8 {
    int count, nbytes, bits;
    long long ssd;
    uint8_t rec[64];
    uint8_t bytes[192];
};

// 64 threads (t = 0..63) code one 8x8 region with the 8x8 transform: forward
// DCT in int32, quantise, dequantise (saturating to int32), inverse in int64
// with >> 36 normalisation, reconstruct.  `bar` names a named barrier shared
// only by these 64 threads (two warps).
__device__ __forceinline__ void bar_sync64(int bar) { asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory"); }

__device__ void region8(const uint8_t *cur, int cs, const uint8_t *pred, int ps, int qp,
                        Reg8 *out, Reg8Scratch *sc, int t, int bar) {
    const int r = t >> 3, c = t & 7;
    const int cv = cur[r * cs + c], pv = pred[r * ps + c];
    sc->X[t] = cv - pv;
    bar_sync64(bar);
    {   // A[u][x] = sum_y C8[u][y] X[y][x]   (u = r, x = c)
        int32_t s = 0;
#pragma unroll
        for (int y = 0; y < 8; ++y) s += c_C8[r * 8 + y] * sc->X[y * 8 + c];
        sc->A[t] = s;
    }
    bar_sync64(bar);
    int32_t Yv;
    {   // Y[u][v] = sum_x A[u][x] C8[v][x]   (u = r, v = c)
        int32_t s = 0;
#pragma unroll
        for (int x = 0; x < 8; ++x) s += sc->A[r * 8 + x] * c_C8[c * 8 + x];
        Yv = s;
    }
    int32_t q = c_QSTEP8[qp], f = q / 3;
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
        for (int u = 0; u < 8; ++u) s += (long long)c_C8[u * 8 + r] * sc->Y[u * 8 + c];
        sc->B[t] = s;
    }
    bar_sync64(bar);
    int rr;
    {   // X[y][x] = (sum_v B[y][v] C8[v][x] + 2^35) >> 36   (y = r, x = c)
        long long s = 0;
#pragma unroll
        for (int v = 0; v < 8; ++v) s += sc->B[r * 8 + v] * (long long)c_C8[v * 8 + c];
        rr = (int16_t)((s + (1LL << 35)) >> 36);
    }
    int rv = clipb(pv + rr);
    out->rec[t] = (uint8_t)rv;
    int d = cv - rv;
    int ssd = __reduce_add_sync(FDVB_FULL, d * d);
    if ((t & 31) == 0) sc->ssd_part[t >> 5] = ssd;
    bar_sync64(bar);
    if (t == 0) {
        int last1 = 0;
        for (int k = 0; k < 64; ++k) if (sc->L[c_ZZ8[k]] != 0) last1 = k + 1;
        int nb = 0, bits = kBitsFlag + bits_val((uint32_t)last1);
        for (int k = 0; k < last1; ++k) {
            uint32_t z = zz_enc(sc->L[c_ZZ8[k]]);
            nb += leb_write(out->bytes + nb, z);
            bits += bits_val(z);
        }
        out->count = last1;
        out->nbytes = nb;
        out->bits = bits;
        out->ssd = (long long)sc->ssd_part[0] + sc->ssd_part[1];
    }
    bar_sync64(bar);
}

// --------------------------------------------------- residual (n x n) --
// Scratch for one chunk of up to NT/64 8x8 regions of a code_residual call.
template <int NT>
struct ResidScratchT {
    static constexpr int RMAX = NT / 64, NW = NT / 32;
    Blk4 blk[4 * RMAX];
    uint8_t recA[RMAX][64];
    Reg8 reg[RMAX];
    Reg8Scratch r8[RMAX];
    Blk4Scratch b4[NW];
    int choice[RMAX];
    long long e;
    int b;
};
using ResidScratch = ResidScratchT<256>;

// The whole block (NT threads) codes an n x n residual, n in {8, 16, 32, 64}:
// per aligned 8x8 region, in raster order, the RD choice between four RDOQ'd
// 4x4 transforms and one 8x8 transform, with the 3-valued region flag
// (fdv.h:5300-5414).  Regions are processed NT/64 at a time: every 4x4 block
// of the chunk on its own warp, every region's 8x8 option on 64 threads, then
// the decisions in order.  cur has stride cs, pred and rec stride ps / rs.
// Appends to `sink` (4x4 symbols to the chroma streams when `chroma`),
// returns the distortion and adds the rate to *bits (uniform on return).
template <int NT>
__device__ long long code_residual_t(const uint8_t *cur, int cs, const uint8_t *pred, int ps, int n, int qp,
                                     double lambda, bool chroma, uint8_t *rec, int rs, CoefSink *sink,
                                     int *bits, ResidScratchT<NT> *sc, unsigned *err) {
    constexpr int RMAX = NT / 64, NW = NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rpl = n / 8, nreg_total = rpl * rpl;
    long long etot = 0;
    int btot = 0;
    for (int r0 = 0; r0 < nreg_total; r0 += RMAX) {
        const int nreg = min(RMAX, nreg_total - r0), nblk = nreg * 4;
        for (int b = warp; b < nblk; b += NW) {
            int rg = b >> 2, s = b & 3, gr = r0 + rg;
            int rx = (gr % rpl) * 8, ry = (gr / rpl) * 8, sx = (s & 1) * 4, sy = (s >> 1) * 4;
            warp_block4(cur + (ry + sy) * cs + rx + sx, cs, pred + (ry + sy) * ps + rx + sx, ps,
                        &sc->recA[rg][sy * 8 + sx], 8, qp, lambda, true, &sc->blk[b], &sc->b4[warp], lane);
        }
        if (tid < nreg * 64) {
            int rg = tid >> 6, gr = r0 + rg, rx = (gr % rpl) * 8, ry = (gr / rpl) * 8;
            region8(cur + ry * cs + rx, cs, pred + ry * ps + rx, ps, qp, &sc->reg[rg], &sc->r8[rg], tid & 63, 1 + rg);
        }
        __syncthreads();
        if (tid == 0) {
            long long e = 0;
            int b = 0;
            for (int rg = 0; rg < nreg; ++rg) {
                long long eA = 0;
                int bA = kBitsFlag, lpA = 0;
                for (int s = 0; s < 4; ++s) { eA += sc->blk[rg * 4 + s].ssd; bA += sc->blk[rg * 4 + s].bits; lpA += sc->blk[rg * 4 + s].nbytes; }
                const Reg8 &R = sc->reg[rg];
                long long eB = R.ssd;
                int bB = R.bits;
                bool emptyA = lpA == 0, emptyB = R.count == 0;
                if (emptyA) bA = kBitsFlag;
                if (emptyB) bB = kBitsFlag;
                if (rd_cost((double)eA, lambda, bA) <= rd_cost((double)eB, lambda, bB)) {
                    if (emptyA) cs_put1(sink, CS_FL, 0, err);
                    else {
                        cs_put1(sink, CS_FL, 1, err);
                        for (int s = 0; s < 4; ++s) {
                            const Blk4 &B4 = sc->blk[rg * 4 + s];
                            cs_put1(sink, chroma ? CS_NC : CS_N, (uint8_t)B4.count, err);
                            cs_put(sink, chroma ? CS_LC : CS_L, B4.bytes, B4.nbytes, err);
                        }
                    }
                    sc->choice[rg] = 0;
                    e += eA; b += bA;
                } else {
                    if (emptyB) cs_put1(sink, CS_FL, 0, err);
                    else {
                        cs_put1(sink, CS_FL, 2, err);
                        cs_put1(sink, CS_N8, (uint8_t)R.count, err);
                        cs_put(sink, CS_L8, R.bytes, R.nbytes, err);
                    }
                    sc->choice[rg] = 1;
                    e += eB; b += bB;
                }
            }
            sc->e = e;
            sc->b = b;
        }
        __syncthreads();
        for (int p = tid; p < nreg * 64; p += NT) {
            int rg = p >> 6, q = p & 63, gr = r0 + rg;
            int y = (gr / rpl) * 8 + (q >> 3), x = (gr % rpl) * 8 + (q & 7);
            rec[y * rs + x] = sc->choice[rg] ? sc->reg[rg].rec[q] : sc->recA[rg][q];
        }
        etot += sc->e;
        btot += sc->b;
        __syncthreads();
    }
    *bits += btot;
    return etot;
}

// The P-frame kernel's form: 256 threads, n in {8, 16}, pred and rec stride n.
__device__ __forceinline__ long long code_residual(const uint8_t *cur, int cs, const uint8_t *pred, int n, int qp,
                                                   double lambda, bool chroma, uint8_t *rec, CoefSink *sink,
                                                   int *bits, ResidScratch *sc, unsigned *err) {
    return code_residual_t<256>(cur, cs, pred, n, n, qp, lambda, chroma, rec, n, sink, bits, sc, err);
}

// A single 4x4 residual (n == 4, the chroma quadrants of INTER8): one warp.
// The caller arranges for exactly one warp to call this.
__device__ long long code_residual4_warp(const uint8_t *cur, int cs, const uint8_t *pred, int qp,
                                         double lambda, uint8_t *rec, Blk4 *out, Blk4Scratch *sc, int lane) {
    warp_block4(cur, cs, pred, 4, rec, 4, qp, lambda, true, out, sc, lane);
    return out->ssd;
}

}  // namespace fdvb

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
// Inside a macroblock the 256 threads run the reference's decision procedure
// (pframe_encode, fdv.h:5808-6162) with its trials parallelised: the SKIP
// candidates' predictions, each motion search step's candidate vectors, the
// sixteen 4x4 blocks and four 8x8 regions of a residual, the RDOQ truncation
// candidates, the four intra sub-modes' SATD screens.  Decisions are made on
// shared values with the reference's comparison operators and order.
#include "common.cuh"
#include "engine_dev.cuh"
#include "inter.cuh"
#include "intra.cuh"
#include "residual.cuh"

namespace fdvb {

struct PShared {
    uint8_t cur[256], curc[2][64];
    uint8_t top[16], left[16];
    uint8_t predS[3][256];
    uint8_t pr[256];
    uint8_t recI[2][256];
    uint8_t predI[4][256];
    uint8_t recIn[256];
    uint8_t pred8[4][64];
    uint8_t rec8[4][64];
    uint8_t cpred[2][64];
    uint8_t crec[2][64];
    uint8_t cpred4[8][16];
    uint8_t ctop[2][8], cleft[2][8];
    uint8_t isS[2][12];       // inter16 structure bytes per ping-pong slot
    uint8_t p8S[20];
    CoefSink sink[4];         // 0/1 inter16 ping-pong, 2 intra, 3 inter8
    uint8_t sinkmem[4][kCsBytes];
    ResidScratch rs;
    Blk4 cblk[8];
    int s_sad[8];
    int satd[64];
    int ssd3[3];
    // macroblock state (written by thread 0, read by all after a barrier)
    MBInfo cand[3];
    int ncand, tl, ht, hl, ctl[2];
    int task, row_ok;
};

__device__ __forceinline__ uint8_t ldcg8(const uint8_t *p) { return __ldcg(p); }

__device__ void write_slot_structs(uint8_t *slot, int k, const uint8_t *b, int n, unsigned *err) {
    uint16_t *len = slot_len(slot);
    if (len[k] + n > c_SlotCap[k]) { atomicOr(err, kErrSlotOverflow); return; }
    uint8_t *d = slot_data(slot, k) + len[k];
    for (int i = 0; i < n; ++i) d[i] = b[i];
    len[k] = (uint16_t)(len[k] + n);
}

__global__ void __launch_bounds__(256, 1)
pframe_kernel(const UnitDev *__restrict__ units, const RowTask *__restrict__ rows, int nrows,
              int *ticket, unsigned *err, unsigned long long wait_ns) {
    __shared__ PShared S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < 4) cs_init(&S.sink[tid], S.sinkmem[tid], c_CsCap);
    __syncthreads();
    for (;;) {
        if (tid == 0) S.task = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = S.task;
        __syncthreads();
        if (t >= nrows) return;
        const UnitDev &U = units[rows[t].unit];
        const int row = rows[t].row, w = U.w, cw = w / 2, mbw = U.mbw;
        if (row == U.stall_row) continue;   // injected stall: this row's progress flag is never set
        const double lambda = U.lambda;
        const int qp = U.qp, R = U.range;
        const double lam14 = __dmul_rn(lambda, 14.0), lam16 = __dmul_rn(lambda, 16.0), lam19 = __dmul_rn(lambda, 19.0);
        int pmvx = 0, pmvy = 0;
        for (int mbx = 0; mbx < mbw; ++mbx) {
            const int bx = mbx * 16, by = row * 16, cbx = bx / 2, cby = by / 2;
            if (row > 0) {
                if (tid == 0) S.row_ok = wait_at_least(&U.progress[row - 1], min(mbx + 2, mbw), err, wait_ns);
            } else if (tid == 0) S.row_ok = 1;
            __syncthreads();
            if (!S.row_ok) break;
            uint8_t *slot = U.slots + (size_t)(row * mbw + mbx) * kSlotBytes;
            if (tid < 16) slot_len(slot)[tid] = 0;
            // ---- load the macroblock and its current-frame neighbours
            for (int p = tid; p < 256; p += 256) S.cur[p] = U.cur[0][(size_t)(by + (p >> 4)) * w + bx + (p & 15)];
            if (tid < 128) {
                int pl = tid >> 6, p = tid & 63;
                S.curc[pl][p] = U.cur[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)];
            }
            if (tid < 16) {
                S.top[tid] = by > 0 ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx + tid]) : 0;
                S.left[tid] = bx > 0 ? ldcg8(&U.rec[0][(size_t)(by + tid) * w + bx - 1]) : 0;
            } else if (tid < 32) {
                int k = tid - 16, pl = k >> 3, q = k & 7;
                S.ctop[pl][q] = cby > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx + q]) : 0;
                S.cleft[pl][q] = cbx > 0 ? ldcg8(&U.rec[1 + pl][(size_t)(cby + q) * cw + cbx - 1]) : 0;
            }
            if (tid == 0) {
                S.ht = by > 0; S.hl = bx > 0;
                S.tl = (by > 0 && bx > 0) ? ldcg8(&U.rec[0][(size_t)(by - 1) * w + bx - 1]) : 128;
                for (int pl = 0; pl < 2; ++pl)
                    S.ctl[pl] = (cby > 0 && cbx > 0) ? ldcg8(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx - 1]) : 128;
                // merge candidates (fdv.h:5711-5729)
                int n = 0;
                S.cand[0].x = (int16_t)pmvx; S.cand[0].y = (int16_t)pmvy; S.cand[0].ref = 0; S.cand[0].inter = 1; n = 1;
                for (int k = 0; k < 2 && n < 3; ++k) {
                    int cx = mbx + k, cy = row - 1;
                    if (cy < 0 || cx >= mbw) continue;
                    const MBInfo *mp = &U.mbi[cy * mbw + cx];
                    MBInfo m;
                    m.x = (int16_t)__ldcg(&mp->x); m.y = (int16_t)__ldcg(&mp->y);
                    m.ref = ldcg8(&mp->ref); m.inter = ldcg8(&mp->inter);
                    if (!m.inter) continue;
                    bool dup = false;
                    for (int j2 = 0; j2 < n; ++j2)
                        if (S.cand[j2].x == m.x && S.cand[j2].y == m.y && S.cand[j2].ref == m.ref) dup = true;
                    if (!dup) S.cand[n++] = m;
                }
                S.ncand = n;
            }
            __syncthreads();
            // mode context (fdv.h:4172): left / above macroblock skipped-ness
            int ctx = 0;
            {
                int Lm = mbx > 0 ? ldcg8(&U.mbi[row * mbw + mbx - 1].mode) : 0;
                int Am = row > 0 ? ldcg8(&U.mbi[(row - 1) * mbw + mbx].mode) : 0;
                ctx = (Lm != 0 ? 2 : 0) + (Am != 0 ? 1 : 0);
            }
            const RefPlanes &R0 = U.ref[0];
            if (U.force_skip) {
                // A held frame: SKIP with the zero vector everywhere (fdv.h:5820-5836).
                for (int p = tid; p < 256; p += 256)
                    U.rec[0][(size_t)(by + (p >> 4)) * w + bx + (p & 15)] = R0.G[(long)(by + (p >> 4)) * R0.ys + bx + (p & 15)];
                if (tid < 128) {
                    int pl = tid >> 6, p = tid & 63;
                    const uint8_t *P = pl ? R0.V : R0.U;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = P[(long)(cby + (p >> 3)) * R0.cs + cbx + (p & 7)];
                }
                if (tid == 0) {
                    uint8_t m0 = 0;
                    write_slot_structs(slot, ctx, &m0, 1, err);
                    MBInfo mi = {0, 0, 0, 1, 0, 0};
                    U.mbi[row * mbw + mbx] = mi;
                }
                pmvx = 0; pmvy = 0;
                __threadfence();
                __syncthreads();
                if (tid == 0) atomicExch(&U.progress[row], mbx + 1);
                continue;
            }
            const int ncand = S.ncand;
            // ---- SKIP: merge candidates (fdv.h:5843-5899)
            for (int p = tid; p < ncand * 256; p += 256) {
                int mi = p >> 8, q = p & 255;
                const MBInfo &c = S.cand[mi];
                int ph = (c.y & 3) * 4 + (c.x & 3);
                S.predS[mi][q] = (uint8_t)mc_px(U.ref[c.ref], bx + (q & 15) + (c.x >> 2), by + (q >> 4) + (c.y >> 2), ph);
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
            double Jbest = Js;
            const bool skip_wins = Js <= lam14;

            // ---- INTER16 over the available references (fdv.h:5901-5943)
            int mvx = 0, mvy = 0, best_ref = 0, sad16 = 0, best_slot = -1, is_len[2] = {0, 0};
            double Ji = 1e30;
            for (int r = 0; r < U.navail && !skip_wins; ++r) {
                if (r > 0 && Jbest <= lam16) break;
                const RefPlanes &Rr = U.ref[r];
                int rmx, rmy;
                int rsad = me_search(S.cur, 16, Rr, bx, by, 16, 16, R, pmvx, pmvy, &rmx, &rmy, S.s_sad);
                {
                    int ph = (rmy & 3) * 4 + (rmx & 3);
                    int q = tid;
                    S.pr[q] = (uint8_t)mc_px(Rr, bx + (q & 15) + (rmx >> 2), by + (q >> 4) + (rmy >> 2), ph);
                }
                const int ts = best_slot == 0 ? 1 : 0;
                if (tid == 0) {
                    cs_reset(&S.sink[ts]);
                    uint8_t *b = S.isS[ts];
                    int n = 0;
                    b[n++] = (uint8_t)r;
                    n += leb_write(b + n, zz_enc(rmx - pmvx));
                    n += leb_write(b + n, zz_enc(rmy - pmvy));
                    is_len[ts] = n;
                    S.ssd3[0] = n;
                }
                __syncthreads();
                is_len[ts] = S.ssd3[0];
                int bb = 2 * kBitsMode + bits_val(zz_enc(rmx - pmvx)) + bits_val(zz_enc(rmy - pmvy));
                long long dd = code_residual(S.cur, 16, S.pr, 16, qp, lambda, false, S.recI[ts], &S.sink[ts], &bb, &S.rs, err);
                double J = rd_cost((double)dd, lambda, bb);
                if (J < Jbest) Jbest = J;
                if (J < Ji) { Ji = J; best_ref = r; mvx = rmx; mvy = rmy; sad16 = rsad; best_slot = ts; }
            }

            // ---- INTRA 16x16, SATD-screened (fdv.h:5945-5988)
            double Jintra = 1e30;
            int best_sub = 0;
            if (!skip_wins && Jbest > lam14) {
                __shared__ NNPred s_nn[4];
                if (tid < 4) s_nn[tid] = nn_setup(tid, S.top, S.left, S.tl, 16, S.ht, S.hl);
                __syncthreads();
                for (int p = tid; p < 4 * 256; p += 256) {
                    int m = p >> 8, q = p & 255;
                    S.predI[m][q] = (uint8_t)nn_px(s_nn[m], S.top, S.left, q & 15, q >> 4);
                }
                __syncthreads();
                if (tid < 64) {
                    int m = tid >> 4, b = tid & 15, oy = (b >> 2) * 4, ox = (b & 3) * 4;
                    S.satd[tid] = satd4(S.cur + oy * 16 + ox, 16, S.predI[m] + oy * 16 + ox, 16);
                }
                __syncthreads();
                int sel = -1, sbest = 0;
                for (int m = 0; m < 4; ++m) {
                    if (!nn_mode_ok(m, 16, S.ht, S.hl)) continue;
                    int sa = 0;
                    for (int b = 0; b < 16; ++b) sa += S.satd[m * 16 + b];
                    if (sel < 0 || sa < sbest) { sbest = sa; sel = m; }
                }
                if (sel >= 0) {
                    if (tid == 0) cs_reset(&S.sink[2]);
                    __syncthreads();
                    int bn = 2 * kBitsMode;
                    long long Dn = code_residual(S.cur, 16, S.predI[sel], 16, qp, lambda, false, S.recIn, &S.sink[2], &bn, &S.rs, err);
                    Jintra = rd_cost((double)Dn, lambda, bn);
                    best_sub = sel;
                    if (Jintra < Jbest) Jbest = Jintra;
                }
            }

            // ---- INTER8: four chained quadrant searches on the nearest reference (fdv.h:5990-6033)
            int qmv[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
            long long D8 = 0;
            int b8 = kBitsMode, p8len = 0;
            bool try8 = !skip_wins && Jbest > lam19;
            if (try8) {
                int ssad = 0, qpx = pmvx, qpy = pmvy;
                for (int q = 0; q < 4; ++q) {
                    int qx = (q & 1) * 8, qy = (q >> 1) * 8, mx, my;
                    ssad += me_search(S.cur + qy * 16 + qx, 16, R0, bx + qx, by + qy, 8, 8, R, qpx, qpy, &mx, &my, S.s_sad);
                    qmv[q][0] = mx; qmv[q][1] = my; qpx = mx; qpy = my;
                }
                if (sad16 > 0 && ssad * 10 >= sad16 * 9) try8 = false;
                if (try8) {
                    if (tid == 0) {
                        cs_reset(&S.sink[3]);
                        int n = 0, px = pmvx, py = pmvy;
                        for (int q = 0; q < 4; ++q) {
                            n += leb_write(S.p8S + n, zz_enc(qmv[q][0] - px));
                            n += leb_write(S.p8S + n, zz_enc(qmv[q][1] - py));
                            px = qmv[q][0]; py = qmv[q][1];
                        }
                        S.ssd3[0] = n;
                    }
                    {
                        int q = tid >> 6, p = tid & 63, qx = (q & 1) * 8, qy = (q >> 1) * 8;
                        int mx = qmv[q][0], my = qmv[q][1], ph = (my & 3) * 4 + (mx & 3);
                        S.pred8[q][p] = (uint8_t)mc_px(R0, bx + qx + (p & 7) + (mx >> 2), by + qy + (p >> 3) + (my >> 2), ph);
                    }
                    __syncthreads();
                    p8len = S.ssd3[0];
                    int px = pmvx, py = pmvy;
                    for (int q = 0; q < 4; ++q) {
                        int qx = (q & 1) * 8, qy = (q >> 1) * 8;
                        b8 += bits_val(zz_enc(qmv[q][0] - px)) + bits_val(zz_enc(qmv[q][1] - py));
                        px = qmv[q][0]; py = qmv[q][1];
                        D8 += code_residual(S.cur + qy * 16 + qx, 16, S.pred8[q], 8, qp, lambda, false, S.rec8[q], &S.sink[3], &b8, &S.rs, err);
                    }
                }
            }
            const double J8 = try8 ? rd_cost((double)D8, lambda, b8) : 1e30;

            // ---- commit the cheapest (fdv.h:6035-6160)
            double Jmin = Js;
            int chosen = 0;
            if (Ji < Jmin) { Jmin = Ji; chosen = 1; }
            if (Jintra < Jmin) { Jmin = Jintra; chosen = 2; }
            if (J8 < Jmin) { Jmin = J8; chosen = 3; }
            __syncthreads();

            CoefSink *M = chosen == 1 ? &S.sink[best_slot] : (chosen == 2 ? &S.sink[2] : &S.sink[3]);
            MBInfo info = {0, 0, 0, 0, (uint8_t)chosen, 0};
            if (chosen == 0) {
                const int smvx = S.cand[best_mi].x, smvy = S.cand[best_mi].y, sref = S.cand[best_mi].ref;
                if (tid == 0) {
                    uint8_t m0 = 0, mi = (uint8_t)best_mi;
                    write_slot_structs(slot, ctx, &m0, 1, err);
                    if (ncand > 1) write_slot_structs(slot, PS_MERGE, &mi, 1, err);
                }
                U.rec[0][(size_t)(by + (tid >> 4)) * w + bx + (tid & 15)] = S.predS[best_mi][tid];
                if (tid < 128) {
                    int pl = tid >> 6, p = tid & 63;
                    const RefPlanes &Rs = U.ref[sref];
                    int cmx = smvx / 2, cmy = smvy / 2;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] =
                        (uint8_t)mc_cpx(pl ? Rs.V : Rs.U, Rs.cs, cbx + (p & 7) + (cmx >> 2), cby + (p >> 3) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                info.x = (int16_t)smvx; info.y = (int16_t)smvy; info.ref = (uint8_t)sref; info.inter = 1;
                pmvx = smvx; pmvy = smvy;
            } else if (chosen == 1) {
                if (tid == 0) {
                    uint8_t m1 = 1;
                    write_slot_structs(slot, ctx, &m1, 1, err);
                    const uint8_t *b = S.isS[best_slot];
                    write_slot_structs(slot, PS_REF, b, 1, err);
                    int part = 0;
                    for (int q = 1; q < is_len[best_slot]; ++q) {
                        write_slot_structs(slot, part ? PS_MVY : PS_MVX, b + q, 1, err);
                        if (!(b[q] & 0x80)) ++part;
                    }
                }
                U.rec[0][(size_t)(by + (tid >> 4)) * w + bx + (tid & 15)] = S.recI[best_slot][tid];
                // chroma INTER: prediction at mv/2, four 4x4 blocks per plane, no RDOQ (fdv.h:5576-5626)
                const RefPlanes &Rb = U.ref[best_ref];
                const int cmx = mvx / 2, cmy = mvy / 2;
                if (tid < 128) {
                    int pl = tid >> 6, p = tid & 63;
                    S.cpred[pl][p] = (uint8_t)mc_cpx(pl ? Rb.V : Rb.U, Rb.cs, cbx + (p & 7) + (cmx >> 2), cby + (p >> 3) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                __syncthreads();
                {
                    int pl = warp >> 2, b = warp & 3, oy = (b >> 1) * 4, ox = (b & 1) * 4;
                    warp_block4(S.curc[pl] + oy * 8 + ox, 8, S.cpred[pl] + oy * 8 + ox, 8, S.crec[pl] + oy * 8 + ox, 8,
                                qp, lambda, false, &S.cblk[warp], &S.rs.b4[warp], lane);
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
                    int pl = tid >> 6, p = tid & 63;
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
                U.rec[0][(size_t)(by + (tid >> 4)) * w + bx + (tid & 15)] = S.recIn[tid];
                // chroma intra with the same sub-mode, through the residual coder (fdv.h:6104-6117)
                for (int pl = 0; pl < 2; ++pl) {
                    __shared__ NNPred s_cn;
                    if (tid == 0) s_cn = nn_setup(best_sub, S.ctop[pl], S.cleft[pl], S.ctl[pl], 8, cby > 0, cbx > 0);
                    __syncthreads();
                    if (tid < 64) S.cpred[pl][tid] = (uint8_t)nn_px(s_cn, S.ctop[pl], S.cleft[pl], tid & 7, tid >> 3);
                    __syncthreads();
                    int bb = 0;
                    code_residual(S.curc[pl], 8, S.cpred[pl], 8, qp, lambda, true, S.crec[pl], M, &bb, &S.rs, err);
                    if (tid < 64) U.rec[1 + pl][(size_t)(cby + (tid >> 3)) * cw + cbx + (tid & 7)] = S.crec[pl][tid];
                }
                info.inter = 0;
            } else {
                if (tid == 0) {
                    uint8_t m3 = 3;
                    write_slot_structs(slot, ctx, &m3, 1, err);
                    int part = 0;
                    for (int q = 0; q < p8len; ++q) {
                        write_slot_structs(slot, (part & 1) ? PS_MVY : PS_MVX, S.p8S + q, 1, err);
                        if (!(S.p8S[q] & 0x80)) ++part;
                    }
                }
                {
                    int q = tid >> 6, p = tid & 63, qx = (q & 1) * 8, qy = (q >> 1) * 8;
                    U.rec[0][(size_t)(by + qy + (p >> 3)) * w + bx + qx + (p & 7)] = S.rec8[q][p];
                }
                // chroma: 4x4 per quadrant at qmv/2 from the nearest reference, RDOQ'd (fdv.h:6143-6159)
                if (tid < 128) {
                    int k = tid >> 4, p = tid & 15, pl = k >> 2, q = k & 3;
                    int cmx = qmv[q][0] / 2, cmy = qmv[q][1] / 2, qcx = (q & 1) * 4, qcy = (q >> 1) * 4;
                    S.cpred4[k][p] = (uint8_t)mc_cpx(pl ? R0.V : R0.U, R0.cs, cbx + qcx + (p & 3) + (cmx >> 2),
                                                     cby + qcy + (p >> 2) + (cmy >> 2), cmx & 3, cmy & 3);
                }
                __syncthreads();
                {
                    int pl = warp >> 2, q = warp & 3, qcx = (q & 1) * 4, qcy = (q >> 1) * 4;
                    warp_block4(S.curc[pl] + qcy * 8 + qcx, 8, S.cpred4[warp], 4, S.crec[pl] + qcy * 8 + qcx, 8,
                                qp, lambda, true, &S.cblk[warp], &S.rs.b4[warp], lane);
                }
                __syncthreads();
                if (tid == 0) {
                    for (int k = 0; k < 8; ++k) {
                        cs_put1(M, CS_NC, (uint8_t)S.cblk[k].count, err);
                        cs_put(M, CS_LC, S.cblk[k].bytes, S.cblk[k].nbytes, err);
                    }
                }
                if (tid < 128) {
                    int pl = tid >> 6, p = tid & 63;
                    U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = S.crec[pl][p];
                }
                info.x = (int16_t)qmv[3][0]; info.y = (int16_t)qmv[3][1]; info.ref = 0; info.inter = 1;
                pmvx = qmv[3][0]; pmvy = qmv[3][1];
            }
            __syncthreads();
            // ---- coefficient streams of the chosen mode into the slot
            if (chosen != 0) {
                for (int k = 0; k < CS_NUM; ++k) {
                    int n = M->len[k];
                    if (n > c_SlotCap[PS_CN + k]) { if (tid == 0) atomicOr(err, kErrSlotOverflow); n = 0; }
                    uint8_t *d = slot_data(slot, PS_CN + k);
                    const uint8_t *s = M->buf[k];
                    for (int i = tid; i < n; i += 256) d[i] = s[i];
                    if (tid == 0) slot_len(slot)[PS_CN + k] = (uint16_t)n;
                }
            }
            if (tid == 0) U.mbi[row * mbw + mbx] = info;
            __threadfence();
            __syncthreads();
            if (tid == 0) atomicExch(&U.progress[row], mbx + 1);
        }
        __syncthreads();
    }
}

}  // namespace fdvb

// The decoder's GPU half: reconstruction of parsed frames (csrc/host/decode.h)
// and the frame loop of fdv_video_decode / fdv_vtile_decode (fdv.h:6856-6930,
// :7245-7370).  Per frame step, every unit (a stream, or a band's stream):
//
//   P-frame   pdec_inter_kernel: one block per inter macroblock (SKIP, INTER16,
//             INTER8) -- quarter-pel luma from the reference's integer and
//             half-pel planes, eighth-pel chroma, the residual (4x4 and 8x8
//             inverse transforms) -- all macroblocks at once, since inter
//             prediction reads only references; then pdec_intra_kernel, one
//             block per unit, the INTRA16 macroblocks in raster order (their
//             neighbours are then final).
//   key frame idec_kernel: each plane's 64x64 CTU rows in a wavefront (a row
//             runs two CTUs behind the one above, bounded waits), the leaves
//             of a CTU in decode order on a shared-memory tile.
//   then      deblocking (the encoder's kernels) and the decoded frame becomes
//             the nearest reference (the encoder's reference preparation).
//
// The same reconstruction arithmetic as the encoder's kernels (bit-exact with
// the reference's decode_block4 / decode_residual / fdv_mc_* /
// fdv_intra_predict_4x4 / fdv_intra_nxn).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/fdv_b200.h"
#include "../host/decode.h"
#include "../host/fdvb_internal.h"
#include "common.cuh"
#include "inter.cuh"
#include "intra.cuh"

namespace fdvb {
namespace dk {

using dec::Leaf;
using dec::PMB;

struct PUnit {
    int w, h, mbw, mbh, qp;
    uint8_t *rec[3];
    RefPlanes ref[2];
    const PMB *mbs;
    const int16_t *coef;
    const int32_t *intra;
    int nintra;
    int ibase;     // first INTRA16 ticket of this unit
    int epoch;     // this frame step's value of a finished macroblock's flag
    int *done;     // per-macroblock flags (INTRA16 macroblocks)
};

struct IPlaneD {
    uint8_t *rec;
    int w, h, cols, rows;
    const Leaf *leaves;
    const int32_t *ctu_first;
    const int16_t *coef;
    const uint8_t *flags;
    int *progress;
    int qp;
};
struct ITask { int plane, row; };

// 16 levels (natural order) -> residual; one thread.
__device__ __forceinline__ void inv4(const int16_t *lv, int qp, int r[16]) {
    int d[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) d[i] = dequant4(lv[i], i, qp);
    idct4_thread(d, r);
}

// 64 levels (natural order) -> residual, on threads t < 64 of a block of nt
// threads (named barrier `bar`, all nt threads take part): dequantisation
// saturated to int32, the int64 inverse with >> 36 (the encoder's region8
// arithmetic).
__device__ __forceinline__ void inv8_coop(const int16_t *lv, int qp, int32_t *Y, long long *B, int *out, int ostride,
                                          int t, int bar, int nt) {
    if (t < 64) {
        const long long dv = (long long)lv[t] * c_QSTEP8[qp];
        Y[t] = dv < INT32_MIN ? INT32_MIN : (dv > INT32_MAX ? INT32_MAX : (int32_t)dv);
    }
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory");
    if (t < 64) {
        const int y = t >> 3, v = t & 7;
        long long s = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) s += (long long)c8(u * 8 + y) * Y[u * 8 + v];
        B[t] = s;
    }
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory");
    if (t < 64) {
        const int y = t >> 3, x = t & 7;
        long long s = 0;
#pragma unroll
        for (int v = 0; v < 8; ++v) s += B[y * 8 + v] * (long long)c8(v * 8 + x);
        out[y * ostride + x] = (int16_t)((s + (1LL << 35)) >> 36);
    }
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory");
}

// The residual of a 16x16 (or four 8x8 quadrants) luma area and two 8x8
// chroma blocks from a macroblock's coefficient block: res[256] luma,
// cres[2][64]; 64 threads.
__device__ void mb_residual(const PMB &mb, const int16_t *cb, int qp, int *res, int (*cres)[64], int32_t *Y,
                            long long *B, int t, bool chroma8) {
    for (int i = t; i < 256; i += 64) res[i] = 0;
    cres[0][t] = 0;
    cres[1][t] = 0;
    __syncthreads();
    if (mb.coef < 0) return;
    if (t < 16) {   // luma 4x4 blocks: region r, block b
        const int r = t >> 2, b = t & 3;
        if (((mb.lfl >> (2 * r)) & 3) == 1) {
            int rr[16];
            inv4(cb + 64 * r + 16 * b, qp, rr);
            const int ox = (r & 1) * 8 + (b & 1) * 4, oy = (r >> 1) * 8 + (b >> 1) * 4;
            for (int i = 0; i < 16; ++i) res[(oy + (i >> 2)) * 16 + ox + (i & 3)] = rr[i];
        }
    } else if (t < 24) {   // chroma 4x4 blocks
        const int pl = (t - 16) >> 2, b = (t - 16) & 3;
        if (((mb.cfl >> (2 * pl)) & 3) == 1) {
            int rr[16];
            inv4(cb + 256 + 64 * pl + 16 * b, qp, rr);
            const int ox = (b & 1) * 4, oy = (b >> 1) * 4;
            for (int i = 0; i < 16; ++i) cres[pl][(oy + (i >> 2)) * 8 + ox + (i & 3)] = rr[i];
        }
    }
    __syncthreads();
    for (int r = 0; r < 4; ++r)
        if (((mb.lfl >> (2 * r)) & 3) == 2)
            inv8_coop(cb + 64 * r, qp, Y, B, res + (r >> 1) * 8 * 16 + (r & 1) * 8, 16, t, 1, 64);
    if (chroma8)
        for (int pl = 0; pl < 2; ++pl)
            if (((mb.cfl >> (2 * pl)) & 3) == 2) inv8_coop(cb + 256 + 64 * pl, qp, Y, B, cres[pl], 8, t, 1, 64);
}

__global__ void __launch_bounds__(64) pdec_inter_kernel(const PUnit *__restrict__ units, const int *__restrict__ uoff,
                                                         int nu) {
    __shared__ uint8_t pred[256], cpred[2][64];
    __shared__ int res[256], cres[2][64];
    __shared__ int32_t Y[64];
    __shared__ long long B[64];
    const int t = threadIdx.x;
    int u = 0;
    while (u + 1 < nu && (int)blockIdx.x >= uoff[u + 1]) ++u;
    const PUnit &U = units[u];
    const int m = blockIdx.x - uoff[u];
    const PMB mb = U.mbs[m];
    if (mb.mode == 2) return;   // INTRA16: pdec_intra_kernel
    const int mbx = m % U.mbw, mby = m / U.mbw, bx = mbx * 16, by = mby * 16, cbx = bx / 2, cby = by / 2;
    const int w = U.w, cw = w / 2;
    if (mb.mode == 3) {
        const int q = t >> 4, k = t & 15, r = k >> 1, c = (k & 1) * 4, qx = (q & 1) * 8, qy = (q >> 1) * 8;
        const int mx = mb.mv[q][0], my = mb.mv[q][1];
        const GlobalLuma L(U.ref[0]);
        *reinterpret_cast<uint32_t *>(&pred[(qy + r) * 16 + qx + c]) =
            mc_word(L, bx + qx + c + (mx >> 2), by + qy + r + (my >> 2), (my & 3) * 4 + (mx & 3));
    } else {
        const int r = t >> 2, c = (t & 3) * 4, mx = mb.mv[0][0], my = mb.mv[0][1];
        const GlobalLuma L(U.ref[mb.ref]);
        *reinterpret_cast<uint32_t *>(&pred[r * 16 + c]) =
            mc_word(L, bx + c + (mx >> 2), by + r + (my >> 2), (my & 3) * 4 + (mx & 3));
    }
    for (int k = t; k < 128; k += 64) {
        const int pl = k >> 6, p = k & 63, x = p & 7, y = p >> 3;
        const int q = (y >> 2) * 2 + (x >> 2);
        const int mvx = mb.mode == 3 ? mb.mv[q][0] : mb.mv[0][0], mvy = mb.mode == 3 ? mb.mv[q][1] : mb.mv[0][1];
        const RefPlanes &R = U.ref[mb.mode == 3 ? 0 : mb.ref];
        const int cmx = mvx / 2, cmy = mvy / 2;
        cpred[pl][p] = (uint8_t)mc_cpx(pl ? R.V : R.U, R.cs, cbx + x + (cmx >> 2), cby + y + (cmy >> 2), cmx & 3,
                                       cmy & 3);
    }
    mb_residual(mb, U.coef + (mb.coef < 0 ? 0 : mb.coef), U.qp, res, cres, Y, B, t, false);
    for (int i = t; i < 256; i += 64)
        U.rec[0][(size_t)(by + (i >> 4)) * w + bx + (i & 15)] = (uint8_t)clipb(pred[i] + res[i]);
    for (int k = t; k < 128; k += 64) {
        const int pl = k >> 6, p = k & 63;
        U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = (uint8_t)clipb(cpred[pl][p] + cres[pl][p]);
    }
}

// INTRA16 macroblocks (fdv.h:6624-6645) of every unit.  Blocks take tickets
// in raster order over the units' INTRA16 lists; a macroblock predicts from
// its left, top and top-left neighbours, so it waits (bounded) only for those
// of them that are INTRA16 themselves -- they hold earlier tickets, so they
// are running or done.  Inter neighbours were finished by pdec_inter_kernel.
__global__ void __launch_bounds__(64) pdec_intra_kernel(const PUnit *__restrict__ units, int nu, int total,
                                                         int *ticket, unsigned *err, unsigned long long wait_ns) {
    __shared__ uint8_t top[16], left[16], pred[256], cpred[2][64], ctop[2][8], cleft[2][8];
    __shared__ int res[256], cres[2][64], tl, ctl[2];
    __shared__ NNPred nn[3];
    __shared__ int32_t Y[64];
    __shared__ long long B[64];
    __shared__ int s_k, s_ok;
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) s_k = atomicAdd(ticket, 1);
        __syncthreads();
        const int k = s_k;
        if (k >= total) return;
        int ui = 0;
        while (ui + 1 < nu && k >= units[ui + 1].ibase) ++ui;
        const PUnit &U = units[ui];
        const int m = U.intra[k - U.ibase];
        const PMB mb = U.mbs[m];
        const int mbx = m % U.mbw, mby = m / U.mbw;
        const int bx = mbx * 16, by = mby * 16, cbx = bx / 2, cby = by / 2;
        const int ht = by > 0, hl = bx > 0;
        const int w = U.w, cw = w / 2;
        if (t == 0) {
            bool ok = true;
            if (hl && U.mbs[m - 1].mode == 2) ok = ok && wait_at_least(&U.done[m - 1], U.epoch, err, wait_ns);
            if (ht && U.mbs[m - U.mbw].mode == 2) ok = ok && wait_at_least(&U.done[m - U.mbw], U.epoch, err, wait_ns);
            if (ht && hl && U.mbs[m - U.mbw - 1].mode == 2)
                ok = ok && wait_at_least(&U.done[m - U.mbw - 1], U.epoch, err, wait_ns);
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) continue;   // the error word is set; the frame is abandoned
        // neighbours through L2: other blocks of this launch wrote some of them
        if (t < 16) {
            top[t] = ht ? __ldcg(&U.rec[0][(size_t)(by - 1) * w + bx + t]) : 0;
            left[t] = hl ? __ldcg(&U.rec[0][(size_t)(by + t) * w + bx - 1]) : 0;
        } else if (t < 32) {
            const int q = t - 16, pl = q >> 3, i = q & 7;
            ctop[pl][i] = ht ? __ldcg(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx + i]) : 0;
            cleft[pl][i] = hl ? __ldcg(&U.rec[1 + pl][(size_t)(cby + i) * cw + cbx - 1]) : 0;
        } else if (t == 32) {
            tl = (ht && hl) ? __ldcg(&U.rec[0][(size_t)(by - 1) * w + bx - 1]) : 128;
            for (int pl = 0; pl < 2; ++pl)
                ctl[pl] = (ht && hl) ? __ldcg(&U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx - 1]) : 128;
        }
        __syncthreads();
        if (t == 0) nn[0] = nn_setup(mb.sub, top, left, tl, 16, ht, hl);
        else if (t < 3) nn[t] = nn_setup(mb.sub, ctop[t - 1], cleft[t - 1], ctl[t - 1], 8, ht, hl);
        __syncthreads();
        for (int i = t; i < 256; i += 64) pred[i] = (uint8_t)nn_px(nn[0], top, left, i & 15, i >> 4);
        for (int i = t; i < 128; i += 64) {
            const int pl = i >> 6, p = i & 63;
            cpred[pl][p] = (uint8_t)nn_px(nn[1 + pl], ctop[pl], cleft[pl], p & 7, p >> 3);
        }
        mb_residual(mb, U.coef + mb.coef, U.qp, res, cres, Y, B, t, true);
        for (int i = t; i < 256; i += 64)
            U.rec[0][(size_t)(by + (i >> 4)) * w + bx + (i & 15)] = (uint8_t)clipb(pred[i] + res[i]);
        for (int i = t; i < 128; i += 64) {
            const int pl = i >> 6, p = i & 63;
            U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = (uint8_t)clipb(cpred[pl][p] + cres[pl][p]);
        }
        __syncthreads();
        if (t == 0) {
            __threadfence();
            atomicExch(&U.done[m], U.epoch);
        }
    }
}

// ------------------------------------------------------------ key frames --
constexpr int kINT = 128, kTileW = 129;   // tile: the row above (x = -1 .. 127), then 64 rows with the left column

__device__ __forceinline__ int zidx4(int lx, int ly) {
    int z = 0;
    for (int b = 8; b; b >>= 1) z = (z << 2) | ((ly & b) ? 2 : 0) | ((lx & b) ? 1 : 0);
    return z;
}
// Whether the 4x4 cell at (x, y) is already decoded when the one at (bx, by)
// is (fdv.h:3659-3684): rows above the CTU, CTUs to the left, Z order within.
__device__ __forceinline__ bool cell_done(int x, int y, int bx, int by) {
    const int cx0 = bx & ~63, cy0 = by & ~63;
    if (y < cy0) return true;
    if (x < cx0) return true;
    if (x >= cx0 + 64) return false;
    return zidx4((x - cx0) >> 2, (y - cy0) >> 2) < zidx4((bx - cx0) >> 2, (by - cy0) >> 2);
}

__global__ void __launch_bounds__(kINT) idec_kernel(const IPlaneD *__restrict__ planes, const ITask *__restrict__ tasks,
                                                     int ntasks, int *ticket, unsigned *err,
                                                     unsigned long long wait_ns) {
    __shared__ uint8_t T[65 * kTileW];
    __shared__ uint8_t top[64], left[64];
    __shared__ int16_t res[4096];
    __shared__ int T9[9], L5[5];
    __shared__ NNPred nn;
    __shared__ int32_t Y[64];
    __shared__ long long B[64];
    __shared__ int s_task, s_ok, tl_s;
    __shared__ int rtmp[64];
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) s_task = atomicAdd(ticket, 1);
        __syncthreads();
        const int ti = s_task;
        __syncthreads();
        if (ti >= ntasks) return;
        const IPlaneD &P = planes[tasks[ti].plane];
        const int row = tasks[ti].row, w = P.w, h = P.h, cy = row * 64;
        for (int col = 0; col < P.cols; ++col) {
            const int cx = col * 64;
            if (t == 0) s_ok = row == 0 ? 1 : wait_at_least(&P.progress[row - 1], min(col + 2, P.cols), err, wait_ns);
            __syncthreads();
            if (!s_ok) break;
            // the row above (x = cx-1 .. cx+127) and the left column
            for (int k = t; k < kTileW; k += kINT) {
                const int x = cx - 1 + k;
                T[k] = (cy > 0 && x >= 0 && x < w) ? __ldcg(&P.rec[(size_t)(cy - 1) * w + x]) : 0;
            }
            for (int k = t; k < 64; k += kINT) {
                const int y = cy + k;
                T[(k + 1) * kTileW] = (cx > 0 && y < h) ? __ldcg(&P.rec[(size_t)y * w + cx - 1]) : 0;
            }
            __syncthreads();
            const int l0 = P.ctu_first[row * P.cols + col], l1 = P.ctu_first[row * P.cols + col + 1];
            for (int li = l0; li < l1; ++li) {
                const Leaf lf = P.leaves[li];
                const int x = lf.x, y = lf.y, n = lf.n, lx = x - cx, ly = y - cy;
                const int ht = y > 0, hl = x > 0;
                if (n == 4) {
                    // gather_neighbors (fdv.h:3689-3706)
                    const int htl = ht && hl, htr = ht && (x + 4 < w) && cell_done(x + 4, y - 1, x, y);
                    if (t < 8) T9[t + 1] = ht ? ((t < 4 || htr) ? T[ly * kTileW + lx + 1 + t] : T[ly * kTileW + lx + 4]) : 0;
                    else if (t < 12) L5[t - 7] = hl ? T[(ly + t - 7) * kTileW + lx] : 0;
                    else if (t == 12) { const int v = htl ? T[ly * kTileW + lx] : 128; T9[0] = v; L5[0] = v; }
                    else if (t == 32) {
                        int rr[16];
                        inv4(P.coef + lf.coef, P.qp, rr);
                        for (int i = 0; i < 16; ++i) rtmp[i] = rr[i];
                    }
                    __syncthreads();
                    if (t < 16) {
                        const int i = t >> 2, j = t & 3;
                        const int pv = pred4_px(lf.mode, T9, L5, ht, hl, j, i);
                        T[(ly + 1 + i) * kTileW + lx + 1 + j] = (uint8_t)clipb(pv + rtmp[t]);
                    }
                    __syncthreads();
                    continue;
                }
                // an n x n leaf (gather_nb, fdv_intra_nxn, decode_residual)
                for (int k = t; k < n; k += kINT) {
                    top[k] = ht ? T[ly * kTileW + lx + 1 + k] : 0;
                    left[k] = hl ? T[(ly + 1 + k) * kTileW + lx] : 0;
                }
                if (t == 0) tl_s = (ht && hl) ? T[ly * kTileW + lx] : 128;
                for (int k = t; k < n * n; k += kINT) res[k] = 0;
                __syncthreads();
                if (t == 0) nn = nn_setup(lf.mode, top, left, tl_s, n, ht, hl);
                const int nr = n / 8;
                for (int b = t; b < 4 * lf.nreg; b += kINT) {   // 4x4 blocks of flag-1 regions
                    const int r = b >> 2, bb = b & 3;
                    if (P.flags[lf.fl + r] != 1) continue;
                    int rr[16];
                    inv4(P.coef + lf.coef + 64 * r + 16 * bb, P.qp, rr);
                    const int ox = (r % nr) * 8 + (bb & 1) * 4, oy = (r / nr) * 8 + (bb >> 1) * 4;
                    for (int i = 0; i < 16; ++i) res[(oy + (i >> 2)) * n + ox + (i & 3)] = (int16_t)rr[i];
                }
                __syncthreads();
                for (int r = 0; r < lf.nreg; ++r)
                    if (P.flags[lf.fl + r] == 2) {
                        inv8_coop(P.coef + lf.coef + 64 * r, P.qp, Y, B, rtmp, 8, t, 1, kINT);
                        if (t < 64) res[((r / nr) * 8 + (t >> 3)) * n + (r % nr) * 8 + (t & 7)] = (int16_t)rtmp[t];
                        __syncthreads();
                    }
                for (int k = t; k < n * n; k += kINT) {
                    const int i = k / n, j = k - i * n;
                    T[(ly + 1 + i) * kTileW + lx + 1 + j] = (uint8_t)clipb(nn_px(nn, top, left, j, i) + res[k]);
                }
                __syncthreads();
            }
            // the CTU into the plane, then this row's progress
            for (int k = t; k < 64 * 64; k += kINT) {
                const int i = k >> 6, j = k & 63;
                if (cy + i < h && cx + j < w) P.rec[(size_t)(cy + i) * w + cx + j] = T[(i + 1) * kTileW + j + 1];
            }
            __syncthreads();
            if (t == 0) {
                __threadfence();
                atomicExch(&P.progress[row], col + 1);
            }
        }
        __syncthreads();
    }
}

}  // namespace dk

// kernels of kernels.cu (frame operations shared with the encoder)
void launch_refprep(const void *tasks, int ntasks, int maxw, int maxh, int border, cudaStream_t st);
void launch_deblock(const void *tasks, int ntasks, cudaStream_t st);

}  // namespace fdvb


// ---------------------------------------------------------------------------
// Host side: the decoder engine and the fdv_video_decode / fdv_vtile_decode
// entry points.
//
// A decode runs as a pipeline over the frames:
//   parse workers  each owns a fixed set of units (bands) and, frame by frame,
//                  entropy-decodes and parses their blobs and packs each one
//                  into a pinned slot (kSlots per unit, so parsing runs up to
//                  kSlots frames ahead of the GPU);
//   the submitter  (the calling thread) uploads a frame's slots and its
//                  launch descriptors, launches the reconstruction, deblocking,
//                  the download of every unit's frame into a pinned output
//                  slot and the reference preparation, all on one stream;
//   copiers        wait for a frame's download and scatter it into the
//                  caller's buffer.
// Frame f+1's reconstruction reads frame f's references, so the GPU work is
// in stream order; parsing never depends on pixels, so it overlaps freely.
// ---------------------------------------------------------------------------
using namespace fdvb;

namespace {

thread_local std::string g_derr;

struct PrepTaskD {   // frame_ops.cuh PrepTask
    const uint8_t *rec[3];
    uint8_t *G, *B, *H, *J, *U, *V;
    int w, h, ys, cs, border;
};
struct DbTaskD { uint8_t *p; int w, h, qp; };   // frame_ops.cuh DbTask

constexpr int kSlots = 3;      // parse slots per unit
constexpr int kOutSlots = 4;   // output frames in flight

int round_up(int v, int a) { return (v + a - 1) / a * a; }
size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

template <class T>
T *dmalloc(size_t n, std::vector<void *> &own) {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    own.push_back(p);
    return static_cast<T *>(p);
}

struct RefBuf {
    RefPlanes rp{};
    uint8_t *G = nullptr, *B = nullptr, *H = nullptr, *J = nullptr, *U = nullptr, *V = nullptr;
};

// One frame of one unit, parsed and packed for a single upload: a P-frame's
// macroblocks, coefficient blocks and INTRA16 list, or per plane of a key
// frame its leaves, CTU leaf ranges, coefficients and region flags.
struct PSlot {
    dec::Syms sy[3];          // entropy-decoded streams (a key frame: one per plane)
    uint8_t *pin = nullptr;   // pinned, the unit's pay_cap bytes
    size_t used = 0;
    int intra = 0, qp = 0, nintra = 0;
    size_t o_mbs = 0, o_coef = 0, o_intra = 0;
    size_t o_leaves[3] = {}, o_ctu[3] = {}, o_icoef[3] = {}, o_flags[3] = {};
    int pqp[3] = {};
};

struct DUnit {
    int w = 0, h = 0, mbw = 0, mbh = 0, cw = 0, ch = 0;
    size_t rec_off = 0, fs = 0;   // the unit's tight I420 frame in the engine's reconstruction buffer
    RefBuf ref[2];
    int near_i = 0, nref = 0;
    fdvb_tabcache tc{};
    uint8_t *d_pay[2] = {};       // payload on the device, by frame-step parity
    size_t pay_cap = 0;
    int *d_prog = nullptr;        // key-frame CTU-row progress, three planes
    int *d_done = nullptr;        // INTRA16 macroblocks' finished flags (frame-step epochs)
    int pw[3] = {}, ph[3] = {}, cols[3] = {}, rows[3] = {};
    PSlot slot[kSlots];
};

struct DecEngine {
    int device = 0, border = 32, nsm = 148;
    std::vector<std::pair<int, int>> sizes;
    cudaStream_t st = nullptr;      // reconstruction, deblocking, reference preparation
    cudaStream_t st_in = nullptr;   // uploads
    cudaStream_t st_out = nullptr;  // downloads
    std::vector<DUnit> units;
    std::vector<void *> own;      // device allocations
    std::vector<void *> pinned;   // host allocations
    uint8_t *d_rec[2] = {};       // every unit's reconstruction, back to back, by frame-step parity
    size_t rec_bytes = 0;
    uint8_t *out_pin[kOutSlots] = {};
    uint8_t *desc_pin[kOutSlots] = {};
    uint8_t *d_desc[2] = {};      // launch descriptors, by frame-step parity
    size_t desc_cap = 0;
    int *d_ticket = nullptr;      // [0] key-frame rows, [1] INTRA16 macroblocks
    unsigned *d_err = nullptr;
    int epoch = 0;                // frame steps run by this engine
    cudaEvent_t ev_in[kSlots] = {}, ev_out[kOutSlots] = {};
    // per parity b: uploads done, kernels done with the payload and
    // descriptors, frame deblocked, frame downloaded
    cudaEvent_t ev_up[2] = {}, ev_used[2] = {}, ev_dbk[2] = {}, ev_d2h[2] = {};
    int ntask_max = 0;
    std::vector<cudaEvent_t> tev;   // timing events (fdvd_timing), reused between calls
    ~DecEngine() {
        cudaSetDevice(device);
        for (auto q : {st, st_in, st_out}) if (q) cudaStreamSynchronize(q);
        for (auto e : tev) cudaEventDestroy(e);
        for (auto e : ev_in) if (e) cudaEventDestroy(e);
        for (auto e : ev_out) if (e) cudaEventDestroy(e);
        for (int b = 0; b < 2; ++b)
            for (auto e : {ev_up[b], ev_used[b], ev_dbk[b], ev_d2h[b]}) if (e) cudaEventDestroy(e);
        for (void *p : own) cudaFree(p);
        for (void *p : pinned) cudaFreeHost(p);
        for (auto q : {st, st_in, st_out}) if (q) cudaStreamDestroy(q);
    }
};

bool ck(cudaError_t e, const char *what, std::string &err) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}
#define DCK(x)                               \
    do {                                     \
        if (!ck((x), #x, g_derr)) return -1; \
    } while (0)

// The transform tables of this translation unit's kernels.
int upload_dec_tables() {
    int32_t c8[64], q8[52], c8t[64];
    fdvb_c8_tables(c8, q8);
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) c8t[j * 8 + i] = c8[i * 8 + j];
    DCK(cudaMemcpyToSymbol(g_C8, c8, sizeof c8));
    DCK(cudaMemcpyToSymbol(g_C8T, c8t, sizeof c8t));
    DCK(cudaMemcpyToSymbol(c_QSTEP8, q8, sizeof q8));
    return 0;
}

// The border the reference decoder's planes carry for the configured search
// range (FDV_BORDER of the matching build): motion vectors past it are
// rejected, as the reference rejects them.
int reference_border() {
    const int r = fdvb_get_search_range();
    return r <= 16 ? 32 : (r <= 32 ? 64 : 96);
}

// Byte sizes of one frame's launch descriptors (the largest frame: every unit
// a P-frame and a key frame at once).
struct DescLayout {
    size_t pu, uoff, planes, tasks, db, prep, total;
    DescLayout(int nu, int ntasks) {
        pu = 0;
        uoff = pu + al256(sizeof(dk::PUnit) * nu);
        planes = uoff + al256(sizeof(int) * (nu + 1));
        tasks = planes + al256(sizeof(dk::IPlaneD) * 3 * nu);
        db = tasks + al256(sizeof(dk::ITask) * std::max(ntasks, 1));
        prep = db + al256(sizeof(DbTaskD) * 3 * nu);
        total = prep + al256(sizeof(PrepTaskD) * nu);
    }
};

int engine_init(DecEngine &E, const std::vector<std::pair<int, int>> &sizes, int device, int border) {
    E.device = device;
    E.border = border;
    E.sizes = sizes;
    DCK(cudaSetDevice(device));
    cudaDeviceGetAttribute(&E.nsm, cudaDevAttrMultiProcessorCount, device);
    for (auto q : {&E.st, &E.st_in, &E.st_out}) DCK(cudaStreamCreateWithFlags(q, cudaStreamNonBlocking));
    for (auto &e : E.ev_in) DCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : E.ev_out) DCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int b = 0; b < 2; ++b)
        for (auto e : {&E.ev_up[b], &E.ev_used[b], &E.ev_dbk[b], &E.ev_d2h[b]})
            DCK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    if (upload_dec_tables()) return -1;
    const int Bp = border + 16;   // allocated border: the checked one plus the filter taps
    const int nu = (int)sizes.size();
    E.units.resize(nu);
    auto fail_alloc = [&]() { g_derr = "device or pinned allocation failed"; return -1; };
    auto pin = [&](size_t n) -> uint8_t * {
        void *p = nullptr;
        if (cudaHostAlloc(&p, std::max<size_t>(n, 1), cudaHostAllocDefault) != cudaSuccess) return nullptr;
        E.pinned.push_back(p);
        return static_cast<uint8_t *>(p);
    };
    int ntasks = 0;
    for (int i = 0; i < nu; ++i) {
        DUnit &u = E.units[i];
        u.w = sizes[i].first;
        u.h = sizes[i].second;
        u.mbw = u.w / 16; u.mbh = u.h / 16; u.cw = u.w / 2; u.ch = u.h / 2;
        u.fs = (size_t)u.w * u.h * 3 / 2;
        u.rec_off = E.rec_bytes;
        E.rec_bytes += u.fs;
        const size_t nmb = (size_t)u.mbw * u.mbh;
        const int ys = round_up(u.w + 2 * Bp, 64), cs = round_up(u.cw + 2 * Bp, 64);
        const size_t lsz = (size_t)ys * (u.h + 2 * Bp), csz = (size_t)cs * (u.ch + 2 * Bp);
        for (int r = 0; r < 2; ++r) {
            uint8_t *m = dmalloc<uint8_t>(4 * lsz + 2 * csz, E.own);
            if (!m) return fail_alloc();
            DCK(cudaMemset(m, 0, 4 * lsz + 2 * csz));
            RefBuf &s = u.ref[r];
            s.G = m + (size_t)Bp * ys + Bp; m += lsz;
            s.B = m + (size_t)Bp * ys + Bp; m += lsz;
            s.H = m + (size_t)Bp * ys + Bp; m += lsz;
            s.J = m + (size_t)Bp * ys + Bp; m += lsz;
            s.U = m + (size_t)Bp * cs + Bp; m += csz;
            s.V = m + (size_t)Bp * cs + Bp;
            s.rp.G = s.G; s.rp.B = s.B; s.rp.H = s.H; s.rp.J = s.J; s.rp.U = s.U; s.rp.V = s.V;
            s.rp.ys = ys; s.rp.cs = cs;
        }
        u.pw[0] = u.w; u.ph[0] = u.h; u.pw[1] = u.pw[2] = u.cw; u.ph[1] = u.ph[2] = u.ch;
        int nprog = 0;
        size_t ipay = 0;
        for (int p = 0; p < 3; ++p) {
            u.cols[p] = (u.pw[p] + 63) / 64;
            u.rows[p] = (u.ph[p] + 63) / 64;
            nprog += u.rows[p];
            ntasks += u.rows[p];
            const size_t px = (size_t)u.pw[p] * u.ph[p];
            // at most one leaf per 4x4 cell, one coefficient per sample, one flag per 8x8 region
            ipay += al256(px / 16 * sizeof(dec::Leaf)) + al256(((size_t)u.cols[p] * u.rows[p] + 1) * 4) +
                    al256(px * 2) + al256(px / 64 + 1);
        }
        const size_t ppay = al256(nmb * sizeof(dec::PMB)) + al256(nmb * 384 * 2) + al256(nmb * 4);
        u.pay_cap = std::max(ppay, ipay);
        for (auto &dp : u.d_pay)
            if (!(dp = dmalloc<uint8_t>(u.pay_cap, E.own))) return fail_alloc();
        u.d_prog = dmalloc<int>(nprog, E.own);
        u.d_done = dmalloc<int>(nmb, E.own);
        if (!u.d_prog || !u.d_done) return fail_alloc();
        DCK(cudaMemset(u.d_done, 0, nmb * sizeof(int)));
        for (auto &sl : u.slot)
            if (!(sl.pin = pin(u.pay_cap))) return fail_alloc();
    }
    E.ntask_max = ntasks;
    const DescLayout D(nu, ntasks);
    E.desc_cap = D.total;
    for (int b = 0; b < 2; ++b)
        if (!(E.d_desc[b] = dmalloc<uint8_t>(D.total, E.own)) || !(E.d_rec[b] = dmalloc<uint8_t>(E.rec_bytes, E.own)))
            return fail_alloc();
    E.d_ticket = dmalloc<int>(2, E.own);
    E.d_err = dmalloc<unsigned>(1, E.own);
    if (!E.d_ticket || !E.d_err) return fail_alloc();
    for (int o = 0; o < kOutSlots; ++o)
        if (!(E.out_pin[o] = pin(E.rec_bytes)) || !(E.desc_pin[o] = pin(D.total))) return fail_alloc();
    return 0;
}

// Timing (fdvd_timing / fdvd_stats): kinds 0 P-frame inter reconstruction,
// 1 INTRA16 reconstruction, 2 key-frame reconstruction, 3 deblocking +
// reference preparation, 4 the whole frame step on the GPU (CUDA events);
// host wall time of 5 symbol decoding (summed over the chains), 6 scattering
// decoded frames (summed over copiers), 7 the submitter waiting for parsed
// frames, 8 building records (summed over the record workers).
constexpr int kTimeKinds = 9;
std::atomic<int> g_dtiming{0};
std::mutex g_dstat_mu;
double g_dms[kTimeKinds];
long long g_dn[kTimeKinds];

// Engines kept between calls, keyed by device, border and unit sizes; taken
// out while in use.
constexpr size_t kCacheMax = 4;
std::mutex g_dcache_mu;
std::vector<DecEngine *> *g_dcache = new std::vector<DecEngine *>();   // never destroyed: outlives the CUDA runtime

DecEngine *engine_acquire(const std::vector<std::pair<int, int>> &sizes) {
    const int device = fdvb_device_setting(), border = reference_border();
    {
        std::lock_guard<std::mutex> lk(g_dcache_mu);
        for (size_t i = 0; i < g_dcache->size(); ++i) {
            DecEngine *E = (*g_dcache)[i];
            if (E->device == device && E->border == border && E->sizes == sizes) {
                g_dcache->erase(g_dcache->begin() + (long)i);
                return E;
            }
        }
    }
    DecEngine *E = new DecEngine();
    if (engine_init(*E, sizes, device, border)) {
        const std::string e = g_derr;
        delete E;
        g_derr = e;
        return nullptr;
    }
    return E;
}

void engine_release(DecEngine *E) {
    DecEngine *evict = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_dcache_mu);
        g_dcache->push_back(E);
        if (g_dcache->size() > kCacheMax) {
            evict = g_dcache->front();
            g_dcache->erase(g_dcache->begin());
        }
    }
    delete evict;
}

struct Stream {   // one fdv_video_encode container
    const uint8_t *in;
    size_t len, p;
    int nf, w, h, qp, keyint;
};

bool open_stream(const uint8_t *in, size_t len, Stream &s) {
    if (!in || len < 8) return false;
    s.in = in; s.len = len; s.p = 0;
    auto g16 = [&]() { const int v = in[s.p] | (in[s.p + 1] << 8); s.p += 2; return v; };
    s.nf = g16(); s.w = g16(); s.h = g16();
    s.qp = in[s.p++];
    s.keyint = in[s.p++];
    return s.nf > 0 && s.w > 0 && s.h > 0 && !(s.w & 15) && !(s.h & 15) && s.w <= 8192 && s.h <= 8192 && s.qp <= 51;
}

bool next_blob(Stream &s, const uint8_t **b, size_t *n) {
    if (s.p + 4 > s.len) return false;
    uint32_t v = 0;
    for (int k = 0; k < 4; ++k) v |= (uint32_t)s.in[s.p + k] << (8 * k);
    s.p += 4;
    if (s.p + v > s.len) return false;
    *b = s.in + s.p;
    *n = v;
    s.p += v;
    return true;
}

// The sequential half of parsing one blob of unit u into slot S: its symbol
// streams (the P-frame table cache carries from frame to frame).  0, or -1
// for a malformed blob.
int parse_symbols(DUnit &u, const uint8_t *blob, size_t blen, int intra, PSlot &S) {
    S.intra = intra;
    if (!intra) return dec::pframe_symbols(blob, blen, u.w, u.h, &u.tc, S.sy[0]);
    memset(&u.tc, 0, sizeof u.tc);   // tables and history restart at a key frame
    size_t p = 0;
    for (int pl = 0; pl < 3; ++pl) {
        if (p + 4 > blen) return -1;
        uint32_t n = 0;
        for (int k = 0; k < 4; ++k) n |= (uint32_t)blob[p + k] << (8 * k);
        p += 4;
        if (p + n > blen || n < 4) return -1;
        if (dec::iplane_symbols(blob + p, n, u.pw[pl], u.ph[pl], S.sy[pl])) return -1;
        p += n;
    }
    return 0;
}

// Record scratch of one worker thread (capacity kept between frames).
struct RecScratch {
    dec::PFrame pf;
    dec::IPlane ip;
};

// The independent half: slot S's symbols into records, packed into its
// pinned payload.
int parse_records(const DUnit &u, int border, PSlot &S, RecScratch &R) {
    size_t off = 0;
    bool room = true;
    auto put = [&](const void *src, size_t n) -> size_t {
        const size_t at = off;
        if (off + n > u.pay_cap) { room = false; return 0; }
        if (n) memcpy(S.pin + off, src, n);
        off = al256(off + n);
        return at;
    };
    if (S.intra) {
        for (int pl = 0; pl < 3; ++pl) {
            dec::IPlane &P = R.ip;
            if (dec::iplane_records(S.sy[pl], P)) return -1;
            S.o_leaves[pl] = put(P.leaves.data(), P.leaves.size() * sizeof(dec::Leaf));
            S.o_ctu[pl] = put(P.ctu_first.data(), P.ctu_first.size() * 4);
            S.o_icoef[pl] = put(P.coef.data(), P.coef.size() * 2);
            S.o_flags[pl] = put(P.flags.data(), P.flags.size());
            S.pqp[pl] = P.qp;
        }
    } else {
        dec::PFrame &f = R.pf;
        if (dec::pframe_records(S.sy[0], u.w, u.h, border, f)) return -1;
        S.qp = f.qp;
        S.nintra = (int)f.intra.size();
        S.o_mbs = put(f.mbs.data(), f.mbs.size() * sizeof(dec::PMB));
        S.o_coef = put(f.coef.data(), f.coef.size() * 2);
        S.o_intra = put(f.intra.data(), f.intra.size() * 4);
    }
    S.used = off;
    return room ? 0 : -1;
}

// Progress shared by the pipeline's threads.
struct Pipe {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::pair<int, int>> jobs;   // (frame, unit) with symbols, awaiting records
    std::vector<int> parsed;   // units parsed, per frame
    std::vector<char> copied;  // frame scattered into the output
    int submitted = 0;         // frames whose GPU work is enqueued
    bool abort = false;
    std::string err;
    void fail(const std::string &e) {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!abort) err = e;
            abort = true;
        }
        cv.notify_all();
    }
    template <class P>
    bool wait(P pred) {   // false when the pipeline was aborted
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return abort || pred(); });
        return !abort;
    }
};

// Decode one stream per band (band b at rows y0[b]) into full W x H frames.
int decode_bands(std::vector<Stream> &bs, const std::vector<int> &y0, int W, int H, int nf, uint8_t *out,
                 int nthreads) {
    std::vector<std::pair<int, int>> sizes;
    for (auto &s : bs) sizes.push_back({s.w, s.h});
    DecEngine *Ep = engine_acquire(sizes);
    if (!Ep) return -1;
    DecEngine &E = *Ep;
    DCK(cudaSetDevice(E.device));
    const int nu = (int)bs.size(), cw = W / 2, ch = H / 2;
    const size_t fsize = (size_t)W * H + 2 * (size_t)cw * ch;
    for (auto &u : E.units) { u.near_i = 0; u.nref = 0; }
    DCK(cudaMemsetAsync(E.d_err, 0, sizeof(unsigned), E.st));

    Pipe P;
    P.parsed.assign(nf, 0);
    P.copied.assign(nf, 0);
    // threads: nwk symbol chains (units split among them), nrec record
    // workers, ncopy copiers, and this one; nthreads bounds the parsing ones
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int ncopy = hw >= 8 ? 2 : 1;
    const int nparse = std::max(2, std::min(nthreads, hw - ncopy - 1));
    const int nwk = std::max(1, std::min(nu, nparse - 1));
    const int nrec = std::max(1, nparse - nwk);
    const int border = E.border, device = E.device;

    const bool timing = g_dtiming.load() != 0;
    std::atomic<long long> host_ns[4] = {{0}, {0}, {0}, {0}};   // symbols, scatter, submit wait, records
    auto now_ns = [] {
        return std::chrono::duration_cast<std::chrono::nanoseconds>(
                   std::chrono::steady_clock::now().time_since_epoch()).count();
    };
    auto parse_worker = [&](int wk) {
        cudaSetDevice(device);
        for (int f = 0; f < nf; ++f) {
            const int s = f % kSlots;
            if (f >= kSlots) {   // slot s last held frame f - kSlots: its upload must be done
                if (!P.wait([&] { return P.submitted >= f - kSlots + 1; })) return;
                std::string e;
                if (!ck(cudaEventSynchronize(E.ev_in[s]), "upload", e)) { P.fail(e); return; }
            }
            for (int i = wk; i < nu; i += nwk) {
                DUnit &u = E.units[i];
                const uint8_t *blob;
                size_t blen;
                const long long t0 = timing ? now_ns() : 0;
                if (!next_blob(bs[i], &blob, &blen)) { P.fail("truncated stream"); return; }
                const int intra = f == 0 || (bs[i].keyint > 0 && f % bs[i].keyint == 0);
                if (parse_symbols(u, blob, blen, intra, u.slot[s])) { P.fail("malformed frame blob"); return; }
                if (timing) host_ns[0] += now_ns() - t0;
                {
                    std::lock_guard<std::mutex> lk(P.mu);
                    P.jobs.push_back({f, i});
                }
                P.cv.notify_all();
            }
        }
    };
    const long long njobs = (long long)nf * nu;
    long long taken = 0;   // jobs handed to record workers (under P.mu)
    auto rec_worker = [&]() {
        RecScratch R;
        for (;;) {
            std::pair<int, int> job;
            {
                std::unique_lock<std::mutex> lk(P.mu);
                P.cv.wait(lk, [&] { return P.abort || taken == njobs || !P.jobs.empty(); });
                if (P.abort || (taken == njobs && P.jobs.empty())) return;
                job = P.jobs.front();
                P.jobs.pop_front();
                ++taken;
            }
            const long long t0 = timing ? now_ns() : 0;
            DUnit &u = E.units[job.second];
            if (parse_records(u, border, u.slot[job.first % kSlots], R)) { P.fail("malformed frame blob"); return; }
            if (timing) host_ns[3] += now_ns() - t0;
            {
                std::lock_guard<std::mutex> lk(P.mu);
                P.parsed[job.first] += 1;
                if (taken == njobs) P.cv.notify_all();   // idle workers can leave
            }
            P.cv.notify_all();
        }
    };
    auto copier = [&](int c) {
        cudaSetDevice(device);
        for (int f = c; f < nf; f += ncopy) {
            if (!P.wait([&] { return P.submitted > f; })) return;
            std::string e;
            if (!ck(cudaEventSynchronize(E.ev_out[f % kOutSlots]), "download", e)) { P.fail(e); return; }
            const long long t0 = timing ? now_ns() : 0;
            const uint8_t *src = E.out_pin[f % kOutSlots];
            uint8_t *fy = out + (size_t)f * fsize, *fu = fy + (size_t)W * H, *fv = fu + (size_t)cw * ch;
            for (int i = 0; i < nu; ++i) {
                const DUnit &u = E.units[i];
                const uint8_t *s = src + u.rec_off;
                memcpy(fy + (size_t)y0[i] * W, s, (size_t)u.w * u.h);
                memcpy(fu + (size_t)(y0[i] / 2) * cw, s + (size_t)u.w * u.h, (size_t)u.cw * u.ch);
                memcpy(fv + (size_t)(y0[i] / 2) * cw, s + (size_t)u.w * u.h + (size_t)u.cw * u.ch,
                       (size_t)u.cw * u.ch);
            }
            if (timing) host_ns[1] += now_ns() - t0;
            {
                std::lock_guard<std::mutex> lk(P.mu);
                P.copied[f] = 1;
            }
            P.cv.notify_all();
        }
    };
    std::vector<std::thread> th;
    for (int k = 0; k < nwk; ++k) th.emplace_back(parse_worker, k);
    for (int k = 0; k < nrec; ++k) th.emplace_back(rec_worker);
    for (int c = 0; c < ncopy; ++c) th.emplace_back(copier, c);

    const DescLayout D(nu, E.ntask_max);
    struct TMark { int kind, a, b; };
    std::vector<TMark> marks;
    int nev = 0;
    auto tev = [&]() -> int {   // record the next timing event on the stream
        if (nev == (int)E.tev.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            E.tev.push_back(e);
        }
        if (cudaEventRecord(E.tev[nev], E.st) != cudaSuccess) return -1;
        return nev++;
    };
    auto mark = [&](int kind, int a) {
        if (a >= 0) {
            const int b = tev();
            if (b >= 0) marks.push_back({kind, a, b});
        }
    };
    std::vector<dk::PUnit> pu;
    std::vector<int> uoff;
    std::vector<dk::IPlaneD> ipl;
    std::vector<dk::ITask> tasks;
    std::vector<DbTaskD> db;
    std::vector<PrepTaskD> prep;
    // Frame step f uses the device buffers of parity b = f & 1: its uploads
    // (st_in) wait until step f-2's kernels are done with them, its kernels
    // (st) wait for the uploads and for step f-2's download of the same
    // reconstruction buffer, its download (st_out) waits for the deblocking.
    auto submit = [&](int f) -> int {
        const int s = f % kSlots, o = f % kOutSlots, b = f & 1;
        const int epoch = ++E.epoch;
        uint8_t *const drec = E.d_rec[b], *const ddesc = E.d_desc[b];
        int nintra = 0;
        pu.clear(); uoff.assign(1, 0); ipl.clear(); tasks.clear(); db.clear(); prep.clear();
        if (f >= 2) DCK(cudaStreamWaitEvent(E.st_in, E.ev_used[b], 0));
        for (int i = 0; i < nu; ++i) {
            DUnit &u = E.units[i];
            const PSlot &S = u.slot[s];
            uint8_t *const pay = u.d_pay[b];
            DCK(cudaMemcpyAsync(pay, S.pin, S.used, cudaMemcpyHostToDevice, E.st_in));
            uint8_t *rec[3] = {drec + u.rec_off, drec + u.rec_off + (size_t)u.w * u.h,
                               drec + u.rec_off + (size_t)u.w * u.h + (size_t)u.cw * u.ch};
            if (!S.intra) {
                dk::PUnit d{};
                d.w = u.w; d.h = u.h; d.mbw = u.mbw; d.mbh = u.mbh; d.qp = S.qp;
                for (int p = 0; p < 3; ++p) d.rec[p] = rec[p];
                d.ref[0] = u.ref[u.near_i].rp;
                d.ref[1] = u.nref >= 2 ? u.ref[1 - u.near_i].rp : u.ref[u.near_i].rp;
                d.mbs = reinterpret_cast<const dec::PMB *>(pay + S.o_mbs);
                d.coef = reinterpret_cast<const int16_t *>(pay + S.o_coef);
                d.intra = reinterpret_cast<const int32_t *>(pay + S.o_intra);
                d.nintra = S.nintra;
                d.ibase = nintra;
                d.epoch = epoch;
                d.done = u.d_done;
                nintra += S.nintra;
                pu.push_back(d);
                uoff.push_back(uoff.back() + u.mbw * u.mbh);
                for (int p = 0; p < 3; ++p) db.push_back({rec[p], u.pw[p], u.ph[p], S.qp});
            } else {
                int prog = 0;
                for (int p = 0; p < 3; ++p) {
                    dk::IPlaneD d{};
                    d.rec = rec[p]; d.w = u.pw[p]; d.h = u.ph[p]; d.cols = u.cols[p]; d.rows = u.rows[p];
                    d.leaves = reinterpret_cast<const dec::Leaf *>(pay + S.o_leaves[p]);
                    d.ctu_first = reinterpret_cast<const int32_t *>(pay + S.o_ctu[p]);
                    d.coef = reinterpret_cast<const int16_t *>(pay + S.o_icoef[p]);
                    d.flags = pay + S.o_flags[p];
                    d.progress = u.d_prog + prog;
                    d.qp = S.pqp[p];
                    prog += u.rows[p];
                    ipl.push_back(d);
                    db.push_back({rec[p], u.pw[p], u.ph[p], S.pqp[p]});
                }
            }
            RefBuf &far = u.ref[1 - u.near_i];
            prep.push_back({{rec[0], rec[1], rec[2]}, far.G, far.B, far.H, far.J, far.U, far.V, u.w, u.h, far.rp.ys,
                            far.rp.cs, border + 16});
        }
        // key-frame rows in (row, plane) order, so every plane's early rows start first
        int maxr = 0;
        for (auto &p : ipl) maxr = std::max(maxr, p.rows);
        for (int r = 0; r < maxr; ++r)
            for (int p = 0; p < (int)ipl.size(); ++p)
                if (r < ipl[p].rows) tasks.push_back({p, r});
        uint8_t *h = E.desc_pin[o];
        memcpy(h + D.pu, pu.data(), pu.size() * sizeof(dk::PUnit));
        memcpy(h + D.uoff, uoff.data(), uoff.size() * sizeof(int));
        memcpy(h + D.planes, ipl.data(), ipl.size() * sizeof(dk::IPlaneD));
        memcpy(h + D.tasks, tasks.data(), tasks.size() * sizeof(dk::ITask));
        memcpy(h + D.db, db.data(), db.size() * sizeof(DbTaskD));
        memcpy(h + D.prep, prep.data(), prep.size() * sizeof(PrepTaskD));
        DCK(cudaMemcpyAsync(ddesc, h, D.total, cudaMemcpyHostToDevice, E.st_in));
        DCK(cudaEventRecord(E.ev_in[s], E.st_in));
        DCK(cudaEventRecord(E.ev_up[b], E.st_in));

        DCK(cudaStreamWaitEvent(E.st, E.ev_up[b], 0));
        if (f >= 2) DCK(cudaStreamWaitEvent(E.st, E.ev_d2h[b], 0));
        const int t_frame = timing ? tev() : -1;
        for (int i = 0; i < nu; ++i)
            if (E.units[i].slot[s].intra) {
                const DUnit &u = E.units[i];
                DCK(cudaMemsetAsync(u.d_prog, 0, sizeof(int) * (u.rows[0] + u.rows[1] + u.rows[2]), E.st));
            }
        const auto *d_pu = reinterpret_cast<const dk::PUnit *>(ddesc + D.pu);
        if (!pu.empty()) {
            int t0 = timing ? tev() : -1;
            dk::pdec_inter_kernel<<<uoff.back(), 64, 0, E.st>>>(d_pu, reinterpret_cast<const int *>(ddesc + D.uoff),
                                                                 (int)pu.size());
            mark(0, t0);
            if (nintra) {
                DCK(cudaMemsetAsync(E.d_ticket + 1, 0, sizeof(int), E.st));
                t0 = timing ? tev() : -1;
                dk::pdec_intra_kernel<<<std::min(nintra, 8 * E.nsm), 64, 0, E.st>>>(d_pu, (int)pu.size(), nintra,
                                                                                  E.d_ticket + 1, E.d_err,
                                                                                  4000000000ull);
                mark(1, t0);
            }
        }
        if (!tasks.empty()) {
            DCK(cudaMemsetAsync(E.d_ticket, 0, sizeof(int), E.st));
            const int t0 = timing ? tev() : -1;
            dk::idec_kernel<<<std::min((int)tasks.size(), E.nsm), dk::kINT, 0, E.st>>>(
                reinterpret_cast<const dk::IPlaneD *>(ddesc + D.planes),
                reinterpret_cast<const dk::ITask *>(ddesc + D.tasks), (int)tasks.size(), E.d_ticket, E.d_err,
                4000000000ull);
            mark(2, t0);
        }
        DCK(cudaGetLastError());
        const int t_ops = timing ? tev() : -1;
        launch_deblock(ddesc + D.db, (int)db.size(), E.st);
        DCK(cudaEventRecord(E.ev_dbk[b], E.st));
        DCK(cudaStreamWaitEvent(E.st_out, E.ev_dbk[b], 0));
        DCK(cudaMemcpyAsync(E.out_pin[o], drec, E.rec_bytes, cudaMemcpyDeviceToHost, E.st_out));
        DCK(cudaEventRecord(E.ev_d2h[b], E.st_out));
        DCK(cudaEventRecord(E.ev_out[o], E.st_out));
        // the decoded frame becomes the nearest reference (load_ref, fdv.h:5183)
        int maxw = 0, maxh = 0;
        for (auto &u : E.units) { maxw = std::max(maxw, u.w); maxh = std::max(maxh, u.h); }
        launch_refprep(ddesc + D.prep, (int)prep.size(), maxw, maxh, border + 16, E.st);
        DCK(cudaGetLastError());
        mark(3, t_ops);
        mark(4, t_frame);
        DCK(cudaEventRecord(E.ev_used[b], E.st));
        for (int i = 0; i < nu; ++i) {
            DUnit &u = E.units[i];
            u.near_i = 1 - u.near_i;
            u.nref = u.slot[s].intra ? 1 : (u.nref < 2 ? u.nref + 1 : 2);
        }
        return 0;
    };
    for (int f = 0; f < nf; ++f) {
        const long long t0 = timing ? now_ns() : 0;
        if (!P.wait([&] { return P.parsed[f] == nu && (f < kOutSlots || P.copied[f - kOutSlots]); })) break;
        if (timing) host_ns[2] += now_ns() - t0;
        if (submit(f)) { P.fail(g_derr); break; }
        {
            std::lock_guard<std::mutex> lk(P.mu);
            P.submitted = f + 1;
        }
        P.cv.notify_all();
    }
    for (auto &t : th) t.join();
    unsigned herr = 0;
    std::string e;
    const bool ok = ck(cudaMemcpyAsync(&herr, E.d_err, sizeof herr, cudaMemcpyDeviceToHost, E.st), "error word", e) &&
                    ck(cudaStreamSynchronize(E.st), "decode", e) && ck(cudaStreamSynchronize(E.st_in), "upload", e) &&
                    ck(cudaStreamSynchronize(E.st_out), "download", e);
    if (!ok) {   // the context may be unusable: drop the engine
        delete Ep;
        g_derr = e;
        return -1;
    }
    if (timing && !P.abort) {
        double ms[kTimeKinds] = {};
        long long n[kTimeKinds] = {};
        for (auto &m : marks) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, E.tev[m.a], E.tev[m.b]) == cudaSuccess) { ms[m.kind] += t; ++n[m.kind]; }
        }
        for (int k = 0; k < 4; ++k) { ms[5 + k] = host_ns[k] * 1e-6; n[5 + k] = nf; }
        std::lock_guard<std::mutex> lk(g_dstat_mu);
        for (int k = 0; k < kTimeKinds; ++k) { g_dms[k] += ms[k]; g_dn[k] += n[k]; }
    }
    engine_release(Ep);
    if (P.abort) { g_derr = P.err; return -1; }
    if (herr) { g_derr = "key-frame wavefront wait timed out"; return -1; }
    return 0;
}

}  // namespace

void fdvd_release_cached(void) {
    std::vector<DecEngine *> v;
    {
        std::lock_guard<std::mutex> lk(g_dcache_mu);
        v.swap(*g_dcache);
    }
    for (DecEngine *E : v) delete E;
}

extern "C" {

const char *fdvd_last_error(void) { return g_derr.c_str(); }

void fdvd_timing(int on) { g_dtiming.store(on ? 1 : 0); }

void fdvd_stats(double *ms, long long *n, int reset) {
    std::lock_guard<std::mutex> lk(g_dstat_mu);
    for (int k = 0; k < kTimeKinds; ++k) {
        if (ms) ms[k] = g_dms[k];
        if (n) n[k] = g_dn[k];
        if (reset) { g_dms[k] = 0; g_dn[k] = 0; }
    }
}

int fdv_video_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h) {
    g_derr.clear();
    Stream s;
    if (!out || !open_stream(in, len, s)) { g_derr = "bad stream header"; return -1; }
    std::vector<Stream> bs{s};
    if (decode_bands(bs, {0}, s.w, s.h, s.nf, out, 1 << 16)) return -1;   // one chain, records on every core
    if (nframes) *nframes = s.nf;
    if (w) *w = s.w;
    if (h) *h = s.h;
    return 0;
}

int fdv_vtile_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h, int nthreads) {
    g_derr.clear();
    if (!in || !out || len < 12) { g_derr = "bad stream header"; return -1; }
    size_t p = 0;
    auto g16 = [&]() { const int v = in[p] | (in[p + 1] << 8); p += 2; return v; };
    const int W = g16(), H = g16(), nf = g16();
    p += 2;   // qp, key interval (each band's stream carries its own)
    const int nb = g16(), band_mbrows = g16();
    if (nf <= 0 || W <= 0 || H <= 0 || (W & 15) || (H & 15) || W > 8192 || H > 8192 || band_mbrows < 1) {
        g_derr = "bad stream header";
        return -1;
    }
    const int bh_full = band_mbrows * 16;
    if (nb != (H + bh_full - 1) / bh_full || nb < 1 || nb > H / 16) { g_derr = "bad band layout"; return -1; }
    std::vector<Stream> bs(nb);
    std::vector<int> y0(nb);
    for (int b = 0; b < nb; ++b) {
        y0[b] = b * bh_full;
        const int bh = y0[b] + bh_full <= H ? bh_full : H - y0[b];
        if (p + 4 > len) { g_derr = "truncated stream"; return -1; }
        uint32_t n = 0;
        for (int k = 0; k < 4; ++k) n |= (uint32_t)in[p + k] << (8 * k);
        p += 4;
        if (p + n > len) { g_derr = "truncated stream"; return -1; }
        if (!open_stream(in + p, n, bs[b]) || bs[b].nf != nf || bs[b].w != W || bs[b].h != bh) {
            g_derr = "bad band stream";
            return -1;
        }
        p += n;
    }
    if (decode_bands(bs, y0, W, H, nf, out, nthreads)) return -1;
    if (nframes) *nframes = nf;
    if (w) *w = W;
    if (h) *h = H;
    return 0;
}

}  // extern "C"

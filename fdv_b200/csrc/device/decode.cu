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
#include <cstdio>
#include <cstring>
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

// INTRA16 macroblocks of one unit, raster order (fdv.h:6624-6645).
__global__ void __launch_bounds__(64) pdec_intra_kernel(const PUnit *__restrict__ units) {
    __shared__ uint8_t top[16], left[16], pred[256], cpred[2][64], ctop[2][8], cleft[2][8];
    __shared__ int res[256], cres[2][64], tl, ctl[2];
    __shared__ NNPred nn[3];
    __shared__ int32_t Y[64];
    __shared__ long long B[64];
    const int t = threadIdx.x;
    const PUnit &U = units[blockIdx.x];
    const int w = U.w, cw = w / 2;
    for (int i = 0; i < U.nintra; ++i) {
        const int m = U.intra[i];
        const PMB mb = U.mbs[m];
        const int bx = (m % U.mbw) * 16, by = (m / U.mbw) * 16, cbx = bx / 2, cby = by / 2;
        const int ht = by > 0, hl = bx > 0;
        if (t < 16) {
            top[t] = ht ? U.rec[0][(size_t)(by - 1) * w + bx + t] : 0;
            left[t] = hl ? U.rec[0][(size_t)(by + t) * w + bx - 1] : 0;
        } else if (t < 32) {
            const int k = t - 16, pl = k >> 3, q = k & 7;
            ctop[pl][q] = ht ? U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx + q] : 0;
            cleft[pl][q] = hl ? U.rec[1 + pl][(size_t)(cby + q) * cw + cbx - 1] : 0;
        } else if (t == 32) {
            tl = (ht && hl) ? U.rec[0][(size_t)(by - 1) * w + bx - 1] : 128;
            for (int pl = 0; pl < 2; ++pl) ctl[pl] = (ht && hl) ? U.rec[1 + pl][(size_t)(cby - 1) * cw + cbx - 1] : 128;
        }
        __syncthreads();
        if (t == 0) nn[0] = nn_setup(mb.sub, top, left, tl, 16, ht, hl);
        else if (t < 3) nn[t] = nn_setup(mb.sub, ctop[t - 1], cleft[t - 1], ctl[t - 1], 8, ht, hl);
        __syncthreads();
        for (int k = t; k < 256; k += 64) pred[k] = (uint8_t)nn_px(nn[0], top, left, k & 15, k >> 4);
        for (int k = t; k < 128; k += 64) {
            const int pl = k >> 6, p = k & 63;
            cpred[pl][p] = (uint8_t)nn_px(nn[1 + pl], ctop[pl], cleft[pl], p & 7, p >> 3);
        }
        mb_residual(mb, U.coef + mb.coef, U.qp, res, cres, Y, B, t, true);
        for (int k = t; k < 256; k += 64)
            U.rec[0][(size_t)(by + (k >> 4)) * w + bx + (k & 15)] = (uint8_t)clipb(pred[k] + res[k]);
        for (int k = t; k < 128; k += 64) {
            const int pl = k >> 6, p = k & 63;
            U.rec[1 + pl][(size_t)(cby + (p >> 3)) * cw + cbx + (p & 7)] = (uint8_t)clipb(cpred[pl][p] + cres[pl][p]);
        }
        __syncthreads();
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
// ---------------------------------------------------------------------------
using namespace fdvb;

namespace {

thread_local std::string g_derr;

struct PrepTaskD {
    const uint8_t *rec[3];
    uint8_t *G, *B, *H, *J, *U, *V;
    int w, h, ys, cs, border;
};
struct DbTaskD { uint8_t *p; int w, h, qp; };

int round_up(int v, int a) { return (v + a - 1) / a * a; }

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

struct DUnit {
    int w = 0, h = 0, mbw = 0, mbh = 0, cw = 0, ch = 0;
    uint8_t *rec = nullptr;           // tight I420
    RefBuf ref[2];
    int near_i = 0, nref = 0;
    fdvb_tabcache tc{};
    // device copies of the parse
    dec::PMB *d_mbs = nullptr;
    int16_t *d_coef = nullptr;
    int32_t *d_intra = nullptr;
    dec::Leaf *d_leaves[3] = {};
    int32_t *d_ctu[3] = {};
    int16_t *d_icoef[3] = {};
    uint8_t *d_flags[3] = {};
    int *d_prog = nullptr;            // key-frame row progress, three planes
    int pw[3], ph[3], cols[3], rows[3];
    // this frame
    const uint8_t *blob = nullptr;
    size_t blen = 0;
    int intra = 0, rc = 0;
    dec::PFrame pf;
    dec::IPlane ip[3];
};

struct DecEngine {
    int device = 0, border = 32, nsm = 148;
    cudaStream_t st = nullptr;
    std::vector<DUnit> units;
    std::vector<void *> own;
    dk::PUnit *d_pu = nullptr;
    int *d_uoff = nullptr;
    dk::IPlaneD *d_planes = nullptr;
    dk::ITask *d_tasks = nullptr;
    PrepTaskD *d_prep = nullptr;
    DbTaskD *d_db = nullptr;
    int *d_ticket = nullptr;
    unsigned *d_err = nullptr;
    uint8_t *stage = nullptr;         // pinned
    size_t stage_cap = 0;
    ~DecEngine() {
        if (st) cudaStreamSynchronize(st);
        for (void *p : own) cudaFree(p);
        if (stage) cudaFreeHost(stage);
        if (st) cudaStreamDestroy(st);
    }
};

bool ck(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    g_derr = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}
#define DCK(x)                          \
    do {                                \
        if (!ck((x), #x)) return -1;    \
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

int engine_init(DecEngine &E, const std::vector<std::pair<int, int>> &sizes) {
    DCK(cudaGetDevice(&E.device));
    cudaDeviceGetAttribute(&E.nsm, cudaDevAttrMultiProcessorCount, E.device);
    DCK(cudaStreamCreateWithFlags(&E.st, cudaStreamNonBlocking));
    if (upload_dec_tables()) return -1;
    E.border = reference_border();
    const int Bp = E.border + 16;   // allocated border: the checked one plus the filter taps
    const int nu = (int)sizes.size();
    E.units.resize(nu);
    size_t stage = 0;
    int ntasks = 0;
    for (int i = 0; i < nu; ++i) {
        DUnit &u = E.units[i];
        u.w = sizes[i].first;
        u.h = sizes[i].second;
        u.mbw = u.w / 16; u.mbh = u.h / 16; u.cw = u.w / 2; u.ch = u.h / 2;
        const size_t fs = (size_t)u.w * u.h * 3 / 2, nmb = (size_t)u.mbw * u.mbh;
        u.rec = dmalloc<uint8_t>(fs, E.own);
        const int ys = round_up(u.w + 2 * Bp, 64), cs = round_up(u.cw + 2 * Bp, 64);
        const size_t lsz = (size_t)ys * (u.h + 2 * Bp), csz = (size_t)cs * (u.ch + 2 * Bp);
        for (int r = 0; r < 2; ++r) {
            uint8_t *m = dmalloc<uint8_t>(4 * lsz + 2 * csz, E.own);
            if (!m) { g_derr = "device allocation failed"; return -1; }
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
        u.d_mbs = dmalloc<dec::PMB>(nmb, E.own);
        u.d_coef = dmalloc<int16_t>(nmb * 384, E.own);
        u.d_intra = dmalloc<int32_t>(nmb, E.own);
        u.pw[0] = u.w; u.ph[0] = u.h; u.pw[1] = u.pw[2] = u.cw; u.ph[1] = u.ph[2] = u.ch;
        int nprog = 0;
        size_t istage = 0;
        for (int p = 0; p < 3; ++p) {
            u.cols[p] = (u.pw[p] + 63) / 64;
            u.rows[p] = (u.ph[p] + 63) / 64;
            nprog += u.rows[p];
            ntasks += u.rows[p];
            const size_t px = (size_t)u.pw[p] * u.ph[p];
            u.d_leaves[p] = dmalloc<dec::Leaf>(px / 16, E.own);
            u.d_ctu[p] = dmalloc<int32_t>((size_t)u.cols[p] * u.rows[p] + 1, E.own);
            u.d_icoef[p] = dmalloc<int16_t>(px, E.own);
            u.d_flags[p] = dmalloc<uint8_t>(px / 64 + 1, E.own);
            if (!u.d_leaves[p] || !u.d_ctu[p] || !u.d_icoef[p] || !u.d_flags[p]) {
                g_derr = "device allocation failed";
                return -1;
            }
            istage += px / 16 * sizeof(dec::Leaf) + ((size_t)u.cols[p] * u.rows[p] + 1) * 4 + px * 2 + px / 64 + 1024;
        }
        u.d_prog = dmalloc<int>(nprog, E.own);
        const size_t pstage = nmb * sizeof(dec::PMB) + nmb * 384 * 2 + nmb * 4 + 1024;
        stage += std::max(pstage, istage) + fs + 256;
        if (!u.rec || !u.d_mbs || !u.d_coef || !u.d_intra || !u.d_prog) { g_derr = "device allocation failed"; return -1; }
    }
    E.d_pu = dmalloc<dk::PUnit>(nu, E.own);
    E.d_uoff = dmalloc<int>(nu + 1, E.own);
    E.d_planes = dmalloc<dk::IPlaneD>(3 * nu, E.own);
    E.d_tasks = dmalloc<dk::ITask>(ntasks, E.own);
    E.d_prep = dmalloc<PrepTaskD>(nu, E.own);
    E.d_db = dmalloc<DbTaskD>(3 * nu, E.own);
    E.d_ticket = dmalloc<int>(1, E.own);
    E.d_err = dmalloc<unsigned>(1, E.own);
    E.stage_cap = stage + 8192 + (size_t)nu * (sizeof(dk::PUnit) + 3 * sizeof(dk::IPlaneD) + sizeof(PrepTaskD) +
                                               3 * sizeof(DbTaskD) + 8 * 256) + (size_t)ntasks * sizeof(dk::ITask);
    if (!E.d_pu || !E.d_uoff || !E.d_planes || !E.d_tasks || !E.d_prep || !E.d_db || !E.d_ticket || !E.d_err ||
        !ck(cudaHostAlloc(reinterpret_cast<void **>(&E.stage), E.stage_cap, cudaHostAllocDefault), "pinned staging")) {
        if (g_derr.empty()) g_derr = "device allocation failed";
        return -1;
    }
    return 0;
}

// One frame of every unit: parse (a host thread per unit), upload, reconstruct,
// deblock, download into the unit's planes of the output frame (strides
// ostride and ostride / 2), then the decoded frame becomes the reference.
int engine_frame(DecEngine &E, uint8_t *const *outY, uint8_t *const *outU, uint8_t *const *outV, int ostride) {
    const int nu = (int)E.units.size();
    auto parse = [&](int i) {
        DUnit &u = E.units[i];
        if (u.intra) {
            memset(&u.tc, 0, sizeof u.tc);   // tables and history restart at a key frame
            size_t p = 0;
            u.rc = 0;
            for (int pl = 0; pl < 3 && u.rc == 0; ++pl) {
                if (p + 4 > u.blen) { u.rc = -1; break; }
                uint32_t n = 0;
                for (int k = 0; k < 4; ++k) n |= (uint32_t)u.blob[p + k] << (8 * k);
                p += 4;
                if (p + n > u.blen || n < 4) { u.rc = -1; break; }
                u.rc = dec::parse_iplane(u.blob + p, n, u.pw[pl], u.ph[pl], u.ip[pl]);
                p += n;
            }
        } else {
            u.rc = dec::parse_pframe(u.blob, u.blen, u.w, u.h, E.border, &u.tc, u.pf);
        }
    };
    if (nu == 1) {
        parse(0);
    } else {
        std::vector<std::thread> th;
        for (int i = 0; i < nu; ++i) th.emplace_back(parse, i);
        for (auto &t : th) t.join();
    }
    for (int i = 0; i < nu; ++i)
        if (E.units[i].rc) { g_derr = "malformed frame blob"; return -1; }

    uint8_t *sp = E.stage, *const send = E.stage + E.stage_cap;
    bool room = true;
    auto put = [&](const void *src, size_t n) -> const uint8_t * {
        const size_t a = (n + 255) / 256 * 256;
        if (sp + a > send) { room = false; return nullptr; }
        memcpy(sp, src, n);
        const uint8_t *r = sp;
        sp += a;
        return r;
    };
    auto up = [&](void *dst, const void *src, size_t n) -> int {
        if (!n) return 0;
        const uint8_t *s = put(src, n);
        if (!s) { g_derr = "staging buffer too small"; return -1; }
        DCK(cudaMemcpyAsync(dst, s, n, cudaMemcpyHostToDevice, E.st));
        return 0;
    };
    std::vector<dk::PUnit> pu;
    std::vector<int> uoff{0};
    std::vector<dk::IPlaneD> ipl;
    std::vector<dk::ITask> tasks;
    std::vector<DbTaskD> db;
    std::vector<PrepTaskD> prep;
    for (int i = 0; i < nu; ++i) {
        DUnit &u = E.units[i];
        uint8_t *rec[3] = {u.rec, u.rec + (size_t)u.w * u.h, u.rec + (size_t)u.w * u.h + (size_t)u.cw * u.ch};
        if (!u.intra) {
            dec::PFrame &f = u.pf;
            if (up(u.d_mbs, f.mbs.data(), f.mbs.size() * sizeof(dec::PMB)) ||
                up(u.d_coef, f.coef.data(), f.coef.size() * 2) || up(u.d_intra, f.intra.data(), f.intra.size() * 4))
                return -1;
            dk::PUnit d{};
            d.w = u.w; d.h = u.h; d.mbw = u.mbw; d.mbh = u.mbh; d.qp = f.qp;
            for (int p = 0; p < 3; ++p) d.rec[p] = rec[p];
            d.ref[0] = u.ref[u.near_i].rp;
            d.ref[1] = u.nref >= 2 ? u.ref[1 - u.near_i].rp : u.ref[u.near_i].rp;
            d.mbs = u.d_mbs; d.coef = u.d_coef; d.intra = u.d_intra; d.nintra = (int)f.intra.size();
            pu.push_back(d);
            uoff.push_back(uoff.back() + u.mbw * u.mbh);
            for (int p = 0; p < 3; ++p) db.push_back({rec[p], u.pw[p], u.ph[p], f.qp});
        } else {
            int prog = 0;
            for (int p = 0; p < 3; ++p) {
                dec::IPlane &P = u.ip[p];
                if (up(u.d_leaves[p], P.leaves.data(), P.leaves.size() * sizeof(dec::Leaf)) ||
                    up(u.d_ctu[p], P.ctu_first.data(), P.ctu_first.size() * 4) ||
                    up(u.d_icoef[p], P.coef.data(), P.coef.size() * 2) ||
                    up(u.d_flags[p], P.flags.data(), P.flags.size()))
                    return -1;
                dk::IPlaneD d{};
                d.rec = rec[p]; d.w = u.pw[p]; d.h = u.ph[p]; d.cols = u.cols[p]; d.rows = u.rows[p];
                d.leaves = u.d_leaves[p]; d.ctu_first = u.d_ctu[p]; d.coef = u.d_icoef[p]; d.flags = u.d_flags[p];
                d.progress = u.d_prog + prog; d.qp = P.qp;
                prog += u.rows[p];
                ipl.push_back(d);
                db.push_back({rec[p], u.pw[p], u.ph[p], P.qp});
            }
            DCK(cudaMemsetAsync(u.d_prog, 0, sizeof(int) * prog, E.st));
        }
    }
    // key-frame rows in (row, plane) order, so every plane's early rows start first
    {
        int maxr = 0;
        for (auto &p : ipl) maxr = std::max(maxr, p.rows);
        for (int r = 0; r < maxr; ++r)
            for (int p = 0; p < (int)ipl.size(); ++p)
                if (r < ipl[p].rows) tasks.push_back({p, r});
    }
    DCK(cudaMemsetAsync(E.d_err, 0, sizeof(unsigned), E.st));
    if (!pu.empty()) {
        if (up(E.d_pu, pu.data(), pu.size() * sizeof(dk::PUnit)) || up(E.d_uoff, uoff.data(), uoff.size() * 4))
            return -1;
        dk::pdec_inter_kernel<<<uoff.back(), 64, 0, E.st>>>(E.d_pu, E.d_uoff, (int)pu.size());
        dk::pdec_intra_kernel<<<(int)pu.size(), 64, 0, E.st>>>(E.d_pu);
    }
    if (!tasks.empty()) {
        if (up(E.d_planes, ipl.data(), ipl.size() * sizeof(dk::IPlaneD)) ||
            up(E.d_tasks, tasks.data(), tasks.size() * sizeof(dk::ITask)))
            return -1;
        DCK(cudaMemsetAsync(E.d_ticket, 0, sizeof(int), E.st));
        dk::idec_kernel<<<std::min((int)tasks.size(), E.nsm), dk::kINT, 0, E.st>>>(
            E.d_planes, E.d_tasks, (int)tasks.size(), E.d_ticket, E.d_err, 4000000000ull);
    }
    DCK(cudaGetLastError());
    if (up(E.d_db, db.data(), db.size() * sizeof(DbTaskD))) return -1;
    launch_deblock(E.d_db, (int)db.size(), E.st);
    // download, and the decoded frame becomes the nearest reference (load_ref, fdv.h:5183)
    std::vector<uint8_t *> hostbuf(nu);
    for (int i = 0; i < nu; ++i) {
        DUnit &u = E.units[i];
        const size_t fs = (size_t)u.w * u.h * 3 / 2, a = (fs + 255) / 256 * 256;
        if (sp + a > send) { g_derr = "staging buffer too small"; return -1; }
        hostbuf[i] = sp;
        sp += a;
        DCK(cudaMemcpyAsync(hostbuf[i], u.rec, fs, cudaMemcpyDeviceToHost, E.st));
        RefBuf &far = u.ref[1 - u.near_i];
        uint8_t *rec[3] = {u.rec, u.rec + (size_t)u.w * u.h, u.rec + (size_t)u.w * u.h + (size_t)u.cw * u.ch};
        prep.push_back({{rec[0], rec[1], rec[2]}, far.G, far.B, far.H, far.J, far.U, far.V, u.w, u.h, far.rp.ys,
                        far.rp.cs, E.border + 16});
    }
    int maxw = 0, maxh = 0;
    for (auto &u : E.units) { maxw = std::max(maxw, u.w); maxh = std::max(maxh, u.h); }
    if (up(E.d_prep, prep.data(), prep.size() * sizeof(PrepTaskD))) return -1;
    launch_refprep(E.d_prep, (int)prep.size(), maxw, maxh, E.border + 16, E.st);
    DCK(cudaGetLastError());
    unsigned herr = 0;
    DCK(cudaMemcpyAsync(&herr, E.d_err, sizeof herr, cudaMemcpyDeviceToHost, E.st));
    DCK(cudaStreamSynchronize(E.st));
    if (herr) { g_derr = "key-frame wavefront wait timed out"; return -1; }
    for (int i = 0; i < nu; ++i) {
        DUnit &u = E.units[i];
        const uint8_t *s = hostbuf[i];
        for (int y = 0; y < u.h; ++y) memcpy(outY[i] + (size_t)y * ostride, s + (size_t)y * u.w, u.w);
        s += (size_t)u.w * u.h;
        for (int y = 0; y < u.ch; ++y) memcpy(outU[i] + (size_t)y * (ostride / 2), s + (size_t)y * u.cw, u.cw);
        s += (size_t)u.cw * u.ch;
        for (int y = 0; y < u.ch; ++y) memcpy(outV[i] + (size_t)y * (ostride / 2), s + (size_t)y * u.cw, u.cw);
        u.near_i = 1 - u.near_i;
        u.nref = u.intra ? 1 : (u.nref < 2 ? u.nref + 1 : 2);
    }
    return 0;
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

// Decode one stream per band (band b at rows y0[b]) into full W x H frames.
int decode_bands(std::vector<Stream> &bs, const std::vector<int> &y0, int W, int H, int nf, uint8_t *out) {
    std::vector<std::pair<int, int>> sizes;
    for (auto &s : bs) sizes.push_back({s.w, s.h});
    DecEngine E;
    if (engine_init(E, sizes)) return -1;
    const int nu = (int)bs.size(), cw = W / 2, ch = H / 2;
    const size_t fsize = (size_t)W * H + 2 * (size_t)cw * ch;
    std::vector<uint8_t *> oy(nu), ou(nu), ov(nu);
    for (int f = 0; f < nf; ++f) {
        uint8_t *fy = out + (size_t)f * fsize, *fu = fy + (size_t)W * H, *fv = fu + (size_t)cw * ch;
        for (int i = 0; i < nu; ++i) {
            DUnit &u = E.units[i];
            if (!next_blob(bs[i], &u.blob, &u.blen)) { g_derr = "truncated stream"; return -1; }
            u.intra = f == 0 || (bs[i].keyint > 0 && f % bs[i].keyint == 0);
            oy[i] = fy + (size_t)y0[i] * W;
            ou[i] = fu + (size_t)(y0[i] / 2) * cw;
            ov[i] = fv + (size_t)(y0[i] / 2) * cw;
        }
        if (engine_frame(E, oy.data(), ou.data(), ov.data(), W)) return -1;
    }
    return 0;
}

}  // namespace

extern "C" {

const char *fdvd_last_error(void) { return g_derr.c_str(); }

int fdv_video_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h) {
    g_derr.clear();
    Stream s;
    if (!out || !open_stream(in, len, s)) { g_derr = "bad stream header"; return -1; }
    std::vector<Stream> bs{s};
    if (decode_bands(bs, {0}, s.w, s.h, s.nf, out)) return -1;
    if (nframes) *nframes = s.nf;
    if (w) *w = s.w;
    if (h) *h = s.h;
    return 0;
}

int fdv_vtile_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h, int nthreads) {
    (void)nthreads;   // the bands are reconstructed together on the GPU, parsed on a host thread each
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
    if (decode_bands(bs, y0, W, H, nf, out)) return -1;
    if (nframes) *nframes = nf;
    if (w) *w = W;
    if (h) *h = H;
    return 0;
}

}  // extern "C"

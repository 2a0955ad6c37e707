// The learned proposal network on the tensor cores: a tcgen05 BF16 GEMM (fp32
// accumulators in TMEM) drives every convolution and fully connected layer of
// training, forward and backward, with hand-written im2col / col2im / ReLU /
// loss / Adam kernels around it; the fused per-frame inference kernel lives in
// learned_infer.cuh.  Training data are (macroblock, chosen motion vector,
// chosen mode, RD cost) tuples the plain encoder produces.
//
// Layer shapes, the parameter layout and the sample record are in learned.cuh.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/fdv_b200.h"
#include "engine_dev.cuh"
#include "learned.cuh"
#include "learned_infer.cuh"
#include "tc.cuh"

namespace fdvb {
namespace lrn {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// GEMM: D[M][N] = A[M][K] * B[N][K]^T, A and B bf16 row-major (K contiguous).
// One CTA of 4 warps per 128-row tile and up to 256 columns (grid.z tiles N);
// grid.y splits K (the partial products are added atomically).  K tiles of 64
// are staged by cp.async into a 3-deep ring in the canonical operand layout;
// one thread issues four 128xNx16 MMAs per tile and commits them to the
// tile's mbarrier, which frees the stage for the copy three tiles later.
// ---------------------------------------------------------------------------
constexpr int GBM = 128, GBK = 64, GST = 3, GBN = 256;
constexpr int kGemmSmem = GST * (GBM + GBN) * GBK * 2 + 64;

__constant__ LayerGeo c_geo[4] = {kGeo[0], kGeo[1], kGeo[2], kGeo[3]};

enum { EPI_F32 = 0, EPI_F32_ADD = 1, EPI_BIAS_RELU_BF16 = 2, EPI_BIAS_F32 = 3 };

struct GemmArgs {
    const bf16 *A, *B;
    int lda, ldb, M, N, kchunks, mode;
    float *D;
    bf16 *Dh;
    int ldd;
    const float *bias;
    int nbias;
    unsigned *err;
};

__global__ void __launch_bounds__(128, 1) gemm_kernel(const GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *As = sm, *Bs = sm + GST * GBM * GBK * 2;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + GST * (GBM + GBN) * GBK * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + GST);
    volatile int *abort_ = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GBM, n0 = blockIdx.z * GBN;
    const int bn = min(GBN, g.N - n0);
    const uint32_t ncols = tmem_cols(bn);
    const int kbase = blockIdx.y * g.kchunks, nk = g.kchunks;
    if (tid == 0) {
        for (int s = 0; s < GST; ++s) mbar_init(&bar[s], 1);
        *abort_ = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, ncols);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;

    auto load = [&](int kt, int s) {
        const int k0 = (kbase + kt) * GBK;
        uint8_t *as = As + s * GBM * GBK * 2, *bs = Bs + s * GBN * GBK * 2;
        for (int i = tid; i < GBM * 8; i += 128) {
            const int r = i >> 3, kc = i & 7, m = m0 + r;
            const bool ok = m < g.M;
            cpa16(as + umma_off(r, kc * 8), g.A + (size_t)(ok ? m : 0) * g.lda + k0 + kc * 8, ok ? 16 : 0);
        }
        for (int i = tid; i < bn * 8; i += 128) {
            const int r = i >> 3, kc = i & 7;
            cpa16(bs + umma_off(r, kc * 8), g.B + (size_t)(n0 + r) * g.ldb + k0 + kc * 8, 16);
        }
    };
    const uint32_t idesc = umma_idesc_bf16(GBM, bn);
    for (int p = 0; p < GST - 1; ++p) {
        if (p < nk) load(p, p);
        cpa_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % GST;
        cpa_wait<GST - 2>();
        fence_async_smem();
        __syncthreads();
        const int nt = kt + GST - 1;
        if (tid == 0) {
            tc_after_sync();
            const uint32_t a0 = smem_u32(As + s * GBM * GBK * 2), b0 = smem_u32(Bs + s * GBN * GBK * 2);
#pragma unroll
            for (int ks = 0; ks < GBK / 16; ++ks)
                umma_bf16(tmem, umma_desc(a0 + ks * 256, 128, 1024), umma_desc(b0 + ks * 256, 128, 1024), idesc,
                          (kt | ks) != 0);
            umma_commit(&bar[s]);
            // the stage the next copy overwrites was read by tile kt-1
            if (kt >= 1 && nt < nk && !mbar_wait(&bar[(kt - 1) % GST], ((kt - 1) / GST) & 1, g.err)) *abort_ = 1;
        }
        __syncthreads();
        if (*abort_) break;
        if (nt < nk) load(nt, nt % GST);
        cpa_commit();
    }
    if (tid == 0 && !*abort_ && !mbar_wait(&bar[(nk - 1) % GST], ((nk - 1) / GST) & 1, g.err)) *abort_ = 1;
    cpa_wait<0>();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (!*abort_) {
        const int m = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < bn; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (m >= g.M) continue;
            const int n = n0 + c0;
            if (g.mode == EPI_F32) {
                float4 *d = reinterpret_cast<float4 *>(g.D + (size_t)m * g.ldd + n);
#pragma unroll
                for (int q = 0; q < 4; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else if (g.mode == EPI_F32_ADD) {
                float *d = g.D + (size_t)m * g.ldd + n;
#pragma unroll
                for (int q = 0; q < 16; ++q) atomicAdd(d + q, v[q]);
            } else if (g.mode == EPI_BIAS_RELU_BF16) {
                __align__(16) bf16 o[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const float b = n + q < g.nbias ? g.bias[n + q] : 0.f;
                    o[q] = __float2bfloat16_rn(fmaxf(v[q] + b, 0.f));
                }
                uint4 *d = reinterpret_cast<uint4 *>(g.Dh + (size_t)m * g.ldd + n);
                d[0] = reinterpret_cast<const uint4 *>(o)[0];
                d[1] = reinterpret_cast<const uint4 *>(o)[1];
            } else {
                float *d = g.D + (size_t)m * g.ldd + n;
#pragma unroll
                for (int q = 0; q < 16; ++q) d[q] = v[q] + (n + q < g.nbias ? g.bias[n + q] : 0.f);
            }
        }
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_after_sync();
        tmem_free(tmem, ncols);
    }
}

// ---------------------------------------------------------------------------
// Elementwise and data-movement kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ int px_at(const uint8_t *p, int stride, int w, int h, int x, int y) {
    x = x < 0 ? 0 : (x >= w ? w - 1 : x);
    y = y < 0 ? 0 : (y >= h ? h - 1 : y);
    return p[(size_t)y * stride + x];
}
__device__ __forceinline__ bf16 feat(int v) { return __float2bfloat16_rn((float)(v - 128) * (1.f / 64.f)); }
__device__ __forceinline__ bf16 qp_feat(int qp) { return __float2bfloat16_rn((float)(qp - 26) * 0.125f); }

// X[s][y][x][c], one thread per (sample, position).
__global__ void features_kernel(const Sample *__restrict__ S, int n, bf16 *__restrict__ X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kPatch * kPatch) return;
    const int s = i >> 10, y = (i >> 5) & 31, x = i & 31;   // X[s][y][x][4]
    const Sample &q = S[s];
    const int c0 = px_at(q.cur, q.cs, q.w, q.h, q.bx - 8 + x, q.by - 8 + y);
    const int c1 = px_at(q.ref, q.rs, q.w, q.h, q.bx - 8 + x, q.by - 8 + y);
    const int gx = q.bx - 24 + 2 * x, gy = q.by - 24 + 2 * y;
    const int c2 = (px_at(q.cur, q.cs, q.w, q.h, gx, gy) + px_at(q.cur, q.cs, q.w, q.h, gx + 1, gy) +
                    px_at(q.cur, q.cs, q.w, q.h, gx, gy + 1) + px_at(q.cur, q.cs, q.w, q.h, gx + 1, gy + 1) + 2) >> 2;
    const int c3 = (px_at(q.ref, q.rs, q.w, q.h, gx, gy) + px_at(q.ref, q.rs, q.w, q.h, gx + 1, gy) +
                    px_at(q.ref, q.rs, q.w, q.h, gx, gy + 1) + px_at(q.ref, q.rs, q.w, q.h, gx + 1, gy + 1) + 2) >> 2;
    __align__(8) bf16 o[4] = {feat(c0), feat(c1), feat(c2), feat(c3)};
    *reinterpret_cast<uint2 *>(X + (size_t)i * 4) = *reinterpret_cast<const uint2 *>(o);
}

// col[(b*So + oy)*So + ox][k] for a 3x3 stride-2 pad-1 convolution of
// X[b][Si][Si][Cin]; k >= 9*Cin is zero.  One thread per 8-element chunk.
// (With S: the first convolution, whose column kQpCol is the sample's quantiser.)
__global__ void im2col_kernel(const bf16 *__restrict__ X, int nb, int si, int cin, int kp, bf16 *__restrict__ col,
                              const Sample *__restrict__ S) {
    const int so = si / 2, kc8 = kp / 8;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nb * so * so * kc8) return;
    const int ch = (int)(i % kc8);
    const long long row = i / kc8;
    const int ox = (int)(row % so), oy = (int)((row / so) % so), b = (int)(row / ((long long)so * so));
    __align__(16) bf16 o[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int k = ch * 8 + j;
        bf16 v = __float2bfloat16_rn(0.f);
        if (k < 9 * cin) {
            const int tap = k / cin, c = k - tap * cin, ky = tap / 3, kx = tap - ky * 3;
            const int y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
            if (y >= 0 && y < si && x >= 0 && x < si) v = X[(((size_t)b * si + y) * si + x) * cin + c];
        } else if (S && k == kQpCol) {
            v = qp_feat(S[b].qp);
        }
        o[j] = v;
    }
    *reinterpret_cast<uint4 *>(col + row * kp + ch * 8) = *reinterpret_cast<const uint4 *>(o);
}

// dX[b][y][x][c] = sum over the taps that read (y, x) of dcol.
__global__ void col2im_kernel(const float *__restrict__ dcol, int ldc, int nb, int si, int cin,
                              float *__restrict__ dX) {
    const int so = si / 2;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nb * si * si * cin) return;
    const int c = (int)(i % cin);
    const long long p = i / cin;
    const int x = (int)(p % si), y = (int)((p / si) % si), b = (int)(p / ((long long)si * si));
    float acc = 0.f;
    for (int ky = 0; ky < 3; ++ky) {
        const int ty = y + 1 - ky;
        if (ty < 0 || (ty & 1) || (ty >> 1) >= so) continue;
        for (int kx = 0; kx < 3; ++kx) {
            const int tx = x + 1 - kx;
            if (tx < 0 || (tx & 1) || (tx >> 1) >= so) continue;
            const size_t row = ((size_t)b * so + (ty >> 1)) * so + (tx >> 1);
            acc += dcol[row * ldc + (ky * 3 + kx) * cin + c];
        }
    }
    dX[i] = acc;
}

// dZ = dY where the ReLU output was positive.  Writes dZ (bf16, row-major,
// columns N..ldz-1 zero) and/or its transpose dZT[N][ldt], and adds the column
// sums into db.  32x32 tiles, 32x8 threads.
__global__ void relu_bwd_kernel(const bf16 *__restrict__ Y, int ldy, const float *__restrict__ dY, int ldg, int M,
                                int N, bf16 *__restrict__ dZ, int ldz, bf16 *__restrict__ dZT, int ldt,
                                float *__restrict__ db) {
    __shared__ float t[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y, c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int c = c0 + tx;
    float cs = 0.f;
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + ty + 8 * i;
        float z = 0.f;
        if (r < M && c < N && __bfloat162float(Y[(size_t)r * ldy + c]) > 0.f) z = dY[(size_t)r * ldg + c];
        t[ty + 8 * i][tx] = z;
        cs += z;
        if (dZ && r < M && c < ldz) dZ[(size_t)r * ldz + c] = __float2bfloat16_rn(z);
    }
    __shared__ float csum[8][32];
    csum[ty][tx] = cs;
    __syncthreads();
    if (db && ty == 0 && c < N) {
        float s = 0.f;
        for (int k = 0; k < 8; ++k) s += csum[k][tx];
        atomicAdd(&db[c], s);
    }
    if (dZT)
        for (int i = 0; i < 4; ++i) {
            const int cc = c0 + ty + 8 * i, r = r0 + tx;
            if (cc < N && r < M) dZT[(size_t)cc * ldt + r] = __float2bfloat16_rn(t[tx][ty + 8 * i]);
        }
}

// out[C][R] = in[R][C]^T (bf16), 32x32 tiles.
__global__ void transpose_kernel(const bf16 *__restrict__ in, int ldi, int R, int C, bf16 *__restrict__ out,
                                 int ldo) {
    __shared__ bf16 t[32][34];
    const int tx = threadIdx.x, ty = threadIdx.y, c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + ty + 8 * i, c = c0 + tx;
        t[ty + 8 * i][tx] = (r < R && c < C) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int i = 0; i < 4; ++i) {
        const int c = c0 + ty + 8 * i, r = r0 + tx;
        if (c < C && r < R) out[(size_t)c * ldo + r] = t[tx][ty + 8 * i];
    }
}

__device__ __forceinline__ float sl1(float d, float &g) {
    constexpr float kD = 0.25f;
    const float a = fabsf(d);
    if (a < kD) { g = d / kD; return 0.5f * d * d / kD; }
    g = d > 0.f ? 1.f : -1.f;
    return a - 0.5f * kD;
}

// Per sample: cross-entropy of the mode logits plus a relaxed winner-takes-all
// smooth-L1 over the four MV hypotheses; gradients of the batch mean.
// loss[s] = {ce, mv}.  dO[s][0..63] (bf16, zero past 11) and dOT[16][ldt].
__global__ void loss_kernel(const float *__restrict__ O, const Sample *__restrict__ S, int n, float scale,
                            float *__restrict__ loss, bf16 *__restrict__ dO, bf16 *__restrict__ dOT, int ldt,
                            float *__restrict__ db) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float *o = O + (size_t)s * kOutPad;
    const Sample &q = S[s];
    float g[kOutPad];
    for (int j = 0; j < kOutPad; ++j) g[j] = 0.f;
    // mode
    const float l0 = o[8], l1 = o[9], l2 = o[10];
    const float mx = fmaxf(l0, fmaxf(l1, l2));
    const float e0 = expf(l0 - mx), e1 = expf(l1 - mx), e2 = expf(l2 - mx), es = e0 + e1 + e2;
    const float lt = q.cls == 0 ? l0 : (q.cls == 1 ? l1 : l2);
    const float ce = (logf(es) + mx - lt) * q.wgt;
    g[8] = (e0 / es - (q.cls == 0)) * q.wgt;
    g[9] = (e1 / es - (q.cls == 1)) * q.wgt;
    g[10] = (e2 / es - (q.cls == 2)) * q.wgt;
    // motion
    float mv = 0.f;
    if (q.has_mv) {
        constexpr float kEps = 0.05f;
        float e[kMvHyp], gx[kMvHyp], gy[kMvHyp];
        int best = 0;
        for (int k = 0; k < kMvHyp; ++k) {
            e[k] = sl1(o[2 * k] - q.tx, gx[k]) + sl1(o[2 * k + 1] - q.ty, gy[k]);
            if (e[k] < e[best]) best = k;
        }
        for (int k = 0; k < kMvHyp; ++k) {
            const float a = (k == best ? 1.f : kEps) * q.wgt;
            mv += a * e[k];
            g[2 * k] = a * gx[k];
            g[2 * k + 1] = a * gy[k];
        }
    }
    loss[2 * s] = ce;
    loss[2 * s + 1] = mv;
    for (int j = 0; j < 64; ++j) dO[(size_t)s * 64 + j] = __float2bfloat16_rn(j < kOutPad ? g[j] * scale : 0.f);
    for (int j = 0; j < kOutPad; ++j) dOT[(size_t)j * ldt + s] = __float2bfloat16_rn(g[j] * scale);
    for (int j = 0; j < kOut; ++j) atomicAdd(&db[j], g[j] * scale);
}

struct AdamSeg {
    int off, cnt, layer, is_bias;
};
struct AdamArgs {
    float *w, *m, *v;
    const float *dWT[4], *db[4];
    bf16 *Wb[4], *WTb[4];
    AdamSeg seg[8];
    float lr, b1, b2, eps, c1, c2;   // c1 = 1 - b1^t, c2 = 1 - b2^t
};

__global__ void adam_kernel(const AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kNParams) return;
    int sg = 0;
    while (sg < 7 && i >= a.seg[sg + 1].off) ++sg;
    const AdamSeg &S = a.seg[sg];
    const int l = S.layer, j = i - S.off;
    const LayerGeo &G = c_geo[l];
    float gr;
    int o = 0, k = 0;
    if (S.is_bias) {
        gr = a.db[l][j];
    } else {
        o = j / G.k;
        k = j - o * G.k;
        gr = a.dWT[l][(size_t)k * G.gn + o];
    }
    const float m = a.b1 * a.m[i] + (1.f - a.b1) * gr;
    const float v = a.b2 * a.v[i] + (1.f - a.b2) * gr * gr;
    a.m[i] = m;
    a.v[i] = v;
    const float w = a.w[i] - a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
    a.w[i] = w;
    if (!S.is_bias) {
        const bf16 wb = __float2bfloat16_rn(w);
        a.Wb[l][(size_t)o * G.kp + k] = wb;
        if (a.WTb[l]) a.WTb[l][(size_t)k * G.nr + o] = wb;
    }
}

// bf16 copies of the master weights (forward operand W[gn][kp], and the
// transposed WT[kp][nr] of the input-gradient GEMMs); pads stay zero.
__global__ void wcopy_kernel(const float *__restrict__ w, int layer, int woff, bf16 *__restrict__ Wb,
                             bf16 *__restrict__ WTb) {
    const LayerGeo &G = c_geo[layer];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= G.cout * G.k) return;
    const int o = j / G.k, k = j - o * G.k;
    const bf16 wb = __float2bfloat16_rn(w[woff + j]);
    Wb[(size_t)o * G.kp + k] = wb;
    if (WTb) WTb[(size_t)k * G.nr + o] = wb;
}

// Output rows -> per-macroblock proposals: softmax confidence of the mode
// logits against the threshold; hypotheses to quarter-pels, clamped to the range.
__global__ void hint_kernel(const float *__restrict__ O, int n, float conf, int lim, Hint *__restrict__ H) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float *o = O + (size_t)s * kOutPad;
    Hint h;
    for (int k = 0; k < kMvHyp; ++k) {
        int x = __float2int_rn(o[2 * k] * 16.f), y = __float2int_rn(o[2 * k + 1] * 16.f);
        x = min(max(x, -lim), lim);
        y = min(max(y, -lim), lim);
        h.mv[k] = make_short2((short)x, (short)y);
    }
    const float mx = fmaxf(o[8], fmaxf(o[9], o[10]));
    const float e0 = expf(o[8] - mx), e1 = expf(o[9] - mx), e2 = expf(o[10] - mx), es = e0 + e1 + e2;
    const int c = (o[8] >= o[9] && o[8] >= o[10]) ? 0 : (o[9] >= o[10] ? 1 : 2);
    const float p = (c == 0 ? e0 : (c == 1 ? e1 : e2)) / es;
    h.cls = p >= conf ? c : -1;
    H[s] = h;
}

}  // namespace lrn
}  // namespace fdvb

using namespace fdvb;
using namespace fdvb::lrn;

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

thread_local std::string g_lerr;
void lerr(const std::string &m) { g_lerr = m; }
bool cu_ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    lerr(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}
#define LCK(x)                           \
    do {                                 \
        if (!cu_ok((x), #x)) return -1;  \
    } while (0)

template <class T>
T *dalloc(size_t n, std::vector<void *> &owned) {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
    owned.push_back(p);
    return static_cast<T *>(p);
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

struct fdvl_net {
    int device = 0, maxb = 0;     // batch capacity (multiple of 64)
    int bank_n = 0, bw = 0, bh = 0;
    cudaStream_t st = nullptr;
    std::vector<void *> owned;
    uint8_t *bank = nullptr;      // bank_n luma planes of bw x bh
    float *w = nullptr, *m = nullptr, *v = nullptr;
    int t = 0;                    // Adam steps taken
    bf16 *Wb[4] = {}, *WTb[4] = {};
    // batch buffers
    Sample *S = nullptr;
    Sample *S_h[2] = {};
    cudaEvent_t S_ev[2] = {};
    int S_cur = 0;
    bf16 *X0 = nullptr, *col[3] = {}, *Y[3] = {}, *colT[3] = {}, *Y3T = nullptr;
    float *O = nullptr, *loss = nullptr, *loss_h = nullptr;
    bf16 *dO = nullptr, *dOT = nullptr, *dZ[3] = {}, *dZT[3] = {};
    float *dWT[4] = {}, *db[4] = {}, *dY[3] = {}, *dcol[2] = {};
    unsigned *err = nullptr;
    uint8_t *wimg = nullptr;      // canonical weight images of the fused inference kernel
    unsigned long long *iprof = nullptr;   // fused-inference phase profile (when enabled)
    float *outf = nullptr;        // fused-inference outputs (tests)
    Hint *hints = nullptr;        // fused-inference hints (tests)
    int nsm = 148;
};

namespace {

int gemm(fdvl_net *n, cudaStream_t st, const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, int mode,
         float *D, bf16 *Dh, int ldd, const float *bias, int nbias, int nsplit = 1) {
    if (K % (GBK * nsplit) || N % 16 || M <= 0) { lerr("gemm: bad shape"); return -1; }
    GemmArgs g{A, B, lda, ldb, M, N, K / GBK / nsplit, mode, D, Dh, ldd, bias, nbias, n->err};
    dim3 grid((M + GBM - 1) / GBM, nsplit, (N + GBN - 1) / GBN);
    gemm_kernel<<<grid, 128, kGemmSmem, st>>>(g);
    return cu_ok(cudaGetLastError(), "gemm launch") ? 0 : -1;
}

int split_for(int K) {   // K splits for the long reductions of the weight gradients
    int s = 1;
    while (s < 128 && (K / GBK) % (2 * s) == 0 && K / GBK / (2 * s) >= 8) s *= 2;
    return s;
}

// Forward of nb samples (device records S): outputs into n->O.
int forward(fdvl_net *n, const Sample *S, int nb, cudaStream_t st) {
    features_kernel<<<(nb * 1024 + 255) / 256, 256, 0, st>>>(S, nb, n->X0);
    const bf16 *x = n->X0;
    for (int l = 0; l < 3; ++l) {
        const LayerGeo &G = kGeo[l];
        const int so = G.sin / 2, rows = nb * so * so;
        const long long chunks = (long long)rows * (G.kp / 8);
        im2col_kernel<<<(unsigned)((chunks + 255) / 256), 256, 0, st>>>(x, nb, G.sin, G.cin, G.kp, n->col[l],
                                                                        l == 0 ? S : nullptr);
        if (gemm(n, st, n->col[l], G.kp, n->Wb[l], G.kp, rows, G.gn, G.kp, EPI_BIAS_RELU_BF16, nullptr, n->Y[l],
                 G.gn, n->w + b_off(l), G.cout))
            return -1;
        x = n->Y[l];
    }
    const LayerGeo &F = kGeo[3];
    if (gemm(n, st, n->Y[2], F.kp, n->Wb[3], F.kp, nb, F.gn, F.kp, EPI_BIAS_F32, n->O, nullptr, kOutPad,
             n->w + b_off(3), F.cout))
        return -1;
    return cu_ok(cudaGetLastError(), "forward") ? 0 : -1;
}

// Loss and gradients of the batch mean (nb a multiple of 64): dWT / db.
int backward(fdvl_net *n, int nb) {
    cudaStream_t st = n->st;
    const dim3 tb(32, 8);
    for (int l = 0; l < 4; ++l) {
        cudaMemsetAsync(n->dWT[l], 0, sizeof(float) * kGeo[l].kp * kGeo[l].gn, st);
        cudaMemsetAsync(n->db[l], 0, sizeof(float) * kGeo[l].gn, st);
    }
    loss_kernel<<<(nb + 127) / 128, 128, 0, st>>>(n->O, n->S, nb, 1.f / nb, n->loss, n->dO, n->dOT, nb, n->db[3]);
    // fully connected layer
    {
        const LayerGeo &F = kGeo[3];
        transpose_kernel<<<dim3(F.kp / 32, (nb + 31) / 32), tb, 0, st>>>(n->Y[2], F.kp, nb, F.kp, n->Y3T, nb);
        if (gemm(n, st, n->Y3T, nb, n->dOT, nb, F.kp, F.gn, nb, EPI_F32_ADD, n->dWT[3], nullptr, F.gn, nullptr, 0,
                 split_for(nb)))
            return -1;
        if (gemm(n, st, n->dO, 64, n->WTb[3], F.nr, nb, F.kp, F.nr, EPI_F32, n->dY[2], nullptr, F.kp, nullptr, 0))
            return -1;
    }
    for (int l = 2; l >= 0; --l) {
        const LayerGeo &G = kGeo[l];
        const int so = G.sin / 2, rows = nb * so * so;
        // dY[l] is the gradient at this layer's (post-ReLU) output, [rows][gn]
        relu_bwd_kernel<<<dim3((std::max(G.gn, G.nr) + 31) / 32, (rows + 31) / 32), tb, 0, st>>>(
            n->Y[l], G.gn, n->dY[l], G.gn, rows, G.cout, l > 0 ? n->dZ[l] : nullptr, G.nr, n->dZT[l], rows, n->db[l]);
        transpose_kernel<<<dim3(G.kp / 32, (rows + 31) / 32), tb, 0, st>>>(n->col[l], G.kp, rows, G.kp, n->colT[l],
                                                                            rows);
        if (gemm(n, st, n->colT[l], rows, n->dZT[l], rows, G.kp, G.gn, rows, EPI_F32_ADD, n->dWT[l], nullptr, G.gn,
                 nullptr, 0, split_for(rows)))
            return -1;
        if (l > 0) {
            if (gemm(n, st, n->dZ[l], G.nr, n->WTb[l], G.nr, rows, G.kp, G.nr, EPI_F32, n->dcol[l - 1], nullptr, G.kp,
                     nullptr, 0))
                return -1;
            const long long cnt = (long long)nb * G.sin * G.sin * G.cin;
            col2im_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(n->dcol[l - 1], G.kp, nb, G.sin, G.cin,
                                                                         n->dY[l - 1]);
        }
    }
    return cu_ok(cudaGetLastError(), "backward") ? 0 : -1;
}

}  // namespace

namespace {

void net_free(fdvl_net *n) {
    if (!n) return;
    cudaSetDevice(n->device);
    if (n->st) cudaStreamSynchronize(n->st);
    for (void *p : n->owned) cudaFree(p);
    if (n->iprof) cudaFree(n->iprof);
    for (int i = 0; i < 2; ++i) {
        if (n->S_h[i]) cudaFreeHost(n->S_h[i]);
        if (n->S_ev[i]) cudaEventDestroy(n->S_ev[i]);
    }
    if (n->loss_h) cudaFreeHost(n->loss_h);
    if (n->st) cudaStreamDestroy(n->st);
    delete n;
}

// Stage nb samples through a pinned buffer (two, alternating) into n->S.
int put_samples(fdvl_net *n, const Sample *s, int nb) {
    const int k = n->S_cur;
    LCK(cudaEventSynchronize(n->S_ev[k]));
    memcpy(n->S_h[k], s, sizeof(Sample) * nb);
    LCK(cudaMemcpyAsync(n->S, n->S_h[k], sizeof(Sample) * nb, cudaMemcpyHostToDevice, n->st));
    LCK(cudaEventRecord(n->S_ev[k], n->st));
    n->S_cur ^= 1;
    return 0;
}

int check_err(fdvl_net *n) {
    unsigned e = 0;
    LCK(cudaMemcpyAsync(&e, n->err, sizeof e, cudaMemcpyDeviceToHost, n->st));
    LCK(cudaStreamSynchronize(n->st));
    if (e) {
        lerr("device error word " + std::to_string(e) + " (an MMA completion wait timed out)");
        cudaMemsetAsync(n->err, 0, sizeof(unsigned), n->st);
        return -1;
    }
    return 0;
}

// fdvl_sample (public, bank-relative) -> Sample (device pointers).
bool to_sample(const fdvl_net *n, const fdvl_sample &a, Sample &s) {
    if (a.cur < 0 || a.cur >= n->bank_n || a.ref < 0 || a.ref >= n->bank_n) return false;
    if (a.mbx < 0 || a.mby < 0 || a.mbx * 16 >= n->bw || a.mby * 16 >= n->bh) return false;
    if (a.cls < 0 || a.cls > 2) return false;
    const size_t plane = (size_t)n->bw * n->bh;
    s.cur = n->bank + plane * a.cur;
    s.ref = n->bank + plane * a.ref;
    s.cs = s.rs = n->bw;
    s.w = n->bw;
    s.h = n->bh;
    s.bx = a.mbx * 16;
    s.by = a.mby * 16;
    s.cls = a.cls;
    s.has_mv = a.has_mv;
    s.tx = (float)a.mvx / 16.f;
    s.ty = (float)a.mvy / 16.f;
    s.wgt = a.weight;
    s.qp = a.qp;
    return true;
}

int adam_step(fdvl_net *n, float lr) {
    AdamArgs a{};
    a.w = n->w;
    a.m = n->m;
    a.v = n->v;
    for (int l = 0; l < 4; ++l) {
        a.dWT[l] = n->dWT[l];
        a.db[l] = n->db[l];
        a.Wb[l] = n->Wb[l];
        a.WTb[l] = n->WTb[l];
        a.seg[2 * l] = {w_off(l), kGeo[l].cout * kGeo[l].k, l, 0};
        a.seg[2 * l + 1] = {b_off(l), kGeo[l].cout, l, 1};
    }
    ++n->t;
    a.lr = lr;
    a.b1 = 0.9f;
    a.b2 = 0.999f;
    a.eps = 1e-8f;
    a.c1 = (float)(1.0 - std::pow(0.9, n->t));
    a.c2 = (float)(1.0 - std::pow(0.999, n->t));
    adam_kernel<<<(kNParams + 255) / 256, 256, 0, n->st>>>(a);
    return cu_ok(cudaGetLastError(), "adam") ? 0 : -1;
}

int refresh_bf16(fdvl_net *n) {
    for (int l = 0; l < 4; ++l) {
        const int cnt = kGeo[l].cout * kGeo[l].k;
        wcopy_kernel<<<(cnt + 255) / 256, 256, 0, n->st>>>(n->w, l, w_off(l), n->Wb[l], n->WTb[l]);
    }
    prep_infer_weights<<<(160 * 576 + 255) / 256, 256, 0, n->st>>>(n->w, n->wimg);
    return cu_ok(cudaGetLastError(), "wcopy") ? 0 : -1;
}

int fused_infer(fdvl_net *n, const Sample *S, int nb, float3 conf, int lim, Hint *hints, float *out, unsigned *err,
                cudaStream_t st) {
    InferW W;
    W.img = n->wimg;
    for (int l = 0; l < 4; ++l) W.b[l] = n->w + b_off(l);
    W.prof = n->iprof;
    infer_kernel<<<std::min(nb, n->nsm), INT, kInferSmem, st>>>(S, nb, W, conf, lim, hints, out, err);
    return cu_ok(cudaGetLastError(), "fused inference") ? 0 : -1;
}

int load_batch(fdvl_net *n, const fdvl_sample *s, int nb, std::vector<Sample> &tmp) {
    tmp.resize(nb);
    for (int i = 0; i < nb; ++i)
        if (!to_sample(n, s[i], tmp[i])) { lerr("sample " + std::to_string(i) + " out of range"); return -1; }
    return put_samples(n, tmp.data(), nb);
}

}  // namespace

namespace fdvb {

fdvl_net *lrn_create(int device, int max_batch, int bank_frames, int w, int h) {
    const bool train = bank_frames > 0;
    if (cudaSetDevice(device) != cudaSuccess) { lerr("fdvl_create: no such device"); return nullptr; }
    fdvl_net *n = new fdvl_net;
    n->device = device;
    n->maxb = round_up(max_batch, 64);
    n->bank_n = bank_frames;
    n->bw = w;
    n->bh = h;
    auto &o = n->owned;
    const size_t B = n->maxb;
    bool ok = cudaStreamCreateWithFlags(&n->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem) == cudaSuccess;
    if (ok) {
        // An encoder engine's network (no training bank) only runs the fused
        // inference: sample descriptors, weights and the error word.  The
        // per-macroblock layer activations of the layered forward and of
        // training (tens of kilobytes per macroblock) exist only with a bank.
        n->w = dalloc<float>(kNParams, o);
        n->wimg = dalloc<uint8_t>(kWImage, o);
        ok = ok && n->wimg &&
             cudaFuncSetAttribute(infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem) ==
                 cudaSuccess &&
             cudaDeviceGetAttribute(&n->nsm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess;
        n->S = dalloc<Sample>(B, o);
        n->err = dalloc<unsigned>(1, o);
        ok = ok && n->w && n->S && n->err;
        for (int l = 0; l < 4; ++l) {
            const LayerGeo &G = kGeo[l];
            n->Wb[l] = dalloc<bf16>((size_t)G.gn * G.kp, o);
            ok = ok && n->Wb[l];
        }
        if (train) {
            n->outf = dalloc<float>(B * kOutPad, o);
            n->hints = dalloc<Hint>(B, o);
            n->X0 = dalloc<bf16>(B * 1024 * kChan, o);
            n->O = dalloc<float>(B * kOutPad, o);
            ok = ok && n->outf && n->hints && n->X0 && n->O;
            for (int l = 0; l < 3; ++l) {
                const size_t rows = B * pos_per_mb(l);
                n->col[l] = dalloc<bf16>(rows * kGeo[l].kp, o);
                n->Y[l] = dalloc<bf16>(rows * kGeo[l].gn, o);
                ok = ok && n->col[l] && n->Y[l];
            }
        }
        if (train) {
            n->bank = dalloc<uint8_t>((size_t)w * h * bank_frames, o);
            n->m = dalloc<float>(kNParams, o);
            n->v = dalloc<float>(kNParams, o);
            for (int l = 0; l < 4; ++l) {
                const LayerGeo &G = kGeo[l];
                n->WTb[l] = l > 0 ? dalloc<bf16>((size_t)G.kp * G.nr, o) : nullptr;
                n->dWT[l] = dalloc<float>((size_t)G.kp * G.gn, o);
                n->db[l] = dalloc<float>(G.gn, o);
                ok = ok && n->dWT[l] && n->db[l] && (l == 0 || n->WTb[l]);
            }
            for (int l = 0; l < 3; ++l) {
                const LayerGeo &G = kGeo[l];
                const size_t rows = B * pos_per_mb(l);
                n->colT[l] = dalloc<bf16>(rows * G.kp, o);
                n->dZT[l] = dalloc<bf16>(rows * G.cout, o);
                n->dZ[l] = l > 0 ? dalloc<bf16>(rows * G.nr, o) : nullptr;
                n->dY[l] = dalloc<float>(rows * G.gn, o);
                ok = ok && n->colT[l] && n->dZT[l] && n->dY[l] && (l == 0 || n->dZ[l]);
            }
            n->dcol[0] = dalloc<float>(B * pos_per_mb(1) * kGeo[1].kp, o);
            n->dcol[1] = dalloc<float>(B * pos_per_mb(2) * kGeo[2].kp, o);
            n->Y3T = dalloc<bf16>(B * kGeo[3].kp, o);
            n->loss = dalloc<float>(B * 2, o);
            n->dO = dalloc<bf16>(B * 64, o);
            n->dOT = dalloc<bf16>(B * kOutPad, o);
            ok = ok && n->bank && n->m && n->v && n->dcol[0] && n->dcol[1] && n->Y3T && n->loss && n->dO && n->dOT;
        }
        for (int i = 0; i < 2 && ok; ++i)
            ok = cudaHostAlloc(reinterpret_cast<void **>(&n->S_h[i]), sizeof(Sample) * B, cudaHostAllocDefault) ==
                     cudaSuccess &&
                 cudaEventCreateWithFlags(&n->S_ev[i], cudaEventDisableTiming) == cudaSuccess &&
                 cudaEventRecord(n->S_ev[i], n->st) == cudaSuccess;
        ok = ok && (!train || cudaHostAlloc(reinterpret_cast<void **>(&n->loss_h), sizeof(float) * B * 2,
                                            cudaHostAllocDefault) == cudaSuccess);
    }
    if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
        lerr("fdvl: device allocation failed");
        net_free(n);
        return nullptr;
    }
    return n;
}


// Per-frame inference for the encoder: one sample per macroblock of every
// listed unit (pu[i] = {unit, first macroblock index}), on the caller's stream.
__global__ void unit_samples_kernel(const UnitDev *__restrict__ U, const int2 *__restrict__ pu, int np, int total,
                                    Sample *__restrict__ S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int k = 0;
    while (k + 1 < np && i >= pu[k + 1].y) ++k;
    const UnitDev &u = U[pu[k].x];
    const int mb = i - pu[k].y;
    Sample q{};
    q.cur = u.cur[0];
    q.cs = u.w;
    q.ref = u.lref ? u.lref : u.ref[0].G;
    q.rs = u.lref ? u.lrs : u.ref[0].ys;
    q.w = u.w;
    q.h = u.h;
    q.bx = (mb % u.mbw) * 16;
    q.by = (mb / u.mbw) * 16;
    q.qp = u.qp;
    S[i] = q;
}

int lrn_infer_units(fdvl_net *n, const UnitDev *units, const int2 *pu, int np, int total, float3 conf, int lim,
                    Hint *hints, unsigned *err, cudaStream_t st) {
    if (total > n->maxb) { lerr("learned inference: more macroblocks than the network was sized for"); return -1; }
    unit_samples_kernel<<<(total + 127) / 128, 128, 0, st>>>(units, pu, np, total, n->S);
    return fused_infer(n, n->S, total, conf, lim, hints, nullptr, err, st);
}

int lrn_max_batch(const fdvl_net *n) { return n->maxb; }
unsigned *lrn_err_word(fdvl_net *n) { return n->err; }

}  // namespace fdvb

extern "C" {

const char *fdvl_last_error(void) { return g_lerr.c_str(); }

int fdvl_nparams(void) { return kNParams; }

fdvl_net *fdvl_create(int device, int max_batch, int bank_frames, int w, int h) {
    if (max_batch < 64 || bank_frames < 1 || w < 16 || h < 16 || w % 16 || h % 16) {
        lerr("fdvl_create: bad arguments");
        return nullptr;
    }
    return fdvb::lrn_create(device, max_batch, bank_frames, w, h);
}

void fdvl_destroy(fdvl_net *n) { net_free(n); }

int fdvl_set_params(fdvl_net *n, const float *p) {
    if (!n || !p) { lerr("fdvl_set_params: null"); return -1; }
    cudaSetDevice(n->device);
    LCK(cudaMemcpyAsync(n->w, p, sizeof(float) * kNParams, cudaMemcpyHostToDevice, n->st));
    if (n->m) LCK(cudaMemsetAsync(n->m, 0, sizeof(float) * kNParams, n->st));
    if (n->v) LCK(cudaMemsetAsync(n->v, 0, sizeof(float) * kNParams, n->st));
    n->t = 0;
    if (refresh_bf16(n)) return -1;
    LCK(cudaStreamSynchronize(n->st));
    return 0;
}

int fdvl_get_params(fdvl_net *n, float *p) {
    if (!n || !p) { lerr("fdvl_get_params: null"); return -1; }
    cudaSetDevice(n->device);
    LCK(cudaMemcpyAsync(p, n->w, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, n->st));
    LCK(cudaStreamSynchronize(n->st));
    return 0;
}

int fdvl_bank_put(fdvl_net *n, int slot, const uint8_t *y) {
    if (!n || !y || slot < 0 || slot >= n->bank_n) { lerr("fdvl_bank_put: bad slot"); return -1; }
    cudaSetDevice(n->device);
    LCK(cudaMemcpyAsync(n->bank + (size_t)n->bw * n->bh * slot, y, (size_t)n->bw * n->bh, cudaMemcpyHostToDevice,
                        n->st));
    LCK(cudaStreamSynchronize(n->st));
    return 0;
}

int fdvl_features(fdvl_net *n, const fdvl_sample *s, int nb, float *x) {
    if (!n || !s || !x || nb < 1 || nb > n->maxb) { lerr("fdvl_features: bad arguments"); return -1; }
    cudaSetDevice(n->device);
    std::vector<Sample> tmp;
    if (load_batch(n, s, nb, tmp)) return -1;
    features_kernel<<<(nb * 1024 + 255) / 256, 256, 0, n->st>>>(n->S, nb, n->X0);
    std::vector<bf16> h((size_t)nb * 1024 * kChan);
    LCK(cudaMemcpyAsync(h.data(), n->X0, h.size() * sizeof(bf16), cudaMemcpyDeviceToHost, n->st));
    LCK(cudaStreamSynchronize(n->st));
    for (size_t i = 0; i < h.size(); ++i) x[i] = __bfloat162float(h[i]);
    return 0;
}

int fdvl_forward(fdvl_net *n, const fdvl_sample *s, int nb, float *out) {
    if (!n || !s || !out || nb < 1 || nb > n->maxb) { lerr("fdvl_forward: bad arguments"); return -1; }
    cudaSetDevice(n->device);
    std::vector<Sample> tmp;
    if (load_batch(n, s, nb, tmp) || forward(n, n->S, nb, n->st)) return -1;
    LCK(cudaMemcpyAsync(out, n->O, sizeof(float) * kOutPad * nb, cudaMemcpyDeviceToHost, n->st));
    return check_err(n);
}

int fdvl_infer_profile(fdvl_net *n, int enable, unsigned long long *out16) {
    if (!n) return -1;
    cudaSetDevice(n->device);
    if (enable && !n->iprof) {
        LCK(cudaMalloc(&n->iprof, 16 * sizeof(unsigned long long)));
        LCK(cudaMemset(n->iprof, 0, 16 * sizeof(unsigned long long)));
    }
    if (out16 && n->iprof) {
        LCK(cudaStreamSynchronize(n->st));
        LCK(cudaMemcpy(out16, n->iprof, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        LCK(cudaMemset(n->iprof, 0, 16 * sizeof(unsigned long long)));
    }
    if (!enable && n->iprof) { cudaFree(n->iprof); n->iprof = nullptr; }
    return 0;
}

int fdvl_forward_fused(fdvl_net *n, const fdvl_sample *s, int nb, float conf, int lim, float *out, void *hints) {
    if (!n || !s || nb < 1 || nb > n->maxb) { lerr("fdvl_forward_fused: bad arguments"); return -1; }
    cudaSetDevice(n->device);
    std::vector<Sample> tmp;
    if (load_batch(n, s, nb, tmp)) return -1;
    prep_infer_weights<<<(160 * 576 + 255) / 256, 256, 0, n->st>>>(n->w, n->wimg);
    if (fused_infer(n, n->S, nb, make_float3(conf, conf, conf), lim, n->hints, n->outf, n->err, n->st)) return -1;
    if (out) LCK(cudaMemcpyAsync(out, n->outf, sizeof(float) * kOutPad * nb, cudaMemcpyDeviceToHost, n->st));
    if (hints) LCK(cudaMemcpyAsync(hints, n->hints, sizeof(Hint) * nb, cudaMemcpyDeviceToHost, n->st));
    return check_err(n);
}

int fdvl_grads(fdvl_net *n, const fdvl_sample *s, int nb, float *grad, float *loss) {
    if (!n || !s || nb < 64 || nb % 64 || nb > n->maxb) { lerr("fdvl_grads: batch must be a multiple of 64"); return -1; }
    cudaSetDevice(n->device);
    std::vector<Sample> tmp;
    if (load_batch(n, s, nb, tmp) || forward(n, n->S, nb, n->st) || backward(n, nb)) return -1;
    if (check_err(n)) return -1;
    if (grad) {
        for (int l = 0; l < 4; ++l) {
            const LayerGeo &G = kGeo[l];
            std::vector<float> wt((size_t)G.kp * G.gn), b(G.gn);
            LCK(cudaMemcpy(wt.data(), n->dWT[l], wt.size() * sizeof(float), cudaMemcpyDeviceToHost));
            LCK(cudaMemcpy(b.data(), n->db[l], b.size() * sizeof(float), cudaMemcpyDeviceToHost));
            for (int o = 0; o < G.cout; ++o)
                for (int k = 0; k < G.k; ++k) grad[w_off(l) + o * G.k + k] = wt[(size_t)k * G.gn + o];
            for (int o = 0; o < G.cout; ++o) grad[b_off(l) + o] = b[o];
        }
    }
    if (loss) {
        std::vector<float> lh((size_t)nb * 2);
        LCK(cudaMemcpy(lh.data(), n->loss, lh.size() * sizeof(float), cudaMemcpyDeviceToHost));
        double ce = 0, mv = 0;
        for (int i = 0; i < nb; ++i) { ce += lh[2 * i]; mv += lh[2 * i + 1]; }
        loss[0] = (float)((ce + mv) / nb);
        loss[1] = (float)(ce / nb);
        loss[2] = (float)(mv / nb);
    }
    return 0;
}

int fdvl_train_step(fdvl_net *n, const fdvl_sample *s, int nb, float lr, float *loss) {
    if (fdvl_grads(n, s, nb, nullptr, loss)) return -1;
    if (adam_step(n, lr)) return -1;
    return check_err(n);
}

int fdvl_train(fdvl_net *n, const fdvl_sample *s, int ns, int batch, int epochs, float lr, unsigned long long seed,
               float *curve) {
    if (!n || !s || batch < 64 || batch % 64 || batch > n->maxb || ns < batch || epochs < 1) {
        lerr("fdvl_train: bad arguments");
        return -1;
    }
    cudaSetDevice(n->device);
    std::vector<int> idx(ns);
    for (int i = 0; i < ns; ++i) idx[i] = i;
    uint64_t r = seed;
    auto rnd = [&r]() {
        uint64_t z = (r += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const int steps_per = ns / batch, total = steps_per * epochs;
    std::vector<fdvl_sample> bsmp(batch);
    std::vector<Sample> tmp;
    int step = 0;
    for (int e = 0; e < epochs; ++e) {
        for (int i = ns - 1; i > 0; --i) std::swap(idx[i], idx[rnd() % (uint64_t)(i + 1)]);
        double ce = 0, mv = 0;
        int sampled = 0;
        for (int b = 0; b < steps_per; ++b, ++step) {
            for (int i = 0; i < batch; ++i) bsmp[i] = s[idx[b * batch + i]];
            if (load_batch(n, bsmp.data(), batch, tmp) || forward(n, n->S, batch, n->st) || backward(n, batch))
                return -1;
            // cosine decay to 5% of the base rate
            const double f = 0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * step / std::max(1, total)));
            if (adam_step(n, (float)(lr * f))) return -1;
            if (curve && (b == steps_per - 1 || (b & 63) == 63)) {
                LCK(cudaMemcpyAsync(n->loss_h, n->loss, sizeof(float) * 2 * batch, cudaMemcpyDeviceToHost, n->st));
                LCK(cudaStreamSynchronize(n->st));
                for (int i = 0; i < batch; ++i) { ce += n->loss_h[2 * i]; mv += n->loss_h[2 * i + 1]; }
                sampled += batch;
            }
        }
        if (check_err(n)) return -1;
        if (curve) {
            curve[2 * e] = (float)(ce / std::max(1, sampled));
            curve[2 * e + 1] = (float)(mv / std::max(1, sampled));
        }
    }
    return 0;
}

int fdvl_gemm(int device, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *D, int nsplit) {
    if (M < 1 || N < 16 || N % 16 || K < 64 || nsplit < 1 || K % (64 * nsplit) || !A || !B || !D) {
        lerr("fdvl_gemm: bad shape");
        return -1;
    }
    if (!cu_ok(cudaSetDevice(device), "device")) return -1;
    fdvl_net tmp;
    tmp.device = device;
    std::vector<void *> &o = tmp.owned;
    bf16 *dA = dalloc<bf16>((size_t)M * K, o), *dB = dalloc<bf16>((size_t)N * K, o);
    float *dD = dalloc<float>((size_t)M * N, o);
    tmp.err = dalloc<unsigned>(1, o);
    int rc = -1;
    if (dA && dB && dD && tmp.err &&
        cu_ok(cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem), "attr") &&
        cu_ok(cudaStreamCreateWithFlags(&tmp.st, cudaStreamNonBlocking), "stream") &&
        cu_ok(cudaMemcpy(dA, A, sizeof(bf16) * M * K, cudaMemcpyHostToDevice), "h2d") &&
        cu_ok(cudaMemcpy(dB, B, sizeof(bf16) * N * K, cudaMemcpyHostToDevice), "h2d") &&
        gemm(&tmp, tmp.st, dA, K, dB, K, M, N, K, nsplit > 1 ? EPI_F32_ADD : EPI_F32, dD, nullptr, N, nullptr, 0, nsplit) == 0 &&
        check_err(&tmp) == 0 && cu_ok(cudaMemcpy(D, dD, sizeof(float) * M * N, cudaMemcpyDeviceToHost), "d2h"))
        rc = 0;
    for (void *p : o) cudaFree(p);
    if (tmp.st) cudaStreamDestroy(tmp.st);
    tmp.owned.clear();
    tmp.st = nullptr;
    return rc;
}

}  // extern "C"

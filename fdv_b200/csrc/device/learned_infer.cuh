// Fused inference of the proposal network: one persistent kernel computes
// every macroblock's proposal of a frame step.  A CTA (8 warps) takes 8
// macroblocks at a time:
//   features  -> X0 (two macroblocks at a time, shared memory)
//   conv1     -> four 128x32x128 tcgen05 MMA tiles (im2col of X0 built in
//                shared memory in the canonical operand layout), ReLU -> Y1
//   conv2     -> one 128x64x320 MMA tile per macroblock pair, ReLU -> Y2
//   conv3     -> one 128x160x576 MMA tile for all eight, weights streamed in
//                64-wide K chunks, ReLU -> Y3
//   fc        -> 2560x11 dot products on the CUDA cores, then the hint.
// Accumulators live in TMEM (conv1 columns 0-127, conv2 128-191, conv3
// 256-415); activations never leave shared memory.  The weights are kept in
// global memory as ready-made canonical operand images (built once per
// parameter upload by prep_infer_weights), so staging a weight chunk is a
// straight copy.
#pragma once
#include <cuda_bf16.h>

#include "learned.cuh"
#include "tc.cuh"

namespace fdvb {
namespace lrn {

using bf16 = __nv_bfloat16;

constexpr int IMB = 8, INT = 256;
// canonical weight images (bytes)
constexpr int kW1c = 32 * 128;              // conv1: 32 rows x 64 K
constexpr int kW2chunk = 64 * 128;          // conv2: 64 rows x 64 K, 5 chunks
constexpr int kW2c = 5 * kW2chunk;
constexpr int kW3chunk = 160 * 128;         // conv3: 160 rows x 64 K, 9 chunks
constexpr int kW3c = 9 * kW3chunk;
// fc as one MMA: B rows (j, p') = j*16 + p' (176), K = channel c (160, padded
// to 192): B[j*16+p'][c] = W4[j][p'*160 + c].  With A rows (m, p) = conv3's
// output rows, D[(m,p)][(j,p')] summed over the diagonal p = p' is the
// macroblock's output j.
constexpr int kFcN = kOut * 16;             // 176
constexpr int kW4chunk = kFcN * 128;
constexpr int kW4c = 3 * kW4chunk;
constexpr int kWImage = kW1c + kW2c + kW3c + kW4c;
// shared memory
constexpr int kAbuf = 128 * 128;            // one 128-row x 64-K operand tile
constexpr int kWin = 65 * 72;               // one 64x64(+1) luma window, 72-byte rows
// A: four operand tiles (conv1's four tiles; conv2's chunks 0-3, chunk 4 in
// X0; conv3's chunks three at a time, their weights in A3 + R1); before that
// the staged luma windows, at the end the fc outputs.
constexpr int O_W1 = 0, O_W2 = O_W1 + kW1c, O_A = O_W2 + kW2c, O_R1 = O_A + 4 * kAbuf;
// R1: X0[2] (16 KB) + Y1[2] (32 KB); then conv3 weight chunks; then the fc operand
constexpr int kR1 = 16384 + 2 * 16384;
constexpr int O_X0 = O_R1, O_Y1 = O_R1 + 16384;
constexpr int O_W3 = O_A + 3 * kAbuf;       // three conv3 weight chunks (A3 + R1)
constexpr int O_Y2 = O_R1 + kR1, O_BAR = O_Y2 + IMB * 8192, O_SMP = O_BAR + 64;
constexpr int kInferSmem = O_SMP + IMB * (int)sizeof(Sample);
// the weight offsets below are the flat parameter layout's
static_assert(kWOff[1] == 1216 && kWOff[2] == 19712 && kWOff[3] == 112032, "parameter layout");
static_assert(O_W3 + 3 * kW3chunk <= O_R1 + kR1 && 3 * kAbuf <= kR1 && 2 * kW4chunk <= IMB * 8192 &&
                  4 * kWin <= 4 * kAbuf && kInferSmem <= 232448,
              "region reuse");

struct InferW {
    const uint8_t *img;                     // kWImage bytes: W1c | W2c | W3c | W4c
    const float *b[4];                      // fp32 biases
    unsigned long long *prof;               // optional per-phase cycle sums (thread 0 of each CTA)
};
enum { IP_STAGE = 0, IP_FEAT, IP_C1, IP_C1E, IP_C2, IP_C2E, IP_C3, IP_FC, IP_NGROUP, IP_N = 16 };

// Canonical operand images of the current bf16-rounded weights.
__global__ void prep_infer_weights(const float *__restrict__ w, uint8_t *__restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bf16 *o = reinterpret_cast<bf16 *>(img);
    if (i < 32 * 64) {   // conv1
        const int n = i / 64, k = i % 64;
        o[umma_off(n, k) / 2] = __float2bfloat16_rn(k < 37 ? w[n * 37 + k] : 0.f);
    }
    if (i < 64 * 320) {   // conv2: 5 chunks
        const int n = i / 320, k = i % 320, c = k / 64;
        const float v = k < 288 ? w[1216 + n * 288 + k] : 0.f;
        o[(kW1c + c * kW2chunk + umma_off(n, k - c * 64)) / 2] = __float2bfloat16_rn(v);
    }
    if (i < 160 * 576) {   // conv3: 9 chunks
        const int n = i / 576, k = i % 576, c = k / 64;
        o[(kW1c + kW2c + c * kW3chunk + umma_off(n, k - c * 64)) / 2] =
            __float2bfloat16_rn(w[19712 + n * 576 + k]);
    }
    if (i < kFcN * 192) {   // fc: 3 chunks of 176 rows
        const int row = i / 192, k = i % 192, c = k / 64, j = row >> 4, pp = row & 15;
        const float v = k < 160 ? w[112032 + j * 2560 + pp * 160 + k] : 0.f;
        o[(kW1c + kW2c + kW3c + c * kW4chunk + umma_off(row, k - c * 64)) / 2] = __float2bfloat16_rn(v);
    }
}

__device__ __forceinline__ bf16 pix_feat(int v) { return __float2bfloat16_rn((float)(v - 128) * (1.f / 64.f)); }

// 16 fp32 accumulators + bias, ReLU, to 16 bf16 (32 bytes) at dst.
__device__ __forceinline__ void relu_store16(const float v[16], const float *__restrict__ bias, bf16 *dst) {
    __align__(16) bf16 o[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) o[q] = __float2bfloat16_rn(fmaxf(v[q] + __ldg(bias + q), 0.f));
    reinterpret_cast<uint4 *>(dst)[0] = reinterpret_cast<const uint4 *>(o)[0];
    reinterpret_cast<uint4 *>(dst)[1] = reinterpret_cast<const uint4 *>(o)[1];
}

__device__ __forceinline__ Hint make_hint(const float o[kOutPad], float3 conf, int lim) {
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
    h.cls = p >= (c == 0 ? conf.x : (c == 1 ? conf.y : conf.z)) ? c : -1;
    return h;
}

// One CTA per SM; CTA b takes the macroblocks [b*n/grid, (b+1)*n/grid) in
// groups of eight (the last one partial, its empty pairs skipped).
__global__ void __launch_bounds__(INT, 1)
infer_kernel(const Sample *__restrict__ S, int n, InferW W, float3 conf, int lim, Hint *__restrict__ hints,
             float *__restrict__ out, unsigned *err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *win = sm + O_A;                                       // [2 macroblocks][cur, ref][65][72] during features
    float *fo = reinterpret_cast<float *>(sm + O_A);               // [8][16] fc outputs at the end
    bf16 *X0 = reinterpret_cast<bf16 *>(sm + O_X0);                // [2][1024][4]
    bf16 *Y1 = reinterpret_cast<bf16 *>(sm + O_Y1);                // [2][256][32]
    uint8_t *Y3c = sm + O_R1;                                      // fc A operand: 3 chunks of 128 x 64
    bf16 *Y2 = reinterpret_cast<bf16 *>(sm + O_Y2);                // [8][64][64]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + O_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + O_BAR + 16);
    Sample *smp = reinterpret_cast<Sample *>(sm + O_SMP);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q4 = warp & 3, half = warp >> 2;
    const int rr = tid & 127, rk = tid >> 7;    // an operand-building thread's row, and its first K chunk

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, 512);
    // resident conv1 / conv2 weights
    for (int i = tid; i < (kW1c + kW2c) / 16; i += INT) cpa16(sm + O_W1 + i * 16, W.img + i * 16, 16);
    cpa_commit();
    cpa_wait<0>();
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t lane_off = (uint32_t)(q4 * 32) << 16;
    // commits issued to / waited on each buffer's mbarrier (scalars: no local memory)
    int iss0 = 0, iss1 = 0, wt0 = 0, wt1 = 0;
    auto wait_buf = [&](int b) {
        if (b == 0 && wt0 < iss0) { mbar_wait(&bar[0], wt0 & 1, err); ++wt0; }
        if (b == 1 && wt1 < iss1) { mbar_wait(&bar[1], wt1 & 1, err); ++wt1; }
    };
    auto mma4 = [&](uint32_t a_s, uint32_t b_s, uint32_t d, int nn, bool acc0, int b) {
        // four K=16 steps of a 64-wide tile; only thread 0 issues
        if (tid == 0) {
            tc_after_sync();
            const uint32_t id = umma_idesc_bf16(128, nn);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
                umma_bf16(d, umma_desc(a_s + ks * 256, 128, 1024), umma_desc(b_s + ks * 256, 128, 1024), id,
                          (acc0 || ks) ? 1u : 0u);
            umma_commit(&bar[b]);
        }
        if (b) ++iss1; else ++iss0;
    };
    const uint32_t a0 = smem_u32(sm + O_A), a1 = a0 + kAbuf, w1s = smem_u32(sm + O_W1), w2s = smem_u32(sm + O_W2);
    const uint32_t t1s[4] = {a0, a0 + kAbuf, a0 + 2 * kAbuf, a0 + 3 * kAbuf};
    const int mb0 = (int)((long long)blockIdx.x * n / gridDim.x), mb1 = (int)((long long)(blockIdx.x + 1) * n / gridDim.x);
    long long tmark = clock64();
    auto mark = [&](int ph) {
        if (W.prof && tid == 0) {
            const long long t = clock64();
            atomicAdd(&W.prof[ph], (unsigned long long)(t - tmark));
            tmark = t;
        }
    };
    for (int g0 = mb0; g0 < mb1; g0 += IMB) {
        const int cnt = min(IMB, mb1 - g0);
        if (tid < cnt) smp[tid] = S[g0 + tid];
        __syncthreads();
        if (W.prof && tid == 0) atomicAdd(&W.prof[IP_NGROUP], 1ull);
        for (int pair = 0; 2 * pair < cnt; ++pair) {
            // the two macroblocks' 64x64 (+1) windows of the current and the
            // reference luma: 8-byte loads where the window is inside the
            // picture, clamped byte loads at its edges
            for (int e = tid; e < 2 * 2 * 65 * 9; e += INT) {
                const int q = e % 9, row = (e / 9) % 65, pl = (e / 585) & 1, j = e / 1170;
                uint2 v = make_uint2(0, 0);
                if (2 * pair + j < cnt) {
                    const Sample &sp = smp[2 * pair + j];
                    const uint8_t *P = pl ? sp.ref : sp.cur;
                    const int st = pl ? sp.rs : sp.cs;
                    const int x0 = sp.bx - 24 + 8 * q, y = sp.by - 24 + row;
                    const bool inner = x0 >= 0 && x0 + 8 <= sp.w && y >= 0 && y < sp.h &&
                                       ((reinterpret_cast<uintptr_t>(P) | (uintptr_t)st) & 7) == 0;
                    if (inner) {
                        cpa8(win + (j * 2 + pl) * kWin + row * 72 + 8 * q, P + (size_t)y * st + x0);
                        continue;
                    } else {
                        const int yy = min(max(y, 0), sp.h - 1);
                        uint32_t b[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) b[u] = __ldg(P + (size_t)yy * st + min(max(x0 + u, 0), sp.w - 1));
                        v.x = b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24);
                        v.y = b[4] | (b[5] << 8) | (b[6] << 16) | (b[7] << 24);
                    }
                }
                *reinterpret_cast<uint2 *>(win + (j * 2 + pl) * kWin + row * 72 + 8 * q) = v;
            }
            cpa_commit();
            cpa_wait<0>();
            __syncthreads();
            mark(IP_STAGE);
            // features: full-resolution 32x32 at window offset 16, 2x2 means of the 64x64
#pragma unroll
            for (int e = tid; e < 2 * 1024; e += INT) {
                const int j = e >> 10, p = e & 1023, px = p & 31, py = p >> 5;
                const uint8_t *cw = win + (j * 2) * kWin, *rw = cw + kWin;
                const int c0 = cw[(py + 16) * 72 + px + 16], c1 = rw[(py + 16) * 72 + px + 16];
                const uint32_t ca = *reinterpret_cast<const uint16_t *>(cw + (2 * py) * 72 + 2 * px);
                const uint32_t cb = *reinterpret_cast<const uint16_t *>(cw + (2 * py + 1) * 72 + 2 * px);
                const uint32_t ra = *reinterpret_cast<const uint16_t *>(rw + (2 * py) * 72 + 2 * px);
                const uint32_t rb = *reinterpret_cast<const uint16_t *>(rw + (2 * py + 1) * 72 + 2 * px);
                const int c2 = ((int)(ca & 255) + (int)(ca >> 8) + (int)(cb & 255) + (int)(cb >> 8) + 2) >> 2;
                const int c3 = ((int)(ra & 255) + (int)(ra >> 8) + (int)(rb & 255) + (int)(rb >> 8) + 2) >> 2;
                __align__(8) bf16 o[4] = {pix_feat(c0), pix_feat(c1), pix_feat(c2), pix_feat(c3)};
                reinterpret_cast<uint2 *>(X0)[e] = *reinterpret_cast<const uint2 *>(o);
            }
            __syncthreads();
            mark(IP_FEAT);
            // conv1: four tiles t = (macroblock j, half h) built at once, rows =
            // output positions h*128 .., K = 9 taps x 4 channels + the quantiser
            {
                const bf16 zero = __float2bfloat16_rn(0.f);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int j = t >> 1, p = (t & 1) * 128 + rr, oy = p >> 4, ox = p & 15;
                    const uint2 *xj = reinterpret_cast<const uint2 *>(X0) + j * 1024;
                    uint8_t *tile = sm + O_A + t * kAbuf;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int kc = rk + 2 * u;   // 8 K values: taps 2kc, 2kc+1
                        uint2 v[2];
#pragma unroll
                        for (int h2 = 0; h2 < 2; ++h2) {
                            const int tap = 2 * kc + h2, ky = (tap * 11) >> 5, kx = tap - 3 * ky;
                            const int y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                            v[h2] = (tap < 9 && y >= 0 && y < 32 && x >= 0 && x < 32) ? xj[y * 32 + x] : make_uint2(0, 0);
                        }
                        if (kc == 4) {   // tap 8, then the quantiser column, then zeros
                            __align__(8) bf16 qv[4] = {__float2bfloat16_rn((float)(smp[2 * pair + j].qp - 26) * 0.125f),
                                                       zero, zero, zero};
                            v[1] = *reinterpret_cast<const uint2 *>(qv);
                        }
                        *reinterpret_cast<uint4 *>(tile + umma_off(rr, kc * 8)) = make_uint4(v[0].x, v[0].y, v[1].x, v[1].y);
                    }
                }
            }
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_after_sync();
                const uint32_t id = umma_idesc_bf16(128, 32);
#pragma unroll
                for (int t = 0; t < 4; ++t)
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                        umma_bf16(tmem + 32 * t, umma_desc(t1s[t] + ks * 256, 128, 1024),
                                  umma_desc(w1s + ks * 256, 128, 1024), id, ks ? 1u : 0u);
                umma_commit(&bar[1]);
            }
            ++iss1;
            wait_buf(1);
            tc_after_sync();
            mark(IP_C1);
            // conv1 epilogue: warps 0-3 macroblock 0, warps 4-7 macroblock 1
            for (int hh = 0; hh < 2; ++hh) {
                const int t = 2 * half + hh, p = hh * 128 + q4 * 32 + lane;
                float v[16];
                tmem_ld16(tmem + lane_off + 32 * t, v);
                relu_store16(v, W.b[0], Y1 + (half * 256 + p) * 32);
                tmem_ld16(tmem + lane_off + 32 * t + 16, v);
                relu_store16(v, W.b[0] + 16, Y1 + (half * 256 + p) * 32 + 16);
            }
            tc_before_sync();
            __syncthreads();
            mark(IP_C1E);
            // conv2: rows = (macroblock r>>6, position r&63); all five 64-wide K
            // chunks built at once (A0-A3, then X0), one MMA batch
            {
                const int j = rr >> 6, p = rr & 63, oy = p >> 3, ox = p & 7;
                const bf16 *yj = Y1 + j * 256 * 32;
#pragma unroll
                for (int c = 0; c < 5; ++c) {
                    uint8_t *chunk = sm + (c < 4 ? O_A + c * kAbuf : O_X0);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int kc = rk + 2 * u, k0 = c * 64 + kc * 8, tap = k0 >> 5, ci = k0 & 31;
                        const int ky = (tap * 11) >> 5, kx = tap - 3 * ky, y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                        uint4 v = make_uint4(0, 0, 0, 0);
                        if (tap < 9 && y >= 0 && y < 16 && x >= 0 && x < 16)
                            v = *reinterpret_cast<const uint4 *>(yj + (y * 16 + x) * 32 + ci);
                        *reinterpret_cast<uint4 *>(chunk + umma_off(rr, kc * 8)) = v;
                    }
                }
                fence_async_smem();
                __syncthreads();
                if (tid == 0) {
                    tc_after_sync();
                    const uint32_t id = umma_idesc_bf16(128, 64);
                    const uint32_t x0s = smem_u32(sm + O_X0);
#pragma unroll
                    for (int c = 0; c < 5; ++c)
#pragma unroll
                        for (int ks = 0; ks < 4; ++ks)
                            umma_bf16(tmem + 128, umma_desc((c < 4 ? a0 + c * kAbuf : x0s) + ks * 256, 128, 1024),
                                      umma_desc(w2s + c * kW2chunk + ks * 256, 128, 1024), id, (c | ks) ? 1u : 0u);
                    umma_commit(&bar[1]);
                }
                ++iss1;
            }
            wait_buf(0);
            wait_buf(1);
            tc_after_sync();
            mark(IP_C2);
            {
                const int r = q4 * 32 + lane, j = r >> 6, p = r & 63, c0 = half * 32;
                float v[16];
                bf16 *dst = Y2 + ((2 * pair + j) * 64 + p) * 64 + c0;
                tmem_ld16(tmem + lane_off + 128 + c0, v);
                relu_store16(v, W.b[1] + c0, dst);
                tmem_ld16(tmem + lane_off + 128 + c0 + 16, v);
                relu_store16(v, W.b[1] + c0 + 16, dst + 16);
            }
            tc_before_sync();
            __syncthreads();
            mark(IP_C2E);
        }
        // conv3: rows = (macroblock r>>4, position r&15); nine 64-wide K chunks
        // in three rounds of three (operands in A0-A2, weights in A3 + R1)
        {
            const uint8_t *w3 = W.img + kW1c + kW2c;
            const int m = rr >> 4, p = rr & 15, oy = p >> 2, ox = p & 3;
            for (int rnd = 0; rnd < 3; ++rnd) {
                wait_buf(1);   // the previous round's MMAs are done with these buffers
                for (int e = tid; e < 3 * kW3chunk / 16; e += INT)
                    cpa16(sm + O_W3 + e * 16, w3 + rnd * 3 * kW3chunk + e * 16, 16);
                cpa_commit();
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const int c = rnd * 3 + cc;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int kc = rk + 2 * u, k0 = c * 64 + kc * 8, tap = k0 >> 6, ci = k0 & 63;
                        const int ky = (tap * 11) >> 5, kx = tap - 3 * ky, y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                        uint4 v = make_uint4(0, 0, 0, 0);
                        if (y >= 0 && y < 8 && x >= 0 && x < 8 && (m < cnt))
                            v = *reinterpret_cast<const uint4 *>(Y2 + (m * 64 + y * 8 + x) * 64 + ci);
                        *reinterpret_cast<uint4 *>(sm + O_A + cc * kAbuf + umma_off(rr, kc * 8)) = v;
                    }
                }
                cpa_wait<0>();
                fence_async_smem();
                __syncthreads();
                if (tid == 0) {
                    tc_after_sync();
                    const uint32_t id = umma_idesc_bf16(128, 160), w3s = smem_u32(sm + O_W3);
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                        for (int ks = 0; ks < 4; ++ks)
                            umma_bf16(tmem + 256, umma_desc(a0 + cc * kAbuf + ks * 256, 128, 1024),
                                      umma_desc(w3s + cc * kW3chunk + ks * 256, 128, 1024), id,
                                      (rnd | cc | ks) ? 1u : 0u);
                    umma_commit(&bar[1]);
                }
                ++iss1;
            }
        }
        wait_buf(0);
        wait_buf(1);
        tc_after_sync();
        mark(IP_C3);
        // fc weight chunks 0 and 1 (the conv2 output region is free now)
        const uint8_t *w4 = W.img + kW1c + kW2c + kW3c;
        for (int e = tid; e < 2 * kW4chunk / 16; e += INT) cpa16(sm + O_Y2 + e * 16, w4 + e * 16, 16);
        cpa_commit();
        // conv3 epilogue straight into the fc's A operand (rows (m, p), K = channels)
        {
            const int r = q4 * 32 + lane;
            for (int cc = 0; cc < 5; ++cc) {
                const int c0 = half * 80 + cc * 16;
                float v[16];
                tmem_ld16(tmem + lane_off + 256 + c0, v);
                __align__(16) bf16 o[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) o[u] = __float2bfloat16_rn(fmaxf(v[u] + __ldg(W.b[2] + c0 + u), 0.f));
                uint8_t *chunk = Y3c + (c0 >> 6) * kAbuf;
                *reinterpret_cast<uint4 *>(chunk + umma_off(r, c0 & 63)) = reinterpret_cast<const uint4 *>(o)[0];
                *reinterpret_cast<uint4 *>(chunk + umma_off(r, (c0 & 63) + 8)) = reinterpret_cast<const uint4 *>(o)[1];
            }
            if (half)   // channels 160..191 of the last chunk are zero
#pragma unroll
                for (int u = 4; u < 8; ++u)
                    *reinterpret_cast<uint4 *>(Y3c + 2 * kAbuf + umma_off(r, u * 8)) = make_uint4(0, 0, 0, 0);
        }
        tc_before_sync();
        cpa_wait<0>();
        fence_async_smem();
        __syncthreads();
        // fc: three 128x176x64 MMAs
        {
            const uint32_t y3s = smem_u32(Y3c), w4s = smem_u32(sm + O_Y2);
            mma4(y3s, w4s, tmem, kFcN, false, 0);
            mma4(y3s + kAbuf, w4s + kW4chunk, tmem, kFcN, true, 1);
            wait_buf(0);   // chunk 2 into weight buffer 0
            for (int e = tid; e < kW4chunk / 16; e += INT) cpa16(sm + O_Y2 + e * 16, w4 + 2 * kW4chunk + e * 16, 16);
            cpa_commit();
            cpa_wait<0>();
            fence_async_smem();
            __syncthreads();
            mma4(y3s + 2 * kAbuf, w4s, tmem, kFcN, true, 0);
        }
        wait_buf(0);
        wait_buf(1);
        tc_after_sync();
        {
            // row (m, p) keeps column j*16 + p of each output block; the 16 rows of a
            // macroblock are 16 consecutive lanes
            const int r = q4 * 32 + lane, m = r >> 4, p = r & 15;
            const int j0 = half ? 6 : 0, j1 = half ? kOut : 6;
            for (int j = j0; j < j1; ++j) {
                float v[16];
                tmem_ld16(tmem + lane_off + 16 * j, v);
                float s = 0.f;
#pragma unroll
                for (int q = 0; q < 16; ++q) s = q == p ? v[q] : s;
                for (int d = 8; d; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
                if (p == 0) fo[m * kOutPad + j] = s + __ldg(W.b[3] + j);
            }
        }
        tc_before_sync();
        __syncthreads();
        if (tid < cnt) {
            const int i = g0 + tid;
            float o[kOutPad];
            for (int j = 0; j < kOutPad; ++j) o[j] = j < kOut ? fo[tid * kOutPad + j] : 0.f;
            if (out)
                for (int j = 0; j < kOutPad; ++j) out[(size_t)i * kOutPad + j] = o[j];
            if (hints) hints[i] = make_hint(o, conf, lim);
        }
        __syncthreads();
        mark(IP_FC);
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_after_sync();
        tmem_free(tmem, 512);
    }
}

}  // namespace lrn
}  // namespace fdvb

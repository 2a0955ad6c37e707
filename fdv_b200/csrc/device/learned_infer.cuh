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
constexpr int kW1chunk = 32 * 128;          // conv1: 32 rows x 64 K, 2 chunks
constexpr int kW1c = 2 * kW1chunk;
constexpr int kW2chunk = 64 * 128;          // conv2: 64 rows x 64 K, 5 chunks
constexpr int kW2c = 5 * kW2chunk;
constexpr int kW3chunk = 160 * 128;         // conv3: 160 rows x 64 K, 9 chunks
constexpr int kW3c = 9 * kW3chunk;
constexpr int kW4 = kOutPad * 2560 * 2;     // fc: bf16 [16][2560], row-major
constexpr int kWImage = kW1c + kW2c + kW3c + kW4;
// shared memory
constexpr int kAbuf = 128 * 128;            // one 128-row x 64-K operand tile
constexpr int O_W1 = 0, O_W2 = O_W1 + kW1c, O_A = O_W2 + kW2c, O_R1 = O_A + 2 * kAbuf;
constexpr int kR1 = 2 * 16384 + 2 * 16384;  // X0[2] + Y1[2]; later conv3 weight chunks, then Y3
constexpr int O_Y2 = O_R1 + kR1, O_BAR = O_Y2 + IMB * 8192, O_SMP = O_BAR + 64;
constexpr int kInferSmem = O_SMP + IMB * (int)sizeof(Sample);
// the weight offsets above are the flat parameter layout's
static_assert(kWOff[1] == 2336 && kWOff[2] == 20832 && kWOff[3] == 113152, "parameter layout");
static_assert(2 * kW3chunk <= kR1 && IMB * 5120 <= kR1, "region reuse");

struct InferW {
    const uint8_t *img;                     // kWImage bytes: W1c | W2c | W3c | W4
    const float *b[4];                      // fp32 biases
};

// Canonical operand images of the current bf16-rounded weights.
__global__ void prep_infer_weights(const float *__restrict__ w, uint8_t *__restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bf16 *o = reinterpret_cast<bf16 *>(img);
    // conv1: 2 chunks
    if (i < 32 * 128) {
        const int n = i / 128, k = i % 128, c = k / 64;
        const float v = k < 72 ? w[n * 72 + k] : 0.f;
        o[(c * kW1chunk + umma_off(n, k - c * 64)) / 2] = __float2bfloat16_rn(v);
    }
    // conv2: 5 chunks
    if (i < 64 * 320) {
        const int n = i / 320, k = i % 320, c = k / 64;
        const float v = k < 288 ? w[2336 + n * 288 + k] : 0.f;
        o[(kW1c + c * kW2chunk + umma_off(n, k - c * 64)) / 2] = __float2bfloat16_rn(v);
    }
    // conv3: 9 chunks
    if (i < 160 * 576) {
        const int n = i / 576, k = i % 576, c = k / 64;
        o[(kW1c + kW2c + c * kW3chunk + umma_off(n, k - c * 64)) / 2] =
            __float2bfloat16_rn(w[20832 + n * 576 + k]);
    }
    // fc
    if (i < kOutPad * 2560) {
        const int j = i / 2560, k = i % 2560;
        o[(kW1c + kW2c + kW3c) / 2 + i] = __float2bfloat16_rn(j < kOut ? w[113152 + j * 2560 + k] : 0.f);
    }
}

__device__ __forceinline__ uint4 feat8(const Sample &q, int x, int y) {
    auto px = [](const uint8_t *p, int s, int w, int h, int xx, int yy) {
        xx = xx < 0 ? 0 : (xx >= w ? w - 1 : xx);
        yy = yy < 0 ? 0 : (yy >= h ? h - 1 : yy);
        return (int)__ldg(p + (size_t)yy * s + xx);
    };
    const int c0 = px(q.cur, q.cs, q.w, q.h, q.bx - 8 + x, q.by - 8 + y);
    const int c1 = px(q.ref, q.rs, q.w, q.h, q.bx - 8 + x, q.by - 8 + y);
    const int gx = q.bx - 24 + 2 * x, gy = q.by - 24 + 2 * y;
    const int c2 = (px(q.cur, q.cs, q.w, q.h, gx, gy) + px(q.cur, q.cs, q.w, q.h, gx + 1, gy) +
                    px(q.cur, q.cs, q.w, q.h, gx, gy + 1) + px(q.cur, q.cs, q.w, q.h, gx + 1, gy + 1) + 2) >> 2;
    const int c3 = (px(q.ref, q.rs, q.w, q.h, gx, gy) + px(q.ref, q.rs, q.w, q.h, gx + 1, gy) +
                    px(q.ref, q.rs, q.w, q.h, gx, gy + 1) + px(q.ref, q.rs, q.w, q.h, gx + 1, gy + 1) + 2) >> 2;
    __align__(16) bf16 o[8];
    o[0] = __float2bfloat16_rn((float)(c0 - 128) * (1.f / 64.f));
    o[1] = __float2bfloat16_rn((float)(c1 - 128) * (1.f / 64.f));
    o[2] = __float2bfloat16_rn((float)(c2 - 128) * (1.f / 64.f));
    o[3] = __float2bfloat16_rn((float)(c3 - 128) * (1.f / 64.f));
    o[4] = __float2bfloat16_rn((float)(q.qp - 26) * 0.125f);
    o[5] = o[6] = o[7] = __float2bfloat16_rn(0.f);
    return *reinterpret_cast<const uint4 *>(o);
}

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

__global__ void __launch_bounds__(INT, 1)
infer_kernel(const Sample *__restrict__ S, int n, InferW W, float3 conf, int lim, Hint *__restrict__ hints,
             float *__restrict__ out, unsigned *err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *A[2] = {sm + O_A, sm + O_A + kAbuf};
    bf16 *X0 = reinterpret_cast<bf16 *>(sm + O_R1);                // [2][1024][8]
    bf16 *Y1 = reinterpret_cast<bf16 *>(sm + O_R1 + 32768);        // [2][256][32]
    uint8_t *W3b[2] = {sm + O_R1, sm + O_R1 + kW3chunk};
    bf16 *Y3 = reinterpret_cast<bf16 *>(sm + O_R1);                // [8][16][160]
    bf16 *Y2 = reinterpret_cast<bf16 *>(sm + O_Y2);                // [8][64][64]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + O_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + O_BAR + 16);
    Sample *smp = reinterpret_cast<Sample *>(sm + O_SMP);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q4 = warp & 3, half = warp >> 2;

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
    int issued[2] = {0, 0}, waited[2] = {0, 0};
    auto wait_buf = [&](int b) {
        if (waited[b] < issued[b]) {
            mbar_wait(&bar[b], waited[b] & 1, err);
            ++waited[b];
        }
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
        ++issued[b];
    };
    const int ngroups = (n + IMB - 1) / IMB;
    const uint32_t a0 = smem_u32(A[0]), a1 = smem_u32(A[1]), w1s = smem_u32(sm + O_W1), w2s = smem_u32(sm + O_W2);
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        if (tid < IMB) {
            const int i = g * IMB + tid;
            if (i < n) smp[tid] = S[i];
        }
        __syncthreads();
        for (int pair = 0; pair < IMB / 2; ++pair) {
            // features of two macroblocks (eight positions per thread, loads in flight together)
#pragma unroll
            for (int e = tid; e < 2 * 1024; e += INT) {
                const int j = e >> 10, p = e & 1023, i = g * IMB + 2 * pair + j;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (i < n) v = feat8(smp[2 * pair + j], p & 31, p >> 5);
                reinterpret_cast<uint4 *>(X0)[e] = v;
            }
            __syncthreads();
            // conv1: tiles t = (macroblock j, half h): rows = output positions
            // h*128 ..; K = 9 taps x 8 channels in two 64-wide chunks (one tap
            // per 16-byte vector), both buffers, one commit
            for (int t = 0; t < 4; ++t) {
                const int j = t >> 1, h = t & 1;
                wait_buf(0);
                wait_buf(1);
                for (int e = tid; e < 128 * 16; e += INT) {
                    const int r = e & 127, tap = e >> 7, p = h * 128 + r, oy = p >> 4, ox = p & 15;
                    const int ky = tap / 3, kx = tap - ky * 3, y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (tap < 9 && y >= 0 && y < 32 && x >= 0 && x < 32)
                        v = reinterpret_cast<const uint4 *>(X0)[j * 1024 + y * 32 + x];
                    *reinterpret_cast<uint4 *>(A[tap >> 3] + umma_off(r, (tap & 7) * 8)) = v;
                }
                fence_async_smem();
                __syncthreads();
                if (tid == 0) {
                    tc_after_sync();
                    const uint32_t id = umma_idesc_bf16(128, 32);
#pragma unroll
                    for (int ks = 0; ks < 8; ++ks)
                        umma_bf16(tmem + 32 * t,
                                  umma_desc((ks < 4 ? a0 : a1) + (ks & 3) * 256, 128, 1024),
                                  umma_desc(w1s + (ks >> 2) * kW1chunk + (ks & 3) * 256, 128, 1024), id,
                                  ks ? 1u : 0u);
                    umma_commit(&bar[1]);
                }
                ++issued[1];
            }
            wait_buf(0);
            wait_buf(1);
            tc_after_sync();
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
            // conv2: rows = (macroblock r>>6, position r&63), K chunks of 64
            for (int c = 0; c < 5; ++c) {
                const int b = c & 1;
                wait_buf(b);
                for (int e = tid; e < 128 * 8; e += INT) {
                    const int r = e & 127, kc = e >> 7, j = r >> 6, p = r & 63, oy = p >> 3, ox = p & 7;
                    const int k0 = c * 64 + kc * 8, tap = k0 >> 5, ci = k0 & 31, ky = tap / 3, kx = tap - ky * 3;
                    const int y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (tap < 9 && y >= 0 && y < 16 && x >= 0 && x < 16)
                        v = *reinterpret_cast<const uint4 *>(Y1 + (j * 256 + y * 16 + x) * 32 + ci);
                    *reinterpret_cast<uint4 *>(A[b] + umma_off(r, kc * 8)) = v;
                }
                fence_async_smem();
                __syncthreads();
                mma4(b ? a1 : a0, w2s + c * kW2chunk, tmem + 128, 64, c > 0, b);
            }
            wait_buf(0);
            wait_buf(1);
            tc_after_sync();
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
        }
        // conv3: rows = (macroblock r>>4, position r&15), K chunks of 64, weights streamed
        const uint8_t *w3 = W.img + kW1c + kW2c;
        for (int c = 0; c < 9; ++c) {
            const int b = c & 1;
            wait_buf(b);
            for (int e = tid; e < kW3chunk / 16; e += INT) cpa16(W3b[b] + e * 16, w3 + c * kW3chunk + e * 16, 16);
            cpa_commit();
            for (int e = tid; e < 128 * 8; e += INT) {
                const int r = e & 127, kc = e >> 7, m = r >> 4, p = r & 15, oy = p >> 2, ox = p & 3;
                const int k0 = c * 64 + kc * 8, tap = k0 >> 6, ci = k0 & 63, ky = tap / 3, kx = tap - ky * 3;
                const int y = 2 * oy - 1 + ky, x = 2 * ox - 1 + kx;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (y >= 0 && y < 8 && x >= 0 && x < 8)
                    v = *reinterpret_cast<const uint4 *>(Y2 + (m * 64 + y * 8 + x) * 64 + ci);
                *reinterpret_cast<uint4 *>(A[b] + umma_off(r, kc * 8)) = v;
            }
            cpa_wait<0>();
            fence_async_smem();
            __syncthreads();
            mma4(b ? a1 : a0, smem_u32(W3b[b]), tmem + 256, 160, c > 0, b);
        }
        wait_buf(0);
        wait_buf(1);
        tc_after_sync();
        {
            const int r = q4 * 32 + lane, m = r >> 4, p = r & 15;
            for (int cc = 0; cc < 5; ++cc) {
                const int c0 = half * 80 + cc * 16;
                float v[16];
                tmem_ld16(tmem + lane_off + 256 + c0, v);
                __align__(16) bf16 o[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) o[u] = __float2bfloat16_rn(fmaxf(v[u] + __ldg(W.b[2] + c0 + u), 0.f));
                uint4 *d = reinterpret_cast<uint4 *>(Y3 + (m * 16 + p) * 160 + c0);
                d[0] = reinterpret_cast<const uint4 *>(o)[0];
                d[1] = reinterpret_cast<const uint4 *>(o)[1];
            }
        }
        tc_before_sync();
        __syncthreads();
        // fc: warp w computes output w (and w + 8) for all eight macroblocks;
        // each lane holds ten 8-element slices of the weight row
        {
            const bf16 *w4 = reinterpret_cast<const bf16 *>(W.img + kW1c + kW2c + kW3c);
            float *fo = reinterpret_cast<float *>(sm + O_A);   // [8][16] outputs (operand buffers are free)
            for (int j = warp; j < kOut; j += 8) {
                uint4 wv[10];
#pragma unroll
                for (int u = 0; u < 10; ++u) wv[u] = __ldg(reinterpret_cast<const uint4 *>(w4 + j * 2560 + (lane + 32 * u) * 8));
                float acc[IMB];
#pragma unroll
                for (int m = 0; m < IMB; ++m) acc[m] = 0.f;
#pragma unroll
                for (int u = 0; u < 10; ++u) {
                    const bf16 *we = reinterpret_cast<const bf16 *>(&wv[u]);
                    float wf[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) wf[e] = __bfloat162float(we[e]);
#pragma unroll
                    for (int m = 0; m < IMB; ++m) {
                        const uint4 yv = *reinterpret_cast<const uint4 *>(Y3 + m * 2560 + (lane + 32 * u) * 8);
                        const bf16 *ye = reinterpret_cast<const bf16 *>(&yv);
                        float sacc = 0.f;
#pragma unroll
                        for (int e = 0; e < 8; ++e) sacc += __bfloat162float(ye[e]) * wf[e];
                        acc[m] += sacc;
                    }
                }
#pragma unroll
                for (int m = 0; m < IMB; ++m) {
                    float v = acc[m];
                    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
                    if (lane == 0) fo[m * kOutPad + j] = v + __ldg(W.b[3] + j);
                }
            }
            __syncthreads();
            if (tid < IMB) {
                const int i = g * IMB + tid;
                float o[kOutPad];
                for (int j = 0; j < kOutPad; ++j) o[j] = j < kOut ? fo[tid * kOutPad + j] : 0.f;
                if (i < n) {
                    if (out)
                        for (int j = 0; j < kOutPad; ++j) out[(size_t)i * kOutPad + j] = o[j];
                    if (hints) hints[i] = make_hint(o, conf, lim);
                }
            }
        }
        __syncthreads();
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

// Measured integer-instruction rate of the device: the denominator of the
// analysis kernels' integer-op roofline.
//
// Every thread runs independent chains of 32-bit integer instructions, in four
// mixes of the kinds the analysis loop is made of (sums of absolute
// differences, transforms, quantisation, addresses): multiply-adds with
// three-input adds, three-input adds with logic ops, multiply-adds alone, and
// packed absolute differences with adds.  Enough warps per SM keep the pipes
// issuing; the best mix is the rate the SMs can retire.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kChains = 8;
constexpr int kOpsPerIter = 2 * kChains;   // two instructions per chain per iteration

template <int MIX>
__global__ void __launch_bounds__(256) int_rate_kernel(uint32_t *sink, int iters, uint32_t seed) {
    uint32_t a[kChains], c[kChains];
    const uint32_t m = (blockIdx.x * 2u + 1u) | seed, k = threadIdx.x + seed;
#pragma unroll
    for (int j = 0; j < kChains; ++j) { a[j] = threadIdx.x * (j + 3u) + seed; c[j] = a[j] ^ (0x9e37u * j); }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) {
            if (MIX == 0) {          // multiply-add, three-input add
                a[j] = a[j] * m + c[j];
                c[j] = c[j] + a[j] + k;
            } else if (MIX == 1) {   // three-input add, logic
                a[j] = a[j] + c[j] + k;
                c[j] = (c[j] ^ a[j]) | m;
            } else if (MIX == 2) {   // multiply-add only
                a[j] = a[j] * m + c[j];
                c[j] = c[j] * k + a[j];
            } else {                 // packed absolute difference, add
                a[j] = __vabsdiffu4(a[j], c[j]) + m;
                c[j] = c[j] + a[j] + k;
            }
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) r ^= a[j] ^ c[j];
    if (r == 0x7f4a7c15u) sink[threadIdx.x] = r;   // keeps the chains live; practically never taken
}

}  // namespace

// 32-bit integer lane-operations per second on `device` (best of `reps`
// timed launches over every SM); 0 on error.
extern "C" double fdvb_measure_int_rate(int device, int reps) {
    if (cudaSetDevice(device) != cudaSuccess) return 0.0;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    uint32_t *sink = nullptr;
    if (nsm <= 0 || cudaMalloc(&sink, 256 * sizeof(uint32_t)) != cudaSuccess) return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int grid = nsm * 8, block = 256, iters = 1 << 14;
    void (*const kern[4])(uint32_t *, int, uint32_t) = {int_rate_kernel<0>, int_rate_kernel<1>, int_rate_kernel<2>,
                                                        int_rate_kernel<3>};
    double best = 0.0;
    for (int mix = 0; mix < 4; ++mix) {
        kern[mix]<<<grid, block>>>(sink, iters / 16, 1u);   // warm-up
        for (int r = 0; r < (reps < 1 ? 1 : reps); ++r) {
            cudaEventRecord(e0);
            kern[mix]<<<grid, block>>>(sink, iters, (uint32_t)r + 2u);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) { best = 0.0; mix = 4; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double ops = (double)grid * block * iters * kOpsPerIter;
            if (ms > 0.f && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return cudaGetLastError() == cudaSuccess ? best : 0.0;
}

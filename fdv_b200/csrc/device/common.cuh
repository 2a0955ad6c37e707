// Shared device-side definitions of the fdv analysis kernels (sm_100a).
//
// All pixel work is 8/16/32-bit integer arithmetic; the rate-distortion
// decisions are IEEE double comparisons evaluated with explicitly rounded
// intrinsics so that no fused multiply-add can change a tie
// (J = D + lambda * bits, fdv.h:2527, :4043, :5390, :5866, :5932).
#pragma once
#include <cstdint>

#define FDVB_FULL 0xffffffffu

namespace fdvb {

// ----------------------------------------------------------- constants --
// H.264 4x4 forward multipliers and dequant rescale by [qp % 6][class]
// (fdv.h:2405-2421), the 4x4 and 8x8 zigzag scans (fdv.h:1699, :2153).
__constant__ int c_MF[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                               {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559}};
__constant__ int c_DQV[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16},
                                {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
// Lookups indexed by lane go through registers or L1, never the constant
// cache (which serialises different addresses within a warp): the 4x4 scans
// are nibble-packed immediates, the 8x8 scan and basis live in global memory.
constexpr int kZZ4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
constexpr int kIZZ4[16] = {0, 1, 5, 6, 2, 4, 7, 12, 3, 8, 11, 13, 9, 10, 14, 15};
constexpr unsigned long long nib_pack(const int (&a)[16]) {
    unsigned long long v = 0;
    for (int i = 15; i >= 0; --i) v = (v << 4) | (unsigned long long)a[i];
    return v;
}
constexpr unsigned long long kZZ4P = nib_pack(kZZ4), kIZZ4P = nib_pack(kIZZ4);
__device__ __forceinline__ int zz4(int k) { return (int)((kZZ4P >> (4 * k)) & 15u); }
__device__ __forceinline__ int izz4(int k) { return (int)((kIZZ4P >> (4 * k)) & 15u); }
__device__ const uint8_t g_ZZ8[64] = {
     0,  1,  8, 16,  9,  2,  3, 10, 17, 24, 32, 25, 18, 11,  4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13,  6,  7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
// 8x8 DCT basis (and its transpose) and quantiser steps, computed on the
// host (fdvb_c8_tables).
__device__ int32_t g_C8[64], g_C8T[64];
__constant__ int32_t c_QSTEP8[52];
__device__ __forceinline__ int32_t c8(int i) { return __ldg(&g_C8[i]); }
__device__ __forceinline__ int32_t c8t(int i) { return __ldg(&g_C8T[i]); }
__device__ __forceinline__ int zz8(int k) { return __ldg(&g_ZZ8[k]); }

// Cost constants (fdv.h:3350-3355).
constexpr int kBitsMode = 3, kBitsFlag = 2;

// ------------------------------------------------------------- helpers --
__device__ __forceinline__ int clipb(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
__device__ __forceinline__ uint32_t zz_enc(int v) { return ((uint32_t)v << 1) ^ (uint32_t)(v >> 31); }
__device__ __forceinline__ int leb_size(uint32_t u) { return u < 0x80u ? 1 : (u < 0x4000u ? 2 : (u < 0x200000u ? 3 : (u < 0x10000000u ? 4 : 5))); }
// 2 * floor(log2(v + 1)) + 1: the exp-Golomb length the reference charges (fdv.h:2487).
__device__ __forceinline__ int bits_val(uint32_t v) { return 2 * (31 - __clz(v + 1u)) + 1; }
__device__ __forceinline__ int leb_write(uint8_t *b, uint32_t u) {
    int n = 0;
    while (u >= 0x80u) { b[n++] = (uint8_t)(u | 0x80u); u >>= 7; }
    b[n++] = (uint8_t)u;
    return n;
}
// Exclusive prefix over the lanes selected by `mask` below this one, and the
// total over them, of v in 0..7 (a level's byte count), from three ballots:
// no chain of shuffles.
__device__ __forceinline__ int ballot_prefix(int v, int lane, unsigned mask, int &total) {
    const unsigned b0 = __ballot_sync(0xffffffffu, v & 1) & mask, b1 = __ballot_sync(0xffffffffu, v & 2) & mask,
                   b2 = __ballot_sync(0xffffffffu, v & 4) & mask;
    const unsigned lt = (1u << lane) - 1u;
    total = __popc(b0) + 2 * __popc(b1) + 4 * __popc(b2);
    return __popc(b0 & lt) + 2 * __popc(b1 & lt) + 4 * __popc(b2 & lt);
}
// The len-byte LEB128 form of u (len = leb_size(u), or 0: nothing) at dst,
// without lane-dependent branches for len <= 3 (every 16-bit level): the
// stores a lane does not need go to its own byte of junk.
__device__ __forceinline__ void leb_put(uint8_t *dst, uint8_t *junk, uint32_t u, int len) {
    *(len > 0 ? dst : junk) = (uint8_t)(len > 1 ? (u | 0x80u) : u);
    *(len > 1 ? dst + 1 : junk) = (uint8_t)(len > 2 ? ((u >> 7) | 0x80u) : (u >> 7));
    *(len > 2 ? dst + 2 : junk) = (uint8_t)(len > 3 ? ((u >> 14) | 0x80u) : (u >> 14));
    if (__any_sync(0xffffffffu, len > 3) && len > 3) leb_write(dst, u);
}
__device__ __forceinline__ int pos_class(int idx) {
    int i = idx >> 2, j = idx & 3;
    if (!(i & 1) && !(j & 1)) return 0;
    if ((i & 1) && (j & 1)) return 1;
    return 2;
}
// J = D + lambda * bits with the same two roundings as the reference's C.
__device__ __forceinline__ double rd_cost(double D, double lambda, int bits) {
    return __dadd_rn(D, __dmul_rn(lambda, (double)bits));
}

// ------------------------------------------------------------ 4x4 core --
// Output m (0..3) of the 1-D forward / inverse butterflies.  Lanes of a warp
// take different m, so the outputs are selected arithmetically: a chain of
// conditionals on m compiles to divergent branches, several times slower.
//   forward: m 0 a0 + a1, 1 2 a3 + a2, 2 a0 - a1, 3 a3 - 2 a2
//   inverse: m 0 z0 + z3, 1 z1 + z2, 2 z1 - z2, 3 z0 - z3
__device__ __forceinline__ int fwd1(int x0, int x1, int x2, int x3, int m) {
    const int a0 = x0 + x3, a3 = x0 - x3, a1 = x1 + x2, a2 = x1 - x2;
    const int sb = (m >> 1) & 1;
    const int ev = a0 + ((a1 ^ -sb) + sb);
    const int od = a3 * (2 - sb) + (((a2 * (1 + sb)) ^ -sb) + sb);
    return ev + ((od - ev) & -(m & 1));
}
__device__ __forceinline__ int inv1(int d0, int d1, int d2, int d3, int m) {
    const int z0 = d0 + d2, z1 = d0 - d2, z2 = (d1 >> 1) - d3, z3 = d1 + (d3 >> 1);
    const int s0 = ((m + 1) >> 1) & 1, sg = (m >> 1) & 1;
    const int A = z0 + ((z1 - z0) & -s0), B = z3 + ((z2 - z3) & -s0);
    return A + ((B ^ -sg) + sg);
}
// Whole-block inverse on one thread (used by RDOQ candidate lanes).
__device__ __forceinline__ void idct4_thread(const int d[16], int r[16]) {
    int t[16];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int z0 = d[i * 4 + 0] + d[i * 4 + 2], z1 = d[i * 4 + 0] - d[i * 4 + 2];
        int z2 = (d[i * 4 + 1] >> 1) - d[i * 4 + 3], z3 = d[i * 4 + 1] + (d[i * 4 + 3] >> 1);
        t[i * 4 + 0] = z0 + z3; t[i * 4 + 1] = z1 + z2; t[i * 4 + 2] = z1 - z2; t[i * 4 + 3] = z0 - z3;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int z0 = t[0 * 4 + j] + t[2 * 4 + j], z1 = t[0 * 4 + j] - t[2 * 4 + j];
        int z2 = (t[1 * 4 + j] >> 1) - t[3 * 4 + j], z3 = t[1 * 4 + j] + (t[3 * 4 + j] >> 1);
        r[0 * 4 + j] = (int16_t)((z0 + z3 + 32) >> 6);
        r[1 * 4 + j] = (int16_t)((z1 + z2 + 32) >> 6);
        r[2 * 4 + j] = (int16_t)((z1 - z2 + 32) >> 6);
        r[3 * 4 + j] = (int16_t)((z0 - z3 + 32) >> 6);
    }
}
__device__ __forceinline__ int quant4(int w, int idx, int qp) {
    int m = qp % 6, qbits = 15 + qp / 6, f = (1 << qbits) / 3;
    int sign = w < 0 ? -1 : 1;
    long long aw = (long long)(w < 0 ? -w : w);
    return (int16_t)(sign * (int)((aw * c_MF[m][pos_class(idx)] + f) >> qbits));
}
__device__ __forceinline__ int dequant4(int lv, int idx, int qp) {
    return (int32_t)(lv * c_DQV[qp % 6][pos_class(idx)]) * (int32_t)(1 << (qp / 6));
}

// ---------------------------------------------------- device structures --
// A reference frame: luma integer plane G and its three half-pel planes
// (H.264 b, h, j -- fdv.h:2949-2959), plus the two chroma planes, all padded
// by `border` replicated samples; pointers address pixel (0,0).
struct RefPlanes {
    const uint8_t *G, *B, *H, *J, *U, *V;
    int ys, cs;          // luma / chroma strides
};

// The same planes as a reference being written (post.cuh).
struct OutPlanes {
    uint8_t *G, *B, *H, *J, *U, *V;
    int ys, cs;
};

// Per-macroblock motion kept for merge candidates (fdv.h:5680) plus the mode.
struct MBInfo {
    int16_t x, y;
    uint8_t ref, inter, mode, pad;
};

// Stream capacities of one macroblock's output slot.  Structure streams are
// indexed by model exactly as the frame blob carries them (fdv.h:4170,
// :6198-6210): mode contexts 0-3, reference, MV x, MV y, intra sub-mode, merge
// index; then the seven coefficient streams.  Level bytes are bounded by two
// LEB bytes per coefficient (|level| < 8192 for 8-bit input); three are
// reserved and overruns are detected and reported.
constexpr int kSlotCap[16] = {1, 1, 1, 1, 1, 8, 8, 1, 1, 16, 768, 8, 1152, 8, 8, 384};
constexpr int slot_off(int k) {
    int o = 0;
    for (int i = 0; i < k; ++i) o += kSlotCap[i];
    return o;
}
__constant__ int c_SlotCap[16] = {1, 1, 1, 1, 1, 8, 8, 1, 1, 16, 768, 8, 1152, 8, 8, 384};
constexpr int kSlotData = slot_off(16);                       // 2375
constexpr int kSlotBytes = ((kSlotData + 32 + 127) / 128) * 128;  // lengths + data, 128-aligned
__constant__ int c_SlotOff[17] = {slot_off(0), slot_off(1), slot_off(2), slot_off(3), slot_off(4),
                                  slot_off(5), slot_off(6), slot_off(7), slot_off(8), slot_off(9),
                                  slot_off(10), slot_off(11), slot_off(12), slot_off(13), slot_off(14),
                                  slot_off(15), slot_off(16)};
// Slot layout: uint16 len[16] at offset 0, data from offset 32.
__device__ __forceinline__ uint16_t *slot_len(uint8_t *slot) { return reinterpret_cast<uint16_t *>(slot); }
__device__ __forceinline__ uint8_t *slot_data(uint8_t *slot, int k) { return slot + 32 + c_SlotOff[k]; }

// Error bits reported through the engine's status word.
enum : unsigned {
    kErrWaitTimeout = 1u,    // a wavefront wait gave up
    kErrSlotOverflow = 2u,   // a symbol stream exceeded its per-block slot
    kErrMmaTimeout = 4u,     // a tensor-core completion wait gave up
    kErrOutCap = 8u,         // the compacted streams do not fit the output buffer
};

// The host-side text of a status word (the first error bit that is set).
inline const char *status_text(unsigned e) {
    return (e & kErrWaitTimeout)  ? "wavefront wait timed out"
           : (e & kErrMmaTimeout) ? "tensor-core completion wait timed out"
           : (e & kErrOutCap)     ? "output buffer too small for the symbol streams"
                                  : "symbol slot overflow";
}

// Bounded spin until *flag >= need.  Gives up after `limit_ns` of wall time
// (device global timer) or when another block has already raised an error.
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool wait_at_least(const int *flag, int need, unsigned *err,
                                              unsigned long long limit_ns) {
    if (*(volatile const int *)flag >= need) { __threadfence(); return true; }
    unsigned long long t0 = globaltimer();
    for (;;) {
        if (*(volatile const int *)flag >= need) { __threadfence(); return true; }
        if (*(volatile unsigned *)err) return false;
        if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrWaitTimeout); return false; }
        __nanosleep(64);
    }
}

// Progress flags between blocks with release/acquire at GPU scope (lighter
// than a full fence plus an atomic exchange).  The publisher's block writes
// are ordered before its release by the block barrier that precedes it; the
// waiter's acquire orders its later loads, and the barrier after the wait
// extends that to its block.
__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Bounded wait until *flag >= need: spins without sleeping at first (the
// flag usually arrives within a few microseconds), checks the error word
// every 16 polls, then backs off.
__device__ __forceinline__ bool wait_progress(const int *flag, int need, unsigned *err,
                                              unsigned long long limit_ns) {
    if (ld_acquire_gpu(flag) >= need) return true;
    const unsigned long long t0 = globaltimer();
    for (unsigned i = 1;; ++i) {
        if (ld_acquire_gpu(flag) >= need) return true;
        if (!(i & 15)) {
            if (*(volatile unsigned *)err) return false;
            if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrWaitTimeout); return false; }
        }
        if (i > 256) __nanosleep(64);
    }
}

// 64-bit progress words (count in bits 0-11, a payload above).
__device__ __forceinline__ unsigned long long ld_acquire_gpu64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Waits until the count reaches need; returns the observed word, or ~0ull
// after the limit or when another block has raised an error.
__device__ __forceinline__ unsigned long long wait_count64(const unsigned long long *flag, int need, unsigned *err,
                                                           unsigned long long limit_ns) {
    unsigned long long v = ld_acquire_gpu64(flag);
    if ((int)(v & 0xfffu) >= need) return v;
    const unsigned long long t0 = globaltimer();
    for (unsigned i = 1;; ++i) {
        v = ld_acquire_gpu64(flag);
        if ((int)(v & 0xfffu) >= need) return v;
        if (!(i & 15)) {
            if (*(volatile unsigned *)err) return ~0ull;
            if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrWaitTimeout); return ~0ull; }
        }
        if (i > 256) __nanosleep(64);
    }
}

// A progress word with the count in bits 8 and up (and a payload below):
// waits until the count reaches need and returns the observed word, or -1
// after the limit or when another block has raised an error.
__device__ __forceinline__ int wait_count(const int *flag, int need, unsigned *err, unsigned long long limit_ns) {
    int v = ld_acquire_gpu(flag);
    if ((v >> 8) >= need) return v;
    const unsigned long long t0 = globaltimer();
    for (unsigned i = 1;; ++i) {
        v = ld_acquire_gpu(flag);
        if ((v >> 8) >= need) return v;
        if (!(i & 15)) {
            if (*(volatile unsigned *)err) return -1;
            if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrWaitTimeout); return -1; }
        }
        if (i > 256) __nanosleep(64);
    }
}

}  // namespace fdvb

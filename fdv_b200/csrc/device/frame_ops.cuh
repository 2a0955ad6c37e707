// Per-frame passes around the analysis kernels.
//
//  * refprep: the deblocked reconstruction becomes a reference frame -- the
//    integer plane with its border replicated (load_ref/plane_extend,
//    fdv.h:5183-5193, :1603-1624) and the three H.264 half-pel planes b, h, j
//    (fdv.h:2932-2959), computed once per frame instead of per probe.
//  * deblock: the 8x8-grid edge filter (fdv.h:3491-3501, :3617-3625), edge
//    parallel: every vertical edge of the plane, then every horizontal edge.
//    Within a pass no two edges touch the same sample (edges are 8 apart and a
//    filter reads +-2 and writes +-1 samples), so each pass is data-parallel;
//    only the order of the passes matters.
//  * compact: per-macroblock symbol slots are concatenated, per stream, in
//    raster order -- the order the reference appends them -- directly into
//    host-mapped memory.
#pragma once
#include "common.cuh"
#include "engine_dev.cuh"

namespace fdvb {

struct PrepTask {
    const uint8_t *rec[3];
    uint8_t *G, *B, *H, *J, *U, *V;   // pointers at pixel (0,0)
    int w, h, ys, cs, border;
};

__device__ __forceinline__ int rpx(const uint8_t *p, int w, int h, int x, int y) {
    x = x < 0 ? 0 : (x >= w ? w - 1 : x);
    y = y < 0 ? 0 : (y >= h ? h - 1 : y);
    return p[(size_t)y * w + x];
}
__device__ __forceinline__ int tap6(int a, int b, int c, int d, int e, int f) {
    return a - 5 * b + 20 * c + 20 * d - 5 * e + f;
}
__device__ __forceinline__ int hfr(const uint8_t *p, int w, int h, int x, int y) {
    return tap6(rpx(p, w, h, x - 2, y), rpx(p, w, h, x - 1, y), rpx(p, w, h, x, y),
                rpx(p, w, h, x + 1, y), rpx(p, w, h, x + 2, y), rpx(p, w, h, x + 3, y));
}

// Luma planes.  A block makes a 128 x 16 tile of the padded plane (32 x 8
// threads, 4 adjacent samples per thread and row, stored as one 32-bit word:
// padded widths and row starts are multiples of 4).  The clamped source tile
// with a 2/3-sample halo is staged in shared memory once, then its horizontal
// 6-tap sums; b, h and j come from those.  Grid: x over 128-column tiles, y over
// 16-row tiles, z = task.
constexpr int kRpTW = 128, kRpTH = 16;
__global__ void __launch_bounds__(256) refprep_luma_kernel(const PrepTask *tasks) {
    __shared__ uint8_t S[kRpTH + 5][kRpTW + 8];   // rows y0-2 .. y0+TH+2, columns x0-2 .. x0+TW+2
    __shared__ int16_t Hs[kRpTH + 5][kRpTW];      // 6-tap horizontal sums at x0 .. x0+TW-1
    const PrepTask &T = tasks[blockIdx.z];
    const int B = T.border, pw = T.w + 2 * B, ph = T.h + 2 * B;
    const int px0 = blockIdx.x * kRpTW, py0 = blockIdx.y * kRpTH;
    if (px0 >= pw || py0 >= ph) return;
    const int x0 = px0 - B, y0 = py0 - B, w = T.w, h = T.h;
    const uint8_t *r = T.rec[0];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int k = tid; k < (kRpTH + 5) * (kRpTW + 5); k += 256) {
        const int i = k / (kRpTW + 5), j = k - i * (kRpTW + 5);
        S[i][j] = (uint8_t)rpx(r, w, h, x0 - 2 + j, y0 - 2 + i);
    }
    __syncthreads();
    for (int k = tid; k < (kRpTH + 5) * kRpTW; k += 256) {
        const int i = k / kRpTW, j = k - i * kRpTW;
        Hs[i][j] = (int16_t)tap6(S[i][j], S[i][j + 1], S[i][j + 2], S[i][j + 3], S[i][j + 4], S[i][j + 5]);
    }
    __syncthreads();
    const int tx = threadIdx.x * 4;
    if (px0 + tx >= pw) return;
    for (int rr = threadIdx.y; rr < kRpTH && py0 + rr < ph; rr += 8) {
        uint32_t g = 0, b = 0, hv = 0, jv = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = tx + q;
            const int v = tap6(S[rr][j + 2], S[rr + 1][j + 2], S[rr + 2][j + 2], S[rr + 3][j + 2], S[rr + 4][j + 2],
                               S[rr + 5][j + 2]);
            const int jj = tap6(Hs[rr][j], Hs[rr + 1][j], Hs[rr + 2][j], Hs[rr + 3][j], Hs[rr + 4][j], Hs[rr + 5][j]);
            g |= (uint32_t)S[rr + 2][j + 2] << (8 * q);
            b |= (uint32_t)clipb((Hs[rr + 2][j] + 16) >> 5) << (8 * q);
            hv |= (uint32_t)clipb((v + 16) >> 5) << (8 * q);
            jv |= (uint32_t)clipb((jj + 512) >> 10) << (8 * q);
        }
        const long o = (long)(y0 + rr) * T.ys + x0 + tx;
        *reinterpret_cast<uint32_t *>(T.G + o) = g;
        *reinterpret_cast<uint32_t *>(T.B + o) = b;
        *reinterpret_cast<uint32_t *>(T.H + o) = hv;
        *reinterpret_cast<uint32_t *>(T.J + o) = jv;
    }
}

// Chroma planes: the border replicated, 4 adjacent samples per thread (32 x 8
// threads make a 128 x 8 tile).
__global__ void __launch_bounds__(256) refprep_chroma_kernel(const PrepTask *tasks) {
    const PrepTask &T = tasks[blockIdx.z];
    const int B = T.border, cw = T.w / 2, ch = T.h / 2, pw = cw + 2 * B, ph = ch + 2 * B;
    const int px = (blockIdx.x * blockDim.x + threadIdx.x) * 4, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= pw || py >= ph) return;
    const int x = px - B, y = py - B;
    uint32_t u = 0, v = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        u |= (uint32_t)rpx(T.rec[1], cw, ch, x + q, y) << (8 * q);
        v |= (uint32_t)rpx(T.rec[2], cw, ch, x + q, y) << (8 * q);
    }
    const long o = (long)y * T.cs + x;
    *reinterpret_cast<uint32_t *>(T.U + o) = u;
    *reinterpret_cast<uint32_t *>(T.V + o) = v;
}

// ------------------------------------------------------------- deblock --
struct DbTask {
    uint8_t *p;
    int w, h, qp;
};

__device__ __forceinline__ void filter_edge(uint8_t *a, long step, int alpha, int beta, int tc) {
    int p1 = a[-2 * step], p0 = a[-step], q0 = a[0], q1 = a[step];
    if (abs(p0 - q0) < alpha && abs(p1 - p0) < beta && abs(q1 - q0) < beta) {
        int d = ((q0 - p0) * 4 + (p1 - q1) + 4) >> 3;
        d = d < -tc ? -tc : (d > tc ? tc : d);
        a[-step] = (uint8_t)clipb(p0 + d);
        a[0] = (uint8_t)clipb(q0 - d);
    }
}

// Vertical edges: one thread per (row, edge x = 8, 16, ...).  Grid z = task.
__global__ void deblock_v_kernel(const DbTask *tasks) {
    const DbTask &T = tasks[blockIdx.z];
    const int ne = T.w / 8 - 1;
    if (ne <= 0) return;
    const long n = (long)ne * T.h;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        int y = (int)(i / ne), e = (int)(i % ne);
        filter_edge(T.p + (long)y * T.w + 8 * (e + 1), 1, 6 + T.qp, 2 + T.qp / 4, 1 + T.qp / 10);
    }
}
// Horizontal edges: one thread per (edge y = 8, 16, ..., column).
__global__ void deblock_h_kernel(const DbTask *tasks) {
    const DbTask &T = tasks[blockIdx.z];
    const int ne = T.h / 8 - 1;
    if (ne <= 0) return;
    const long n = (long)ne * T.w;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        int e = (int)(i / T.w), x = (int)(i % T.w);
        filter_edge(T.p + (long)8 * (e + 1) * T.w + x, T.w, 6 + T.qp, 2 + T.qp / 4, 1 + T.qp / 10);
    }
}

// ------------------------------------------------------------- compact --
// Streams of one unit-frame: `nstreams` streams, slot k of block b at
// slots + b*slot_bytes, lengths uint16 at slot start, data at 32 + off[k].
struct CompactTask {
    const uint8_t *slots;
    int nslots, slot_bytes, nstreams;
    const int *off;        // device array [nstreams] of data offsets within a slot
    uint8_t *out;          // host-mapped: uint32 len[nstreams], then the streams back to back
    size_t cap;
    uint32_t *hist;        // host-mapped [nstreams][256] symbol counts, or NULL
    uint8_t *tmp;          // device scratch of cap bytes, the output assembled before it is sent
                           // (NULL: assembled in place, for an output in device memory)
};

// One block per task, 1024 threads: 64 threads per stream scan the slot
// lengths, then each thread copies its chunk of slots into the device scratch
// and counts its bytes into the stream's 256-bin histogram (the entropy
// tail's per-stream counts, fdv.h:6228-6236 and :4899-4905), kept in shared
// memory and written out beside the streams.  The assembled output then
// crosses to host-mapped memory in 16-byte stores, consecutive threads on
// consecutive words (scattered byte stores would each be a bus write).
__global__ void __launch_bounds__(1024) compact_kernel(const CompactTask *tasks, unsigned *err) {
    const CompactTask &T = tasks[blockIdx.x];
    const int tid = threadIdx.x, k = tid >> 6, t = tid & 63;
    __shared__ unsigned s_tot[16][64];
    __shared__ unsigned s_base[17];
    __shared__ unsigned s_hist[16][256];
    for (int i = tid; i < 16 * 256; i += 1024) (&s_hist[0][0])[i] = 0u;
    const int nb = T.nslots, chunk = (nb + 63) / 64, b0 = t * chunk, b1 = min(nb, b0 + chunk);
    unsigned mine = 0;
    if (k < T.nstreams)
        for (int b = b0; b < b1; ++b) mine += reinterpret_cast<const uint16_t *>(T.slots + (size_t)b * T.slot_bytes)[k];
    s_tot[k][t] = mine;
    __syncthreads();
    if (tid < 16) {
        unsigned acc = 0;
        for (int i = 0; i < 64; ++i) { unsigned v = s_tot[tid][i]; s_tot[tid][i] = acc; acc += v; }
        s_base[tid] = acc;  // stream total, turned into a base below
    }
    __syncthreads();
    if (tid == 0) {
        unsigned acc = 0;
        for (int s = 0; s < T.nstreams; ++s) { unsigned tot = s_base[s]; s_base[s] = acc; acc += tot; }
        s_base[16] = acc;
    }
    __syncthreads();
    const size_t hdr = 4 * (size_t)T.nstreams;
    if (hdr + s_base[16] > T.cap) { if (tid == 0) atomicOr(err, kErrOutCap); return; }
    uint8_t *const asmb = T.tmp ? T.tmp : T.out;
    if (tid < T.nstreams) {
        unsigned len = (tid + 1 < T.nstreams ? s_base[tid + 1] : s_base[16]) - s_base[tid];
        reinterpret_cast<unsigned *>(asmb)[tid] = len;
    }
    if (k < T.nstreams) {
        uint8_t *dst = asmb + hdr + s_base[k] + s_tot[k][t];
        for (int b = b0; b < b1; ++b) {
            const uint8_t *slot = T.slots + (size_t)b * T.slot_bytes;
            int n = reinterpret_cast<const uint16_t *>(slot)[k];
            const uint8_t *src = slot + 32 + T.off[k];
            for (int i = 0; i < n; ++i) {
                const uint8_t v = src[i];
                dst[i] = v;
                if (T.hist) atomicAdd(&s_hist[k][v], 1u);
            }
            dst += n;
        }
    }
    __syncthreads();
    const size_t total = hdr + s_base[16];
    if (!T.tmp) {
        // assembled in place
    } else if (((reinterpret_cast<uintptr_t>(T.out) | reinterpret_cast<uintptr_t>(T.tmp)) & 15) == 0) {
        const uint4 *s4 = reinterpret_cast<const uint4 *>(T.tmp);
        uint4 *d4 = reinterpret_cast<uint4 *>(T.out);
        for (size_t i = tid; i < total / 16; i += 1024) d4[i] = s4[i];
        for (size_t i = total / 16 * 16 + tid; i < total; i += 1024) T.out[i] = T.tmp[i];
    } else {
        for (size_t i = tid; i < total; i += 1024) T.out[i] = T.tmp[i];
    }
    if (T.hist)
        for (int i = tid; i < T.nstreams * 256; i += 1024) T.hist[i] = s_hist[i >> 8][i & 255];
}

// The same compaction by a block of NT threads inside another kernel (the
// P-frame wavefront compacts a frame as soon as its last row is done): NT / 16
// threads per stream.  The slots were written by other blocks of the launch,
// which published them with a fence before counting their rows, so they are
// read through L2.  Every thread of the block calls it.
template <int NT> struct CompactScratch {
    unsigned tot[16][NT / 16];
    unsigned base[17];
    unsigned hist[16][256];
};
template <int NT>
__device__ __noinline__ void compact_block(const CompactTask &T, unsigned *err, CompactScratch<NT> &S, int tid) {
    constexpr int TPS = NT / 16;
    const int k = tid / TPS, t = tid % TPS;
    for (int i = tid; i < 16 * 256; i += NT) (&S.hist[0][0])[i] = 0u;
    const int nb = T.nslots, chunk = (nb + TPS - 1) / TPS, b0 = t * chunk, b1 = min(nb, b0 + chunk);
    unsigned mine = 0;
    if (k < T.nstreams)
        for (int b = b0; b < b1; ++b)
            mine += __ldcg(reinterpret_cast<const unsigned short *>(T.slots + (size_t)b * T.slot_bytes) + k);
    S.tot[k][t] = mine;
    __syncthreads();
    if (tid < 16) {
        unsigned acc = 0;
        for (int i = 0; i < TPS; ++i) { const unsigned v = S.tot[tid][i]; S.tot[tid][i] = acc; acc += v; }
        S.base[tid] = acc;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned acc = 0;
        for (int s = 0; s < T.nstreams; ++s) { const unsigned tot = S.base[s]; S.base[s] = acc; acc += tot; }
        S.base[16] = acc;
    }
    __syncthreads();
    const size_t hdr = 4 * (size_t)T.nstreams, total = hdr + S.base[16];
    if (total > T.cap) {
        if (tid == 0) atomicOr(err, kErrOutCap);
        __syncthreads();
        return;
    }
    uint8_t *const asmb = T.tmp ? T.tmp : T.out;
    if (tid < T.nstreams) {
        const unsigned len = (tid + 1 < T.nstreams ? S.base[tid + 1] : S.base[16]) - S.base[tid];
        reinterpret_cast<unsigned *>(asmb)[tid] = len;
    }
    if (k < T.nstreams) {
        uint8_t *dst = asmb + hdr + S.base[k] + S.tot[k][t];
        for (int b = b0; b < b1; ++b) {
            const uint8_t *slot = T.slots + (size_t)b * T.slot_bytes;
            const int n = __ldcg(reinterpret_cast<const unsigned short *>(slot) + k);
            const uint8_t *src = slot + 32 + T.off[k];
            for (int i = 0; i < n; ++i) {
                const uint8_t v = __ldcg(src + i);
                dst[i] = v;
                if (T.hist) atomicAdd(&S.hist[k][v], 1u);
            }
            dst += n;
        }
    }
    __syncthreads();
    if (T.tmp) {
        if (((reinterpret_cast<uintptr_t>(T.out) | reinterpret_cast<uintptr_t>(T.tmp)) & 15) == 0) {
            const uint4 *s4 = reinterpret_cast<const uint4 *>(T.tmp);
            uint4 *d4 = reinterpret_cast<uint4 *>(T.out);
            for (size_t i = tid; i < total / 16; i += NT) d4[i] = s4[i];
            for (size_t i = total / 16 * 16 + tid; i < total; i += NT) T.out[i] = T.tmp[i];
        } else {
            for (size_t i = tid; i < total; i += NT) T.out[i] = T.tmp[i];
        }
    }
    if (T.hist)
        for (int i = tid; i < T.nstreams * 256; i += NT) T.hist[i] = S.hist[i >> 8][i & 255];
    __syncthreads();
}

}  // namespace fdvb

// All analysis kernels in one translation unit, so the constant-memory tables
// (the H.264 quant tables, the scans, and the host-computed 8x8 DCT basis and
// quantiser steps) exist once, plus the host-callable launch wrappers the
// engine uses.
#include <cuda_runtime.h>

#include "common.cuh"
#include "frame_ops.cuh"
#include "iframe.cuh"
#include "pframe.cuh"

namespace fdvb {

void upload_tables(const int32_t c8[64], const int32_t q8[52]) {
    cudaMemcpyToSymbol(c_C8, c8, sizeof(int32_t) * 64);
    cudaMemcpyToSymbol(c_QSTEP8, q8, sizeof(int32_t) * 52);
}

void launch_iframe(const void *planes, const void *tasks, int ntasks, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, cudaStream_t st) {
    static bool attr = false;
    const size_t smem = sizeof(IShared);
    if (!attr) {
        cudaFuncSetAttribute(iframe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    iframe_kernel<<<grid, INT, smem, st>>>(static_cast<const IPlaneDev *>(planes), static_cast<const ITask *>(tasks),
                                           ntasks, ticket, err, wait_ns);
}

void launch_pframe(const UnitDev *units, const RowTask *rows, int nrows, int *ticket, unsigned *err,
                   unsigned long long wait_ns, int grid, cudaStream_t st) {
    pframe_kernel<<<grid, 256, 0, st>>>(units, rows, nrows, ticket, err, wait_ns);
}

void launch_refprep(const void *tasks, int ntasks, int maxw, int maxh, int border, cudaStream_t st) {
    dim3 blk(32, 8);
    dim3 gl((maxw + 2 * border + 31) / 32, (maxh + 2 * border + 7) / 8, ntasks);
    refprep_luma_kernel<<<gl, blk, 0, st>>>(static_cast<const PrepTask *>(tasks));
    dim3 gc((maxw / 2 + 2 * border + 31) / 32, (maxh / 2 + 2 * border + 7) / 8, ntasks);
    refprep_chroma_kernel<<<gc, blk, 0, st>>>(static_cast<const PrepTask *>(tasks));
}

void launch_deblock(const void *tasks, int ntasks, cudaStream_t st) {
    dim3 g(64, 1, ntasks);
    deblock_v_kernel<<<g, 256, 0, st>>>(static_cast<const DbTask *>(tasks));
    deblock_h_kernel<<<g, 256, 0, st>>>(static_cast<const DbTask *>(tasks));
}

void launch_compact(const void *tasks, int ntasks, unsigned *err, cudaStream_t st) {
    compact_kernel<<<ntasks, 1024, 0, st>>>(static_cast<const CompactTask *>(tasks), err);
}

}  // namespace fdvb

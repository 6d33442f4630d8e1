// Translation unit of the chain decoder kernel (k_decode_chains).
//
// It is compiled apart from the rest of libcuopus because its ptxas
// optimisation level differs: at ptxas -O2 and -O3 this kernel decodes
// stereo SILK and hybrid frames with wrong samples (the mid/side to left/right
// stage diverges from libopus on the first stereo frame), while ptxas -O0 and
// -O1, nvcc -G, and the same sources built for the host with g++ (also under
// AddressSanitizer and UndefinedBehaviorSanitizer, and with every local
// variable pattern-initialised) are bit-exact.  The stage in isolation is
// bit-exact at every level, so the fault is in the optimised kernel as a
// whole; build.py compiles this file with -Xptxas -O1 and the GPU parity
// tests hold the kernel to libopus on stereo streams.
#define CUO_DECODE_KERNEL_TU 1
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace cuo {

cudaError_t decode_kernel_occupancy(int block, int width, int *blocks_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_decode_chains, block,
                                                         (size_t)stage_smem_bytes(block, width));
}

cudaError_t decode_kernel_launch(const DecodeArgs &a, int blocks, int block, cudaStream_t st)
{
    DecodeArgs b = a;
    int smem = stage_smem_bytes(block, a.width);
    b.stage = smem > 0;
    k_decode_chains<<<blocks, block, (size_t)smem, st>>>(b);
    return cudaGetLastError();
}

} // namespace cuo

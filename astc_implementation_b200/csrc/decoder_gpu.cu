// ASTC LDR decoding on the GPU (no counterpart in the reference, which has no decoder):
// the same block decoding as the host decoder (decode_block.cuh), so the texels are the
// same, for quality measurement and round-trip checks of large textures without
// copying them back to the host.
//
// k_decode: one CTA of 128 threads per 128 blocks in raster block order.  Each thread
// parses one block into shared memory (block mode, partitioning, endpoints, unquantised
// weights); the CTA's threads then evaluate the texels of its blocks, consecutive threads
// taking consecutive texels, and either write the RGBA8 image or add up the squared
// error per channel against a reference image (warp reduction, then one 64-bit atomic
// per channel and warp).
#include <cuda_runtime.h>

#include "astcb200.h"
#include "decode_block.cuh"
#include "tables.h"

namespace astcb200 {
namespace {

constexpr int kDecodeThreads = 128;

template <bool kError>
__global__ void __launch_bounds__(kDecodeThreads) k_decode(const uint8_t* __restrict__ blocks, int bx, int by, int dx, int dy,
                                                            int nbx, int nblocks, uchar4* __restrict__ out,
                                                            const uchar4* __restrict__ ref, unsigned long long* __restrict__ sse) {
    __shared__ dec::Block kb[kDecodeThreads];
    const int b0 = blockIdx.x * kDecodeThreads;
    const int tid = threadIdx.x;
    if (b0 + tid < nblocks) {
        uint8_t raw[16];
        const uint8_t* src = blocks + (size_t)(b0 + tid) * 16;
#pragma unroll
        for (int i = 0; i < 16; i++) raw[i] = src[i];
        dec::parse_block(raw, bx, by, kb[tid]);
    }
    __syncthreads();
    const int T = bx * by;
    const int nb = min(kDecodeThreads, nblocks - b0);
    unsigned long long acc[4] = {0, 0, 0, 0};
    for (int it = tid; it < nb * T; it += kDecodeThreads) {
        const int k = it / T, t = it - k * T;
        const int x = t % bx, y = t / bx;
        const int blk = b0 + k;
        const int px = (blk % nbx) * bx + x, py = (blk / nbx) * by + y;
        if (px >= dx || py >= dy) continue;
        uint16_t v[4];
        dec::texel16(kb[k], bx, by, x, y, v);
        const uchar4 o = make_uchar4(dec::to_unorm8(v[0]), dec::to_unorm8(v[1]), dec::to_unorm8(v[2]), dec::to_unorm8(v[3]));
        const size_t at = (size_t)py * dx + px;
        if constexpr (kError) {
            const uchar4 r = ref[at];
            const int d0 = (int)o.x - (int)r.x, d1 = (int)o.y - (int)r.y, d2 = (int)o.z - (int)r.z, d3 = (int)o.w - (int)r.w;
            acc[0] += (unsigned long long)(d0 * d0); acc[1] += (unsigned long long)(d1 * d1);
            acc[2] += (unsigned long long)(d2 * d2); acc[3] += (unsigned long long)(d3 * d3);
        } else {
            out[at] = o;
        }
    }
    if constexpr (kError) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            unsigned long long s = acc[c];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
            if ((tid & 31) == 0 && s) atomicAdd(&sse[c], s);
        }
    }
}

// image: RGBA8, 4-byte aligned (uchar4 accesses)
int check_args(uint32_t bx, uint32_t by, uint32_t dx, uint32_t dy, const void* blocks, const void* image) {
    if (!blocks || !image || dx == 0 || dy == 0 || ((uintptr_t)image & 3)) return ASTCB200_BAD_ARG;
    if (!valid_footprint((int)bx, (int)by)) return ASTCB200_INVALID_FOOTPRINT;
    const uint64_t nb = (uint64_t)((dx + bx - 1) / bx) * ((dy + by - 1) / by);
    if (nb > (uint64_t)0x7FFFFFFF) return ASTCB200_BAD_ARG;
    return ASTCB200_OK;
}

}  // namespace
}  // namespace astcb200

using namespace astcb200;

extern "C" {

int astcb200_decode_device(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y, const uint8_t* d_blocks,
                           uint8_t* d_rgba8, void* cuda_stream) {
    const int rc = check_args(block_x, block_y, dim_x, dim_y, d_blocks, d_rgba8);
    if (rc) return rc;
    const int nbx = (int)((dim_x + block_x - 1) / block_x), nby = (int)((dim_y + block_y - 1) / block_y);
    const int nblocks = nbx * nby;
    k_decode<false><<<(nblocks + kDecodeThreads - 1) / kDecodeThreads, kDecodeThreads, 0, (cudaStream_t)cuda_stream>>>(
        d_blocks, (int)block_x, (int)block_y, (int)dim_x, (int)dim_y, nbx, nblocks, reinterpret_cast<uchar4*>(d_rgba8), nullptr,
        nullptr);
    return cudaGetLastError() == cudaSuccess ? ASTCB200_OK : ASTCB200_CUDA_ERROR;
}

int astcb200_decode_error_device(uint32_t block_x, uint32_t block_y, uint32_t dim_x, uint32_t dim_y, const uint8_t* d_blocks,
                                 const uint8_t* d_ref_rgba8, uint64_t* d_sse, void* cuda_stream) {
    int rc = check_args(block_x, block_y, dim_x, dim_y, d_blocks, d_ref_rgba8);
    if (rc) return rc;
    if (!d_sse) return ASTCB200_BAD_ARG;
    const int nbx = (int)((dim_x + block_x - 1) / block_x), nby = (int)((dim_y + block_y - 1) / block_y);
    const int nblocks = nbx * nby;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    if (cudaMemsetAsync(d_sse, 0, 4 * sizeof(uint64_t), s) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    k_decode<true><<<(nblocks + kDecodeThreads - 1) / kDecodeThreads, kDecodeThreads, 0, s>>>(
        d_blocks, (int)block_x, (int)block_y, (int)dim_x, (int)dim_y, nbx, nblocks, nullptr,
        reinterpret_cast<const uchar4*>(d_ref_rgba8), reinterpret_cast<unsigned long long*>(d_sse));
    return cudaGetLastError() == cudaSuccess ? ASTCB200_OK : ASTCB200_CUDA_ERROR;
}

}  // extern "C"

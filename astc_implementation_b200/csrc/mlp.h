// Learned proposal network: shapes, device weights and the launches of its
// inference (tcgen05 tensor cores) and proposal-selection kernels.
//
// The network maps one block's texels, normalised to [0,1] (RGBA8 / 255) and
// rounded to bf16, through two hidden layers of 256 ReLU units to one logit
// per class:
//   [0, 3072)            partitionings: table entry e of P = 2, 3, 4 at (P-2)*1024 + e
//                        (only entries below the footprint's selected count are classes)
//   3072                 the single-partition block
//   [3200 + p*nbm_pad, +nbm)  block modes (trial indices) for P = p + 1 partitions
// padded to a multiple of 128 outputs.  Inputs are padded to a multiple of 16.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace astcb200 {
namespace mlp {

constexpr int kHidden = 256;
constexpr int kPartClasses = 3072;
constexpr int kClassP1 = 3072;
constexpr int kHeadBase = 3200;
constexpr int kTileRows = 128;   // blocks per CTA of the inference kernel
constexpr int kChunkN = 64;      // output columns per layer-3 MMA chunk
constexpr int kOutAlign = 128;   // outputs are padded to a multiple of this

struct Shape {
    int k0, k0p;        // inputs (4 * texels) and padded to a multiple of 16
    int nbm, nbm_pad;   // block-mode classes per head and the head stride
    int nout;           // outputs, padded to a multiple of kOutAlign
};

inline Shape shape_for(int texels, int nbm) {
    Shape s;
    s.k0 = 4 * texels;
    s.k0p = (s.k0 + 15) & ~15;
    s.nbm = nbm;
    s.nbm_pad = (nbm + 31) & ~31;
    s.nout = (kHeadBase + 4 * s.nbm_pad + kOutAlign - 1) / kOutAlign * kOutAlign;
    return s;
}

// Element index of (row n, column k) in the no-swizzle K-major layout the
// tensor core reads: 8x8 core matrices of 128 contiguous bytes, row groups of
// 8 adjacent (128 B apart), 8-column groups rows/8 core matrices apart.
__host__ __device__ inline uint32_t core_index(uint32_t n, uint32_t k, uint32_t rows) {
    return (k >> 3) * (rows >> 3) * 64 + (n >> 3) * 64 + (n & 7) * 8 + (k & 7);
}

// Device copy of one footprint's network (weights bf16 in core_index order;
// layer 3 as nout/kChunkN chunks of kChunkN rows, each in its own core_index order).
struct Net {
    const uint16_t* w1;   // [256 x k0p]
    const uint16_t* w2;   // [256 x 256]
    const uint16_t* w3;   // [nout/128][128 x 256]
    const float* b1;      // [256]
    const float* b2;      // [256]
    const float* b3;      // [nout]
    Shape s;
};

// Selection rule applied to the logits of one block.
struct Select {
    int kmax;          // partitionings proposed at most (<= kMaxProposals)
    float coverage;    // stop proposing once P=1 plus the proposed mass reaches this
    float threshold;   // the block takes the full search when P=1 plus the kmax best mass is below this
    int kbm;           // block modes per partition count in the masks (<= 64)
    float p1_floor;    // with proposals, P = 1 is searched only when its probability reaches this
    int sel[3];        // selected table entries for P = 2, 3, 4 (valid classes)
};

// Output of the selection kernel for one chunk.
struct Routes {
    int* counts;          // [0] pruned blocks, [1] full-search blocks, [2..5] partitioned blocks
                          // of P = 1..4 in pb_list (zeroed before the launch)
    int* pruned;          // [chunk] global block indices taking the proposal search
    int* full;            // [chunk] global block indices taking the full search
    float* full_err;      // [chunk] error of a result already written for full[i] (3e38: none)
    PropPicks* prop;      // [chunk] by position in `pruned`
    uint64_t* masks;      // [chunk][4][kMaskWords] by position in `pruned`
    float* confidence;    // [chunk] by chunk row (P=1 plus kmax-best probability), may be null
    uint32_t* pb_list;    // [4][pb_stride]: position << 5 | slot of every partitioned block to search
    int pb_stride;
};

constexpr int kRouteCounters = 8;  // ints per chunk: routes, then partitioned-block counts, padding

constexpr int kMlpSmemBytes = 200704 + 1024 + 1024;  // operands and staging, barriers, alignment slack

cudaError_t configure_mlp();
// logits[lb * nout + c] for the chunk's blocks lb < a.nblocks (addressing as for the search kernels)
cudaError_t launch_mlp_logits(const KernelArgs& a, const Net& net, float* logits, int* error_flag, cudaStream_t s);
cudaError_t launch_select(const KernelArgs& a, const Net& net, const float* logits, const Select& sel, const Routes& r,
                          cudaStream_t s);

}  // namespace mlp
}  // namespace astcb200

// Learned proposal network: shapes, device weights and the launches of its
// inference (tcgen05 tensor cores) and proposal-selection kernels.
//
// The network maps one block's texels, normalised to [0,1] (RGBA8 / 255) and
// rounded to bf16, through two hidden layers of 256 ReLU units to one logit
// per class:
//   [0, p1)              partitionings: the selected table entries e < sel[P-2] of P = 2, 3, 4
//                        one count after another, entry e of P at part_base[P-2] + e
//   p1                   the single-partition block (p1 = sel[0] + sel[1] + sel[2])
//   [head_base + p*nbm_pad, +nbm)  block modes (trial indices) for P = p + 1 partitions,
//                        head_base = p1 + 1 rounded up to a multiple of 32
// padded to a multiple of 128 outputs.  Inputs are padded to a multiple of 16.  Outside
// the network a partitioning is named (P - 2) << 10 | e (pick_of_class).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace astcb200 {
namespace mlp {

constexpr int kHidden = 256;
constexpr int kTileRows = 128;   // blocks per CTA of the inference kernel
constexpr int kChunkN = 64;      // output columns per layer-3 MMA chunk
constexpr int kOutAlign = 128;   // outputs are padded to a multiple of this

struct Shape {
    int k0, k0p;        // inputs (4 * texels) and padded to a multiple of 16
    int nbm, nbm_pad;   // block-mode classes per head and the head stride
    int sel[3];         // selected table entries of P = 2, 3, 4
    int part_base[3];   // their first classes
    int p1;             // the single-partition class
    int head_base;      // the first block-mode class
    int nout;           // outputs, padded to a multiple of kOutAlign
};

// sel3: the footprint's selected table entries of P = 2, 3, 4 (TableLayout::count_selected[1..3])
inline Shape shape_for(int texels, int nbm, const uint32_t* sel3) {
    Shape s;
    s.k0 = 4 * texels;
    s.k0p = (s.k0 + 15) & ~15;
    s.nbm = nbm;
    s.nbm_pad = (nbm + 31) & ~31;
    int o = 0;
    for (int i = 0; i < 3; i++) { s.sel[i] = (int)sel3[i]; s.part_base[i] = o; o += s.sel[i]; }
    s.p1 = o;
    s.head_base = (s.p1 + 1 + 31) & ~31;
    s.nout = (s.head_base + 4 * s.nbm_pad + kOutAlign - 1) / kOutAlign * kOutAlign;
    return s;
}

// The partitioning of class c < p1 as (P - 2) << 10 | table entry.
__host__ __device__ inline int pick_of_class(const Shape& s, int c) {
    const int q = c >= s.part_base[2] ? 2 : c >= s.part_base[1] ? 1 : 0;
    return (q << 10) | (c - s.part_base[q]);
}
// Block-mode head (0..3 for P = 1..4) of partition class c <= p1.
__host__ __device__ inline int head_of_class(const Shape& s, int c) {
    return c == s.p1 ? 0 : 1 + (c >= s.part_base[2] ? 2 : c >= s.part_base[1] ? 1 : 0);
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
};

// Output of the selection kernel for one chunk.
struct Routes {
    int* counts;          // [0] pruned blocks, [1] full-search blocks, [2..5] partitioned blocks
                          // of P = 1..4 in pb_list, [6] refinement-tail entries of the proposal
                          // pass (zeroed before the launch)
    int* pruned;          // [chunk] global block indices taking the proposal search
    int* full;            // [chunk] global block indices taking the full search
    float* full_err;      // [chunk] error of a result already written for full[i] (3e38: none)
    PropPicks* prop;      // [chunk] by position in `pruned`
    uint64_t* masks;      // [chunk][4][kMaskWords] by position in `pruned`
    float* confidence;    // [chunk] by chunk row (P=1 plus kmax-best probability), may be null
    uint32_t* pb_list;    // [4][pb_stride]: position << 5 | slot of every partitioned block to search
    int pb_stride;
};

constexpr int kRouteCounters = 8;  // ints per chunk: routes, partitioned-block counts, refinement-tail entries and claims
// Textures of fewer texels take the (reference's) full search even with a network: their
// blocks are mostly edge-clamped copies of a few texels, unlike what the networks learned
// from, and searching them fully costs next to nothing.
constexpr int kMinProposalTexels = 1024;

constexpr int kMlpSmemBytes = 200704 + 1024 + 1024;  // operands and staging, barriers, alignment slack

cudaError_t configure_mlp();
// logits[lb * nout + c] for the chunk's blocks lb < a.nblocks (addressing as for the search kernels)
cudaError_t launch_mlp_logits(const KernelArgs& a, const Net& net, float* logits, int* error_flag, cudaStream_t s);
cudaError_t launch_select(const KernelArgs& a, const Net& net, const float* logits, const Select& sel, const Routes& r,
                          cudaStream_t s);

}  // namespace mlp
}  // namespace astcb200
